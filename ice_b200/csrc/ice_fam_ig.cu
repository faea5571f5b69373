// The IG family's stage kernels (Rusanov and HLLE fluxes).
#include "ice_fam.cuh"
namespace ice {
void launch_family_ig(const LaunchArgs& a) {
  if (a.F.riemann == ICE_RIEMANN_HLLE) launch_family_t<IG, ICE_RIEMANN_HLLE>(a);
  else launch_family_t<IG, ICE_RIEMANN_RUSANOV>(a);
}
}  // namespace ice
