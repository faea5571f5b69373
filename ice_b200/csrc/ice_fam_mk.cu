// The MK family's stage kernels (Saurel, Rusanov and HLLE fluxes).
#include "ice_fam.cuh"
namespace ice {
void launch_family_mk(const LaunchArgs& a) {
  if (a.F.riemann == ICE_RIEMANN_SAUREL) launch_family_t<MK, ICE_RIEMANN_SAUREL>(a);
  else if (a.F.riemann == ICE_RIEMANN_HLLE) launch_family_t<MK, ICE_RIEMANN_HLLE>(a);
  else launch_family_t<MK, ICE_RIEMANN_RUSANOV>(a);
}
}  // namespace ice
