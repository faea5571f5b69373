// The IG family's stage kernels, FP32 reconstruction, fluxes and sources (the chosen form).
#include "ice_stage.cuh"
namespace ice {
void launch_stage_ig_f32(const LaunchArgs& a, bool write_r) { launch_stage_t<IG, float>(a, write_r); }
void launch_source_ig_f32(const LaunchArgs& a) { launch_source_t<IG, float>(a); }
void launch_bound_ig_f32(const LaunchArgs& a) { launch_bound_t<IG, float>(a); }
void launch_pack_beta_ig_f32(const LaunchArgs& a, const int4* e, int n, double* out) {
  launch_pack_beta_t<float>(a, e, n, out);
}
}  // namespace ice
