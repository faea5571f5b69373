// The AG family's stage kernels, FP32 reconstruction, fluxes and sources (the chosen form).
#include "ice_stage.cuh"
namespace ice {
void launch_stage_ag_f32(const LaunchArgs& a, bool write_r) { launch_stage_t<AG, float>(a, write_r); }
void launch_source_ag_f32(const LaunchArgs& a) { launch_source_t<AG, float>(a); }
void launch_bound_ag_f32(const LaunchArgs& a) { launch_bound_t<AG, float>(a); }
void launch_pack_beta_ag_f32(const LaunchArgs& a, const int4* e, int n, double* out) {
  launch_pack_beta_t<float>(a, e, n, out);
}
}  // namespace ice
