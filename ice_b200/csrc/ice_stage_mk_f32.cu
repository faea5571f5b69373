// The MK family's stage kernels, FP32 reconstruction, fluxes and sources (the chosen form).
#include "ice_stage.cuh"
namespace ice {
void launch_stage_mk_f32(const LaunchArgs& a, bool write_r) { launch_stage_t<MK, float>(a, write_r); }
void launch_source_mk_f32(const LaunchArgs& a) { launch_source_t<MK, float>(a); }
void launch_bound_mk_f32(const LaunchArgs& a) { launch_bound_t<MK, float>(a); }
void launch_pack_beta_mk_f32(const LaunchArgs& a, const int4* e, int n, double* out) {
  launch_pack_beta_t<float>(a, e, n, out);
}
}  // namespace ice
