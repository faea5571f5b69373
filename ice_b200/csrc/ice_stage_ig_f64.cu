// The IG family's stage kernels, FP64 (plain form and the IRS residual).
#include "ice_stage.cuh"
namespace ice {
void launch_stage_ig_f64(const LaunchArgs& a, bool write_r) { launch_stage_t<IG, double>(a, write_r); }
void launch_source_ig_f64(const LaunchArgs& a) { launch_source_t<IG, double>(a); }
void launch_bound_ig_f64(const LaunchArgs& a) { launch_bound_t<IG, double>(a); }
void launch_pack_beta_ig_f64(const LaunchArgs& a, const int4* e, int n, double* out) {
  launch_pack_beta_t<double>(a, e, n, out);
}
}  // namespace ice
