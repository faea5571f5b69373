// The MK family's stage kernels, FP64 (plain form and the IRS residual).
#include "ice_stage.cuh"
namespace ice {
void launch_stage_mk_f64(const LaunchArgs& a, bool write_r) { launch_stage_t<MK, double>(a, write_r); }
void launch_source_mk_f64(const LaunchArgs& a) { launch_source_t<MK, double>(a); }
void launch_bound_mk_f64(const LaunchArgs& a) { launch_bound_t<MK, double>(a); }
void launch_pack_beta_mk_f64(const LaunchArgs& a, const int4* e, int n, double* out) {
  launch_pack_beta_t<double>(a, e, n, out);
}
}  // namespace ice
