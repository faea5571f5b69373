// ice_fam.cuh -- the launcher of one family's RK stage, templated on its closure and Riemann
// solver; each closure's translation unit (ice_fam_mk.cu, ice_fam_ig.cu, ice_fam_ag.cu)
// instantiates its own, so the heavy FP64 kernels compile in parallel.
#pragma once
#include "ice_kernels.cuh"

namespace ice {

inline size_t stage_slots(int TX, int TY, int TZ) {
  size_t sx = (size_t)(TX + 1) * TY * TZ;
  size_t sy = TY > 1 ? (size_t)TX * (TY + 1) * TZ : 0;
  size_t sz = TZ > 1 ? (size_t)TX * TY * (TZ + 1) : 0;
  return std::max(sx, std::max(sy, sz));
}

template <int CL, int RS>
void launch_family_t(const LaunchArgs& a) {
  constexpr int nc = NC<CL>::v;
  cudaStream_t s = a.s;
  auto tick = [&](int cls) { if (a.tick) a.tick(a.tick_ctx, cls, s); };
  auto grid = [](long long n, int t) { return (unsigned)((n + t - 1) / t); };
  if (a.nrec > 0) {
    k_ghost1<CL><<<grid(a.nrec, 128), 128, 0, s>>>(a.G, a.F, a.recs, a.nrec);
    k_ghost2<CL><<<grid(a.nrec, 128), 128, 0, s>>>(a.G, a.F, a.recs, a.nrec);
    tick(KC_GHOST);
  }
  if (a.sd) {
    k_beta<<<grid(a.G.NI, 256), 256, 0, s>>>(a.G, a.F);
    tick(KC_BETA);
  }
  if (a.nown > 0) k_conn<CL, RS><<<grid(a.nown, 64), 64, 0, s>>>(a.G, a.F, a.recs, a.own, a.nown, a.st);
  if (a.nbc > 0) k_bound<CL, RS><<<grid(a.nbc, 64), 64, 0, s>>>(a.G, a.F, a.recs, a.bfirst, a.blist, a.nbc, a.st);
  if (a.nown > 0 || a.nbc > 0) tick(KC_BOUND);
  size_t sh = sizeof(double) * nc * stage_slots(a.TX, a.TY, a.TZ);
  if (!a.irs) {
    if (a.precision == ICE_PREC_FP32FLUX)
      k_stage<CL, RS, false, float><<<a.ntile, 256, sh, s>>>(a.G, a.F, a.tiles, a.ndir, a.TX, a.TY, a.TZ, a.st);
    else
      k_stage<CL, RS, false, double><<<a.ntile, 256, sh, s>>>(a.G, a.F, a.tiles, a.ndir, a.TX, a.TY, a.TZ, a.st);
    tick(KC_STAGE);
    return;
  }
  k_stage<CL, RS, true, double><<<a.ntile, 256, sh, s>>>(a.G, a.F, a.tiles, a.ndir, a.TX, a.TY, a.TZ, a.st);
  tick(KC_STAGE);
  // two Jacobi sweeps per direction; each direction smooths the residual the last one left
  const long long NI = a.G.NI;
  for (int d = 0; d < a.ndir; ++d) {
    k_irs<<<grid(NI, 256), 256, 0, s>>>(a.G, nc, a.resid, a.resid, a.resid2, d, a.irs_beta);
    k_irs<<<grid(NI, 256), 256, 0, s>>>(a.G, nc, a.resid, a.resid2, a.resid3, d, a.irs_beta);
    cudaMemcpyAsync(a.resid, a.resid3, sizeof(double) * nc * NI, cudaMemcpyDeviceToDevice, s);
  }
  tick(KC_IRS);
  k_update<CL><<<grid(NI, 256), 256, 0, s>>>(a.G, a.F, a.st);
  tick(KC_STAGE);
}

}  // namespace ice
