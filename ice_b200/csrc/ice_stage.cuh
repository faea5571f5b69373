// ice_stage.cuh -- the launcher of the stage kernel of one closure and precision: the Riemann
// solver and the limiter are compile-time parameters of the kernel (van Leer and minmod
// specialised, every other limiter through the run-time switch).
#pragma once
#include "ice_kernels.cuh"
#include "ice_stage3.cuh"

namespace ice {

// 2-D and 3-D runs: the staged kernel (ice_stage3.cuh); 1-D runs: the plane kernel of ice_kernels.cuh
// (one tile of 256 cells per CTA) with the source in its own kernel before it.
template <int CL, int RS, int LIM, typename R>
void launch_stage_k(const LaunchArgs& a, bool write_r) {
  constexpr int nc = NC<CL>::v;
  if (a.ntile3 > 0) {
    constexpr size_t sh = StageSmem<CL, R>::bytes;
    static bool attr3 = false;
    if (!attr3) {
      cudaFuncSetAttribute(k_stage3<CL, RS, LIM, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
      attr3 = true;
    }
    k_stage3<CL, RS, LIM, R><<<a.ntile3, Shape<CL>::NT, sh, a.s>>>(a.G, a.F, a.maps, a.tiles3, write_r ? 1 : 0, a.st);
    return;
  }
  const size_t sh = sizeof(double) * 4 * nc * (size_t)a.TX * a.TY;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_stage<CL, RS, LIM_ANY, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 98304);
    attr = true;
  }
  k_stage<CL, RS, LIM_ANY, R><<<a.ntile, a.TX * a.TY, sh, a.s>>>(a.G, a.F, a.tiles, a.TX, a.TY, a.KZ,
                                                                 write_r ? 1 : 0, a.st);
}

template <int CL, int RS, typename R>
void launch_stage_l(const LaunchArgs& a, bool write_r) {
  if (a.F.limiter == ICE_LIM_VANLEER) launch_stage_k<CL, RS, ICE_LIM_VANLEER, R>(a, write_r);
  else if (a.F.limiter == ICE_LIM_MINMOD) launch_stage_k<CL, RS, ICE_LIM_MINMOD, R>(a, write_r);
  else launch_stage_k<CL, RS, LIM_ANY, R>(a, write_r);
}

// connection-face fluxes by their owners, then every boundary cell's records in face order
template <int CL, int RS, int LIM, typename R>
void launch_bound_k(const LaunchArgs& a) {
  auto grid = [](long long n, int t) { return (unsigned)((n + t - 1) / t); };
  if (a.nown > 0) k_conn<CL, RS, LIM, R><<<grid(a.nown, 128), 128, 0, a.s>>>(a.G, a.F, a.recs, a.own, a.nown, a.st);
  if (a.xchg) a.xchg(a, ICE_GPU_HALO_FLUX);    // connection fluxes to the partners another rank steps
  if (a.nbc > 0)
    k_bound<CL, RS, LIM, R><<<grid(a.nbc, 128), 128, 0, a.s>>>(a.G, a.F, a.recs, a.bfirst, a.blist, a.bperm, a.nbc, a.st);
}

template <int CL, int RS, typename R>
void launch_bound_l(const LaunchArgs& a) {
  if (a.F.limiter == ICE_LIM_VANLEER) launch_bound_k<CL, RS, ICE_LIM_VANLEER, R>(a);
  else if (a.F.limiter == ICE_LIM_MINMOD) launch_bound_k<CL, RS, ICE_LIM_MINMOD, R>(a);
  else launch_bound_k<CL, RS, LIM_ANY, R>(a);
}

template <int CL, typename R>
void launch_bound_t(const LaunchArgs& a) {
  if constexpr (CL == MK) {
    if (a.F.riemann == ICE_RIEMANN_SAUREL) { launch_bound_l<CL, ICE_RIEMANN_SAUREL, R>(a); return; }
  }
  if (a.F.riemann == ICE_RIEMANN_HLLE) launch_bound_l<CL, ICE_RIEMANN_HLLE, R>(a);
  else launch_bound_l<CL, ICE_RIEMANN_RUSANOV, R>(a);
}

template <typename R>
void launch_pack_beta_t(const LaunchArgs& a, const int4* e, int n, double* out) {
  k_pack_beta<R><<<(unsigned)((n + 127) / 128), 128, 0, a.s>>>(a.G, a.F, e, n, out);
}

template <int CL, typename R>
void launch_source_t(const LaunchArgs& a) {
  k_source<CL, R><<<(unsigned)((a.G.NI + 255) / 256), 256, 0, a.s>>>(a.G, a.F);
}

template <int CL, typename R>
void launch_stage_t(const LaunchArgs& a, bool write_r) {
  if constexpr (CL == MK) {
    if (a.F.riemann == ICE_RIEMANN_SAUREL) { launch_stage_l<CL, ICE_RIEMANN_SAUREL, R>(a, write_r); return; }
  }
  if (a.F.riemann == ICE_RIEMANN_HLLE) launch_stage_l<CL, ICE_RIEMANN_HLLE, R>(a, write_r);
  else launch_stage_l<CL, ICE_RIEMANN_RUSANOV, R>(a, write_r);
}

}  // namespace ice
