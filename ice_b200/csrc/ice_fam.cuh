// ice_fam.cuh -- the launcher of one family's RK stage, templated on its closure and Riemann
// solver: ghost layers, sensor, connection and boundary fluxes, then the stage kernel of the
// closure and precision (ice_stage.cuh), and the IRS sweeps when they are on.
#pragma once
#include "ice_kernels.cuh"
#include "ice_mlp.cuh"

namespace ice {

template <int CL> inline void launch_stage_of(const LaunchArgs& a, bool write_r) {
  const bool f32 = a.precision == ICE_PREC_FP32FLUX && !write_r;
  if constexpr (CL == MK) { if (f32) launch_stage_mk_f32(a, write_r); else launch_stage_mk_f64(a, write_r); }
  else if constexpr (CL == IG) { if (f32) launch_stage_ig_f32(a, write_r); else launch_stage_ig_f64(a, write_r); }
  else { if (f32) launch_stage_ag_f32(a, write_r); else launch_stage_ag_f64(a, write_r); }
}

template <int CL> inline void launch_bound_of(const LaunchArgs& a) {
  const bool f32 = a.precision == ICE_PREC_FP32FLUX && !a.irs;
  if constexpr (CL == MK) { if (f32) launch_bound_mk_f32(a); else launch_bound_mk_f64(a); }
  else if constexpr (CL == IG) { if (f32) launch_bound_ig_f32(a); else launch_bound_ig_f64(a); }
  else { if (f32) launch_bound_ag_f32(a); else launch_bound_ag_f64(a); }
}

template <int CL> inline void launch_source_of(const LaunchArgs& a) {
  const bool f32 = a.precision == ICE_PREC_FP32FLUX;
  if constexpr (CL == MK) { if (f32) launch_source_mk_f32(a); else launch_source_mk_f64(a); }
  else if constexpr (CL == IG) { if (f32) launch_source_ig_f32(a); else launch_source_ig_f64(a); }
  else { if (f32) launch_source_ag_f32(a); else launch_source_ag_f64(a); }
}

template <int CL, int RS>
void launch_family_t(const LaunchArgs& a) {
  constexpr int nc = NC<CL>::v;
  cudaStream_t s = a.s;
  auto tick = [&](int cls) { if (a.tick) a.tick(a.tick_ctx, cls, s); };
  auto grid = [](long long n, int t) { return (unsigned)((n + t - 1) / t); };
  // compute_source comes first in the stage (Mod_Explicit.f90:111-117). The staged stage kernel
  // evaluates it per cell itself for a family without evaporation; an evaporating family's source
  // (iterative, with lane-divergent trip counts) runs in its own kernel at full occupancy, or in the
  // surrogate's source kernel, and the stage kernel reads it (FamDev::src_ready)
  if (a.F.coupled && a.mlp_img) {
    launch_source_mlp(CL, a, a.mlp_img, *a.mlp_norm);
    tick(KC_SOURCE);
  } else if (a.F.coupled && (a.ntile3 == 0 || a.F.src_ready)) {
    launch_source_of<CL>(a);
    tick(KC_SOURCE);
  }
  if (a.xchg) a.xchg(a, ICE_GPU_HALO_CELLS);   // the remote source cells of the ghost layers
  if (a.nrec > 0) {
    if (a.ghost_split) {
      k_ghost<CL><<<grid(a.nrec, 128), 128, 0, s>>>(a.G, a.F, a.grecs, a.nrec, 1);
      k_ghost<CL><<<grid(a.nrec, 128), 128, 0, s>>>(a.G, a.F, a.grecs, a.nrec, 2);
    } else {
      k_ghost<CL><<<grid(a.nrec, 128), 128, 0, s>>>(a.G, a.F, a.grecs, a.nrec, 3);
    }
    tick(KC_GHOST);
  }
  // the Jameson sensor: the staged stage kernel and the boundary kernels evaluate it from the
  // density they read; only the 1-D stage kernel reads it from a field
  if (a.sd && a.ntile3 == 0) {
    k_beta<<<grid(a.G.NI, 256), 256, 0, s>>>(a.G, a.F);
    tick(KC_BETA);
  }
  if (a.xchg) a.xchg(a, ICE_GPU_HALO_BETA);    // the weights of partner cells another rank steps
  if (a.nown > 0 || a.nbc > 0 || a.xchg) {
    launch_bound_of<CL>(a);
    tick(KC_BOUND);
  }
  if (!a.irs) {
    launch_stage_of<CL>(a, false);
    tick(KC_STAGE);
    return;
  }
  launch_stage_of<CL>(a, true);
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
