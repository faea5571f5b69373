// ice_kernels.cuh -- the kernels of the solve stage that depend on the closure (and the Riemann
// solver): per-cell dt, the ghost fill of both layers, connection and boundary fluxes, the fused
// stage kernel and the separate update of the IRS path. Included by the per-closure units
// (ice_fam_*.cu) and by ice_gpu.cu, each instantiating what it launches.
#pragma once
#include "ice_layout.cuh"

namespace ice {
namespace {

// ------------------------------------------------------------------ stencil functor
struct GStencil {            // q(s, v): cell s = 0..3 of the stencil, variable v
  const double* P; long long NG, g0, st;
  __device__ __forceinline__ double operator()(int s, int v) const { return __ldg(P + (long long)v * NG + g0 + s * st); }
};

template <typename R> struct CStencil {        // converted to R (FP32-flux form)
  const double* P; long long NG, g0, st;
  __device__ __forceinline__ R operator()(int s, int v) const { return (R)__ldg(P + (long long)v * NG + g0 + s * st); }
};

template <typename R, int NC_> struct RegStencil {   // the four cells held in registers (FP32 form)
  R v[4][NC_];
  __device__ __forceinline__ R operator()(int s, int q) const { return v[s][q]; }
};

// One interior face along d between the 0-based cells (i,j,k) and its upper neighbour:
// face_flux + compute_flux_ (Mod_Fluxes.f90:599-685). Returns true on an unphysical
// first-order face. The plain form reads the stencil through L1 as the reconstruction needs it;
// the FP32 form converts it once into registers.
template <int CL, int RS, int LIM, typename R>
__device__ __forceinline__ bool face_flux(const Geo& G, const FamDev& F, const DBlock& B, int d, int i, int j, int k,
                                         R* flux) {
  constexpr int nc = NC<CL>::v;
  const int c = d == 0 ? i : d == 1 ? j : k;
  const int n = d == 0 ? B.ni : d == 1 ? B.nj : B.nk;
  const int o0 = d == 0, o1 = d == 1, o2 = d == 2;
  R bf = (R)1;
  if (F.beta) bf = (R)mn(F.beta[iidx(B, i, j, k)], F.beta[iidx(B, i + o0, j + o1, k + o2)]);
  const double* dl = G.dl + (long long)d * G.NR;
  const long long r0 = ridx(B, i, j, k);
  const long long rs = d == 0 ? 1LL : d == 1 ? (long long)(B.ni + 2) : (long long)(B.ni + 2) * (B.nj + 2);
  R l0 = (R)dl[r0 - rs], l1 = (R)dl[r0], l2 = (R)dl[r0 + rs], l3 = (R)dl[r0 + 2 * rs];
  const long long st = gstride(B, d);
  const long long g0 = gidx(B, i, j, k) - st;
  if (c == 0 && F.inj[g0]) l0 = (R)0;
  if (c == n - 2 && F.inj[g0 + 3 * st]) l3 = (R)0;
  R dl0 = (R)0.5*(l0 + l1), dl1 = (R)0.5*(l1 + l2), dl2 = (R)0.5*(l2 + l3);
  R dll = (R)0.5*l1, dlr = (R)0.5*l2;
  R pl[nc], pr[nc], fl[nc];
  bool bad;
  if constexpr (sizeof(R) == 8) {
    CStencil<R> q{F.Up, G.NG, g0, st};
    bad = reconstruct<CL, LIM, R>(F.limiter, q, dl0, dl1, dl2, dll, dlr, pl, pr, bf);
  } else {
    RegStencil<R, nc> q;
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2)
#pragma unroll
      for (int v = 0; v < nc; ++v) q.v[s2][v] = (R)__ldg(F.Up + (long long)v * G.NG + g0 + s2 * st);
    bad = reconstruct<CL, LIM, R>(F.limiter, q, dl0, dl1, dl2, dll, dlr, pl, pr, bf);
  }
  const long long fi = fidx(B, d, i, j, k, c + 1);
  const long long NF = G.NF[d];
  const double* fc = G.face[d];
  R nrm[3] = {(R)fc[fi], (R)fc[NF + fi], (R)fc[2 * NF + fi]};
  R area = (R)fc[3 * NF + fi];
  riemann<CL, RS, R>(pl, pr, nrm, fl, (R)F.mat.cp);
#pragma unroll
  for (int v = 0; v < nc; ++v) flux[v] = fl[v] * area;
  return bad;
}

// Normal and area of face fi along d: the FP64 arrays in the plain form, the packed single-precision
// copy (one 16-byte load, the same roundings) in the FP32-flux form.
template <typename R>
__device__ __forceinline__ void face_geometry(const Geo& G, int d, long long fi, R* nrm, R& area) {
  if constexpr (sizeof(R) == 4) {
    const float4 f = G.ff[d][fi];
    nrm[0] = f.x; nrm[1] = f.y; nrm[2] = f.z; area = f.w;
  } else {
    const long long NF = G.NF[d];
    const double* fc = G.face[d];
    nrm[0] = fc[fi]; nrm[1] = fc[NF + fi]; nrm[2] = fc[2 * NF + fi]; area = fc[3 * NF + fi];
  }
}

// The length along d of the cell at ring index r, in the precision of R (the same rounding either way).
template <typename R>
__device__ __forceinline__ R cell_length(const Geo& G, int d, long long r) {
  if constexpr (sizeof(R) == 4) return G.dlf[(long long)d * G.NR + r];
  else return G.dl[(long long)d * G.NR + r];
}

// The Jameson weight of cell (i,j,k) of block B from the stage's density in global memory (the
// boundary kernels; compute_beta, Mod_Fluxes.f90:366-389).
template <typename R>
__device__ __forceinline__ R beta_cell(const FamDev& F, const DBlock& B, int i, int j, int k) {
  const double* P = F.Up;
  return sd_rho<R>((R)P[gidx(B, i, j, k)], (R)P[gidx(B, i - 1, j, k)], (R)P[gidx(B, i + 1, j, k)],
                   (R)P[gidx(B, i, j - 1, k)], (R)P[gidx(B, i, j + 1, k)],
                   (R)P[gidx(B, i, j, k - 1)], (R)P[gidx(B, i, j, k + 1)]);
}

// record_flux (Mod_BC_Fluxes.f90:180-272): the flux through a record's face into its cell. R is the
// reconstruction and Riemann type (double in the plain form, float in the FP32-flux form); LIM the
// limiter the kernel is specialised for (the same formulas as the run-time switch in double).
// The four stencil cells are read into registers before the reconstruction, so that their loads
// are in flight together (the reconstruction's branches would otherwise order them).
template <int CL, int RS, int LIM, typename R>
__device__ bool record_flux(const Geo& G, const FamDev& F, const DRec& r, double* flux, const double* beta_face) {
  constexpr int nc = NC<CL>::v;
  const DBlock& B = G.blk[r.b];
  int f = r.f, i = r.i, j = r.j, k = r.k;
  int g0 = (f == 1) - (f == 2), g1 = (f == 3) - (f == 4), g2 = (f == 5) - (f == 6);  // guide(f,:)
  int ig = i - g0, jg = j - g1, kg = k - g2;
  int ig2 = i - 2 * g0, jg2 = j - 2 * g1, kg2 = k - 2 * g2;
  int ip = i + g0, jp = j + g1, kp = k + g2;
  int dir = (f + 1) / 2 - 1;
  R bv = beta_face ? (R)*beta_face : (F.sd ? beta_cell<R>(F, B, i, j, k) : (R)1);
  R dl_g1 = cell_length<R>(G, dir, ridx(B, ig, jg, kg));
  R dl_m = cell_length<R>(G, dir, ridx(B, i, j, k));
  R dl_4 = cell_length<R>(G, dir, ridx(B, ip, jp, kp));
  R dl0, dl1, dl2, dll, dlr;
  R pl[nc], pr[nc], fl[nc];
  bool bad;
  const double* P = F.Up;
  if (f % 2 == 1) {
    long long fi = fidx(B, dir, i, j, k, (dir == 0 ? i : dir == 1 ? j : k));   // the face below the cell
    R nrm[3], area;
    face_geometry<R>(G, dir, fi, nrm, area);
    dl0 = dl_g1; dl1 = (R)0.5*(dl_g1 + dl_m); dl2 = (R)0.5*(dl_m + dl_4);
    dll = (R)0.5*dl_g1; dlr = (R)0.5*dl_m;
    if (F.inj[gidx(B, ig, jg, kg)]) { dl1 = (R)0.5*dl_m; dll = (R)0; }
    if (F.inj[gidx(B, ip, jp, kp)]) dl2 = (R)0.5*dl_m;
    long long a[4] = {gidx(B, ig2, jg2, kg2), gidx(B, ig, jg, kg), gidx(B, i, j, k), gidx(B, ip, jp, kp)};
    R stn[4][nc];
#pragma unroll
    for (int s4 = 0; s4 < 4; ++s4)
#pragma unroll
      for (int v = 0; v < nc; ++v) stn[s4][v] = (R)P[(long long)v * G.NG + a[s4]];
    auto q = [&](int s, int v) { return stn[s][v]; };
    bad = reconstruct<CL, LIM, R>(F.limiter, q, dl0, dl1, dl2, dll, dlr, pl, pr, bv);
    riemann<CL, RS, R>(pl, pr, nrm, fl, (R)F.mat.cp);
#pragma unroll
    for (int v = 0; v < nc; ++v) flux[v] = (double)(fl[v] * area);
  } else {
    long long fi = fidx(B, dir, i, j, k, (dir == 0 ? i : dir == 1 ? j : k) + 1);  // the face above the cell
    R nrm[3], area;
    face_geometry<R>(G, dir, fi, nrm, area);
    dl0 = (R)0.5*(dl_4 + dl_m); dl1 = (R)0.5*(dl_m + dl_g1); dl2 = dl_g1;
    dll = (R)0.5*dl_m; dlr = (R)0.5*dl_g1;
    if (F.inj[gidx(B, ig, jg, kg)]) { dl1 = (R)0.5*dl_m; dlr = (R)0; }
    if (F.inj[gidx(B, ip, jp, kp)]) dl0 = (R)0.5*dl_m;
    long long a[4] = {gidx(B, ip, jp, kp), gidx(B, i, j, k), gidx(B, ig, jg, kg), gidx(B, ig2, jg2, kg2)};
    R stn[4][nc];
#pragma unroll
    for (int s4 = 0; s4 < 4; ++s4)
#pragma unroll
      for (int v = 0; v < nc; ++v) stn[s4][v] = (R)P[(long long)v * G.NG + a[s4]];
    auto q = [&](int s, int v) { return stn[s][v]; };
    bad = reconstruct<CL, LIM, R>(F.limiter, q, dl0, dl1, dl2, dll, dlr, pl, pr, bv);
    riemann<CL, RS, R>(pl, pr, nrm, fl, (R)F.mat.cp);
#pragma unroll
    for (int v = 0; v < nc; ++v) flux[v] = (double)(-(fl[v] * area));
  }
  return bad;
}

// ------------------------------------------------------------------ step control
// Locates the block of interior cell q (flat over every block) by binary search on ioff.
__device__ __forceinline__ int find_block(const DBlock* blk, int nb, long long q) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (blk[mid].ioff <= q) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void decode(const DBlock& B, long long q, int& i, int& j, int& k) {
  long long l = q - B.ioff;
  i = (int)(l % B.ni); l /= B.ni;
  j = (int)(l % B.nj);
  k = (int)(l / B.nj);
}

// compute_dt for every family in one pass (Mod_dt.f90:11-112, 256-275; Mod_Explicit.f90:46-61): each
// cell's metric rows are read once for all families; the cell's indices come from its block by 32-bit
// arithmetic (ice_gpu_create refuses a block of 2^31 cells or more). Per family the operations of
// compute_dt_ in its order; the global step is the smallest over every family and cell (an exact
// minimum, so the order of the families does not matter).
struct DtFam {
  const double* Up;
  const double* tau;
  double* dt_out;   // the per-cell step (steady runs), or null
  int closure, coupled;
};
struct DtArgs {
  DtFam f[ICE_GPU_MAX_FAMILIES];
  int nf, ramp, ndir;
  double cfl, dt_max, tau_factor;
};

template <int CL>
__device__ __forceinline__ double family_dt(const Geo& G, const DtFam& f, const DtArgs& a, long long q, long long g,
                                            const double (*vs)[3], const double* gn, int it) {
  constexpr int nc = NC<CL>::v;
  double p[nc];
#pragma unroll
  for (int v = 0; v < nc; ++v) p[v] = f.Up[(long long)v * G.NG + g];
  double rate = 0.0;
  for (int d = 0; d < a.ndir; ++d)
    rate = rate + (fabs(p[1]*vs[d][0] + p[2]*vs[d][1] + p[3]*vs[d][2]) + wavespeed<CL>(p, vs[d])) * gn[d];
  double dt = (double)1e+5f;
  if (rate > 0.0) dt = mn(dt, 1.0/rate);
  dt = dt * a.cfl;
  if (it <= a.ramp) dt = dt * (double)it / (double)a.ramp;
  dt = mn(dt, a.dt_max);
  if (f.coupled && a.tau_factor > 0.0) {
    double tau = f.tau[q];
    if (p[0] > kRhoEmpty && !not_finite(tau) && tau > 0.0) dt = mn(dt, a.tau_factor*tau);
  }
  if (f.dt_out) f.dt_out[q] = dt;
  return dt;
}

__global__ void __launch_bounds__(256, 6) k_dt_all(Geo G, DtArgs a, Status* st) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double dt = INFINITY;
  const int bq = q < G.NI ? find_block(G.blk, G.nb, q) : 0;
  if (q < G.NI && stepped(G, bq)) {
    const DBlock& B = G.blk[bq];
    const unsigned l = (unsigned)(q - B.ioff), ni = (unsigned)B.ni, nj = (unsigned)B.nj;
    const unsigned i = l % ni, jk = l / ni, j = jk % nj, k = jk / nj;
    const long long g = gidx(B, (int)i, (int)j, (int)k);
    double vs[3][3], gn[3];
    for (int d = 0; d < a.ndir; ++d) {
      double t0 = G.M[(long long)d * G.NI + q], t1 = G.M[(long long)(3 + d) * G.NI + q], t2 = G.M[(long long)(6 + d) * G.NI + q];
      gn[d] = norm2_3(t0, t1, t2);
      vs[d][0] = t0 / gn[d]; vs[d][1] = t1 / gn[d]; vs[d][2] = t2 / gn[d];
    }
    const int it = st->iter;
    for (int p = 0; p < a.nf; ++p) {
      const DtFam& f = a.f[p];
      double d = f.closure == ICE_CLOSURE_MK ? family_dt<MK>(G, f, a, q, g, vs, gn, it)
               : f.closure == ICE_CLOSURE_IG ? family_dt<IG>(G, f, a, q, g, vs, gn, it)
                                             : family_dt<AG>(G, f, a, q, g, vs, gn, it);
      dt = mn(dt, d);
    }
  }
  // warp and block min; a positive double orders as its bits
  unsigned long long bits = (unsigned long long)__double_as_longlong(dt);
  for (int o = 16; o > 0; o >>= 1) bits = min(bits, __shfl_xor_sync(0xffffffffu, bits, o));
  __shared__ unsigned long long wmin[8];
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = bits;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = wmin[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = min(m, wmin[w]);
    atomicMin(&st->dtbits, m);
  }
}

// The rate of compute_dt_ (Mod_dt.f90:256-275): sum over the resolved directions of (|u . versor| +
// the closure's signal speed) times the modulus of the metric row, for the state p of cell q.
template <int CL>
__device__ __forceinline__ double dt_rate(const Geo& G, long long q, const double* p, int ndir) {
  double rate = 0.0;
  for (int d = 0; d < ndir; ++d) {
    double t0 = G.M[(long long)d * G.NI + q], t1 = G.M[(long long)(3 + d) * G.NI + q], t2 = G.M[(long long)(6 + d) * G.NI + q];
    double gn = norm2_3(t0, t1, t2);
    double vs[3] = {t0 / gn, t1 / gn, t2 / gn};
    rate = rate + (fabs(p[1]*vs[0] + p[2]*vs[1] + p[3]*vs[2]) + wavespeed<CL>(p, vs)) * gn;
  }
  return rate;
}

__global__ void k_empty_init(EmptyScan* e) {
  e->floor_bits = (unsigned long long)__double_as_longlong(1.79769313486231570e+308);
  e->src_bits = e->floor_bits;
  e->umax_bits[0] = e->umax_bits[1] = e->umax_bits[2] = 0ULL;
  e->filled = 0u;
}

// bound_empty_dt's first pass (Mod_dt.f90:134-196) over one family's cells, with the coupler's
// imports as the only source: an occupied cell (density above rho_empty) gives its step and speeds;
// an empty cell with a positive mass rate gives the speeds of what it receives (the rate's momentum
// over its mass) and the step of compute_dt_ at that speed, times cfl.
template <int CL>
__global__ void __launch_bounds__(256) k_empty_scan(Geo G, FamDev F, const double* dt_cell, double cfl, int ndir,
                                                    EmptyScan* e) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G.NI) return;
  const DBlock& B = G.blk[find_block(G.blk, G.nb, q)];
  int i, j, k; decode(B, q, i, j, k);
  constexpr int nc = NC<CL>::v;
  const long long g = gidx(B, i, j, k);
  double p[nc];
#pragma unroll
  for (int v = 0; v < nc; ++v) p[v] = F.Up[(long long)v * G.NG + g];
  double s[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) s[v] = F.imports[(long long)v * G.NI + q];
  if (s[0] > 0.0) atomicOr(&e->filled, 1u);
  if (p[0] > kRhoEmpty) {
    if (dt_cell) atomicMin(&e->floor_bits, (unsigned long long)__double_as_longlong(dt_cell[q]));
    for (int a = 0; a < 3; ++a) atomicMax(&e->umax_bits[a], (unsigned long long)__double_as_longlong(fabs(p[1 + a])));
    return;
  }
  if (!(s[0] > 0.0)) return;
  p[1] = s[1]/s[0]; p[2] = s[2]/s[0]; p[3] = s[3]/s[0];
  for (int a = 0; a < 3; ++a) atomicMax(&e->umax_bits[a], (unsigned long long)__double_as_longlong(fabs(p[1 + a])));
  double dts = (double)1e+5f;
  const double rate = dt_rate<CL>(G, q, p, ndir);
  if (rate > 0.0) dts = mn(dts, 1.0/rate);
  atomicMin(&e->src_bits, (unsigned long long)__double_as_longlong(dts*cfl));
}

// bound_empty_dt's second pass (Mod_dt.f90:197-214) and bound_removal_dt (Mod_dt.f90:220-242). Time-
// accurate: the global step lowered to the sources' step (when a source fills anything) and to each
// cell's removal step (its density over the rate the coupler takes out). Steady: each empty cell's
// step lowered to the smaller of the occupied cells' smallest step and the sources', and to cfl over
// its rate at the largest speeds; each cell's to its removal step. Only minima: the order of the two
// bounds does not change a bit.
template <int CL>
__global__ void __launch_bounds__(256) k_empty_apply(Geo G, FamDev F, double* dt_cell, double cfl, int ndir,
                                                     const EmptyScan* e, Status* st) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G.NI) return;
  const DBlock& B = G.blk[find_block(G.blk, G.nb, q)];
  int i, j, k; decode(B, q, i, j, k);
  const double rho = F.Up[gidx(B, i, j, k)];
  const bool filled = e->filled != 0u;
  const double src_dt = __longlong_as_double((long long)e->src_bits);
  if (!dt_cell) {                                    // time-accurate
    if (q == 0 && filled) atomicMin(&st->dtbits, e->src_bits);
  } else if (filled && !(rho > kRhoEmpty)) {
    const double floor_dt = mn(__longlong_as_double((long long)e->floor_bits), src_dt);
    double umax[3];
    for (int a = 0; a < 3; ++a) umax[a] = __longlong_as_double((long long)e->umax_bits[a]);
    double rate = 0.0;
    for (int d = 0; d < ndir; ++d) {
      double sum = umax[0]*fabs(G.M[(long long)d * G.NI + q]);
      sum = sum + umax[1]*fabs(G.M[(long long)(3 + d) * G.NI + q]);
      sum = sum + umax[2]*fabs(G.M[(long long)(6 + d) * G.NI + q]);
      rate = rate + sum;
    }
    double dts = floor_dt;
    if (rate > 0.0) dts = mn(dts, cfl/rate);
    dt_cell[q] = mn(dt_cell[q], dts);
  }
  const double out = -F.imports[q];
  if (!(out > 0.0)) return;
  const double dts = rho/out;
  if (!dt_cell) atomicMin(&st->dtbits, (unsigned long long)__double_as_longlong(dts));
  else dt_cell[q] = mn(dt_cell[q], dts);
}

// ------------------------------------------------------------------ ghosts
__device__ __forceinline__ int ghost_rule(const DRec& r, double veln) {
  int rule = 0;  // copy
  if (r.type == 200) rule = 1;
  else if (r.type == 300 || r.type == 301) {
    if (veln*(double)(1 - 2*(r.f % 2)) <= 0.0 || r.f == 3) rule = 1;
  } else if (r.type >= 401 && r.type <= 403) {
    if (!(veln*(double)(1 - 2*(r.f % 2)) > 0.0)) {
      rule = 2;
      if (r.massflux == 0.0) rule = 1;
    }
  }
  return rule;
}

__device__ __forceinline__ void rec_normal(const Geo& G, const DBlock& B, const DRec& r, double* n, double* area) {
  int d = (r.f - 1) / 2;
  int F = (d == 0 ? r.i : d == 1 ? r.j : r.k) + 1 - (r.f % 2);   // im - mod(fm,2), 1-based
  long long fi = fidx(B, d, r.i, r.j, r.k, F);
  long long NF = G.NF[d];
  n[0] = G.face[d][fi]; n[1] = G.face[d][NF + fi]; n[2] = G.face[d][2 * NF + fi];
  if (area) *area = G.face[d][3 * NF + fi];
}

// ghost_chimera (Lib_Ghost.f90:439-466): ghost cell gg (layer 1 or 2) of a chimera record from its
// donors, the weighted sum of their conservative states in donor order, back to primitive with the
// closure's floors. The donors are interior cells, which no ghost fill writes.
template <int CL>
__device__ __forceinline__ void chimera_ghost(const Geo& G, const FamDev& F, const DRec& r, int layer, long long gg) {
  constexpr int nc = NC<CL>::v;
  const double* P = F.Ug;
  const long long NG = G.NG;
  const int d0 = r.cd0 + (layer == 1 ? 0 : r.cn1), d1 = d0 + (layer == 1 ? r.cn1 : r.cn2);
  double cs[nc];
#pragma unroll
  for (int v = 0; v < nc; ++v) cs[v] = 0.0;
  for (int d = d0; d < d1; ++d) {
    const int4 dn = F.cdon[d];
    const long long gd = gidx(G.blk[dn.x], dn.y, dn.z, dn.w);
    const double w = F.cw[d];
    double pd[nc], cd[nc];
#pragma unroll
    for (int v = 0; v < nc; ++v) pd[v] = P[v * NG + gd];
    prim2cons<CL, double>(pd, cd, F.mat.cp);
#pragma unroll
    for (int v = 0; v < nc; ++v) cs[v] = cs[v] + w*cd[v];
  }
  double pg[nc];
  cons2prim<CL>(cs, pg, F.mat.cp);
#pragma unroll
  for (int v = 0; v < nc; ++v) F.Ug[v * NG + gg] = pg[v];
}

// ghost_record (Lib_Ghost.f90:76-267)
template <int CL>
__device__ __forceinline__ void ghost1_rec(const Geo& G, const FamDev& F, const DRec& r) {
  constexpr int nc = NC<CL>::v;
  const DBlock& B = G.blk[r.b];
  int g0 = (r.f == 1) - (r.f == 2), g1 = (r.f == 3) - (r.f == 4), g2 = (r.f == 5) - (r.f == 6);
  long long gg = gidx(B, r.i - g0, r.j - g1, r.k - g2);
  long long gm = gidx(B, r.i, r.j, r.k);
  double* P = F.Ug;
  const long long NG = G.NG;
  switch (r.type) {
    case 101: case 201: {
      const DBlock& S = G.blk[r.bs];
      long long gs = gidx(S, r.is, r.js, r.ks);
#pragma unroll
      for (int v = 0; v < nc; ++v) P[v * NG + gg] = P[v * NG + gs];
      break;
    }
    case 200: case 300: case 301: {
      double nrm[3]; rec_normal(G, B, r, nrm, nullptr);
      double m[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v) m[v] = P[v * NG + gm];
      double gv[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v) gv[v] = m[v];
      double vel[3] = {m[1], m[2], m[3]};
      double veln = vel[0]*nrm[0] + vel[1]*nrm[1] + vel[2]*nrm[2];
      if (ghost_rule(r, veln) == 1) {
        for (int a = 0; a < 3; ++a) vel[a] = vel[a] - 2.0*veln*nrm[a];
        if constexpr (CL == AG) mirror_tensor(m + 4, nrm, gv + 4);
      }
      gv[1] = vel[0]; gv[2] = vel[1]; gv[3] = vel[2];
#pragma unroll
      for (int v = 0; v < nc; ++v) P[v * NG + gg] = gv[v];
      break;
    }
    case 0: case 400: {
#pragma unroll
      for (int v = 0; v < nc; ++v) P[v * NG + gg] = P[v * NG + gm];
      break;
    }
    case 401: case 402: case 403: {
      double nrm[3]; rec_normal(G, B, r, nrm, nullptr);
      double m[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v) m[v] = P[v * NG + gm];
      double vel[3] = {m[1], m[2], m[3]};
      double veln = vel[0]*nrm[0] + vel[1]*nrm[1] + vel[2]*nrm[2];
      int rule = ghost_rule(r, veln);
      F.inj[gg] = (rule == 2);
      double gv[nc];
      if (rule == 0) {
#pragma unroll
        for (int v = 0; v < nc; ++v) gv[v] = m[v];
      } else if (rule == 1) {
#pragma unroll
        for (int v = 0; v < nc; ++v) gv[v] = m[v];
        for (int a = 0; a < 3; ++a) vel[a] = vel[a] - 2.0*veln*nrm[a];
        gv[1] = vel[0]; gv[2] = vel[1]; gv[3] = vel[2];
        if constexpr (CL == AG) mirror_tensor(m + 4, nrm, gv + 4);
      } else {
#pragma unroll
        for (int v = 0; v < nc; ++v) gv[v] = 0.0;
        double sgn = (double)(2*(r.f % 2) - 1);
        double inward[3] = {sgn*nrm[0], sgn*nrm[1], sgn*nrm[2]};
        long long q = iidx(B, r.i, r.j, r.k);
        const double* gas = G.gas;
        double v3[3], speed;
        auto injv = [&](double sp) {
          if (r.normal_dir) { v3[0] = sp*inward[0]; v3[1] = sp*inward[1]; v3[2] = sp*inward[2]; }
          else { v3[0] = sp*r.cb*r.ca; v3[1] = sp*r.cb*r.sa; v3[2] = sp*r.sb; }
        };
        if (r.type == 401) {
          double gu = gas[1 * G.NI + q], gvv = gas[2 * G.NI + q], gw = gas[3 * G.NI + q];
          double vn = gu*inward[0] + gvv*inward[1] + gw*inward[2];
          injv(r.velocity*vn);
          gv[1] = v3[0]; gv[2] = v3[1]; gv[3] = v3[2];
          gv[0] = r.massflux*gas[q]/r.velocity;
          vn = fabs(gv[1]*nrm[0] + gv[2]*nrm[1] + gv[3]*nrm[2]);
          if (r.gfixed > 0.0 && vn > 0.0) gv[0] = gv[0] + r.massflux*r.gfixed/vn;
          gv[nc - 2] = r.temperature*gas[4 * G.NI + q];
        } else if (r.type == 402) {
          injv(r.velocity);
          gv[1] = v3[0]; gv[2] = v3[1]; gv[3] = v3[2];
          double vn = gv[1]*nrm[0] + gv[2]*nrm[1] + gv[3]*nrm[2];
          gv[0] = r.massflux/fabs(vn);
          gv[nc - 2] = r.temperature;
        } else {
          speed = norm2_3(gas[1 * G.NI + q], gas[2 * G.NI + q], gas[3 * G.NI + q]);
          injv(r.velocity*speed);
          gv[1] = v3[0]; gv[2] = v3[1]; gv[3] = v3[2];
          double vn = gv[1]*nrm[0] + gv[2]*nrm[1] + gv[3]*nrm[2];
          gv[0] = r.massflux/fabs(vn);
          gv[nc - 2] = r.temperature;
        }
        gv[nc - 1] = gv[0]/F.mat.rho/r.vol_p;
        if constexpr (CL == IG) gv[4] = 1e-6;
        if constexpr (CL == AG) { gv[4] = 1e-6; gv[7] = 1e-6; gv[9] = 1e-6; }
      }
#pragma unroll
      for (int v = 0; v < nc; ++v) P[v * NG + gg] = gv[v];
      break;
    }
    case 102:
      chimera_ghost<CL>(G, F, r, 1, gg);
      break;
    default: break;
  }
}

// second_ghost_record (Lib_Ghost.f90:312-387)
template <int CL>
__device__ __forceinline__ void ghost2_rec(const Geo& G, const FamDev& F, const DRec& r) {
  constexpr int nc = NC<CL>::v;
  if (r.type == 0) return;
  const DBlock& B = G.blk[r.b];
  int g0 = (r.f == 1) - (r.f == 2), g1 = (r.f == 3) - (r.f == 4), g2 = (r.f == 5) - (r.f == 6);
  long long gg1 = gidx(B, r.i - g0, r.j - g1, r.k - g2);
  long long gg2 = gidx(B, r.i - 2 * g0, r.j - 2 * g1, r.k - 2 * g2);
  long long gm = gidx(B, r.i, r.j, r.k);
  long long gp = gidx(B, r.i + g0, r.j + g1, r.k + g2);
  double* P = F.Ug;
  const long long NG = G.NG;
  switch (r.type) {
    case 101: case 201: {
      const DBlock& S = G.blk[r.bs];
      int s0 = (r.fs == 1) - (r.fs == 2), s1 = (r.fs == 3) - (r.fs == 4), s2 = (r.fs == 5) - (r.fs == 6);
      long long gs = gidx(S, r.is + s0, r.js + s1, r.ks + s2);
#pragma unroll
      for (int v = 0; v < nc; ++v) P[v * NG + gg2] = P[v * NG + gs];
      break;
    }
    case 200: case 300: case 301: case 401: case 402: case 403: {
      double nrm[3]; rec_normal(G, B, r, nrm, nullptr);
      double m1 = P[1 * NG + gm], m2 = P[2 * NG + gm], m3 = P[3 * NG + gm];
      double veln = m1*nrm[0] + m2*nrm[1] + m3*nrm[2];
      int rule = ghost_rule(r, veln);
      double gv[nc];
      if (rule == 2) {
#pragma unroll
        for (int v = 0; v < nc; ++v) gv[v] = P[v * NG + gg1];
      } else {
        double mp[nc];
#pragma unroll
        for (int v = 0; v < nc; ++v) { mp[v] = P[v * NG + gp]; gv[v] = mp[v]; }
        if (rule == 1) {
          double d = mp[1]*nrm[0] + mp[2]*nrm[1] + mp[3]*nrm[2];
          for (int a = 0; a < 3; ++a) gv[1 + a] = mp[1 + a] - 2.0*d*nrm[a];
          if constexpr (CL == AG) mirror_tensor(mp + 4, nrm, gv + 4);
        }
      }
#pragma unroll
      for (int v = 0; v < nc; ++v) P[v * NG + gg2] = gv[v];
      break;
    }
    case 102:
      chimera_ghost<CL>(G, F, r, 2, gg2);
      break;
    default: {
#pragma unroll
      for (int v = 0; v < nc; ++v) P[v * NG + gg2] = 3.0*P[v * NG + gg1] - 3.0*P[v * NG + gm] + P[v * NG + gp];
      break;
    }
  }
}

// The ghost layers of every record, one thread per record; layers: 1 the first, 2 the second, 3 both.
// compute_ghost fills layer 1 of every record and then fill_second_ghost layer 2 (Lib_Ghost.f90:29-387).
// A record's layer 2 reads its own layer-1 cell and the cell one further inside (of its block, or of the
// source block of a connection). Where that block is two cells or more deep along the record's face
// direction the cell is interior, no other record writes it, and one thread does both layers in turn
// (layers = 3). Where it is one cell deep the cell is the opposite face's layer-1 ghost, which another
// record writes: then the host launches layer 1 of every record first and layer 2 after it.
//
// Both layers of the copying records at once (layers = 3: 0 and 400 extrapolate, 101 and 201 copy
// from the partner block): every load first, then every store, the values and operations of
// ghost1_rec followed by ghost2_rec (layer 2 of a 400 record, 3 g1 - 3 m + p, with g1 the layer-1
// value just copied from m).
template <int CL>
__device__ __forceinline__ void ghost12_copy(const Geo& G, const FamDev& F, const DRec& r) {
  constexpr int nc = NC<CL>::v;
  const DBlock& B = G.blk[r.b];
  const int g0 = (r.f == 1) - (r.f == 2), g1 = (r.f == 3) - (r.f == 4), g2 = (r.f == 5) - (r.f == 6);
  const long long gg1 = gidx(B, r.i - g0, r.j - g1, r.k - g2);
  const long long gg2 = gidx(B, r.i - 2 * g0, r.j - 2 * g1, r.k - 2 * g2);
  double* P = F.Ug;
  const long long NG = G.NG;
  double a[nc], b[nc];
  if (r.type == 101 || r.type == 201) {
    const DBlock& S = G.blk[r.bs];
    const int s0 = (r.fs == 1) - (r.fs == 2), s1 = (r.fs == 3) - (r.fs == 4), s2 = (r.fs == 5) - (r.fs == 6);
    const long long gs1 = gidx(S, r.is, r.js, r.ks), gs2 = gidx(S, r.is + s0, r.js + s1, r.ks + s2);
#pragma unroll
    for (int v = 0; v < nc; ++v) { a[v] = P[v * NG + gs1]; b[v] = P[v * NG + gs2]; }
  } else {
    const long long gm = gidx(B, r.i, r.j, r.k), gp = gidx(B, r.i + g0, r.j + g1, r.k + g2);
#pragma unroll
    for (int v = 0; v < nc; ++v) a[v] = P[v * NG + gm];
    if (r.type == 400) {
#pragma unroll
      for (int v = 0; v < nc; ++v) b[v] = 3.0*a[v] - 3.0*a[v] + P[v * NG + gp];
    }
  }
#pragma unroll
  for (int v = 0; v < nc; ++v) P[v * NG + gg1] = a[v];
  if (r.type != 0) {
#pragma unroll
    for (int v = 0; v < nc; ++v) P[v * NG + gg2] = b[v];
  }
}

template <int CL>
__global__ void k_ghost(Geo G, FamDev F, const DRec* recs, int nrec, int layers) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nrec) return;
  const DRec r = recs[n];
  if (!stepped(G, r.b)) return;
  if (layers == 3 && (r.type == 0 || r.type == 400 || r.type == 101 || r.type == 201)) {
    ghost12_copy<CL>(G, F, r);
    return;
  }
  if (layers & 1) ghost1_rec<CL>(G, F, r);
  if (layers & 2) ghost2_rec<CL>(G, F, r);
}

// ------------------------------------------------------------------ boundary fluxes
// A split run's BETA exchange: the Jameson weight of each listed cell (0-based block, i, j, k), as the
// connection kernel of the same precision and translation unit evaluates it (k_conn).
template <typename R>
__global__ void k_pack_beta(Geo G, FamDev F, const int4* __restrict__ e, int n, double* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int4 x = e[q];
  out[q] = F.sd ? (double)beta_cell<R>(F, G.blk[x.x], x.y, x.z, x.w) : 1.0;
}

template <int CL, int RS, int LIM, typename R>
__global__ void __launch_bounds__(128, 4) k_conn(Geo G, FamDev F, const DRec* recs, const int* own, int nown, Status* st) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nown) return;
  constexpr int nc = NC<CL>::v;
  const DRec& r = recs[own[n]];
  if (!stepped(G, r.b)) return;
  R bo = (R)1, bq = (R)1;
  if (F.sd) {
    bo = beta_cell<R>(F, G.blk[r.b], r.i, r.j, r.k);
    // a partner in a block another rank steps: its weight, which that rank sent (ICE_GPU_HALO_BETA)
    bq = stepped(G, r.pb) ? beta_cell<R>(F, G.blk[r.pb], r.pi, r.pj, r.pk)
                          : (R)F.beta[iidx(G.blk[r.pb], r.pi, r.pj, r.pk)];
  }
  const double bf = (double)mn(bo, bq);
  double fl[nc];
  if (record_flux<CL, RS, LIM, R>(G, F, r, fl, &bf)) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_BAD_RECON);
#pragma unroll
  for (int v = 0; v < nc; ++v) F.connF[(long long)r.cf * nc + v] = fl[v];
}

template <int CL, int RS, int LIM, typename R>
__global__ void __launch_bounds__(128, 4) k_bound(Geo G, FamDev F, const DRec* recs, const int* first, const int* list,
                                                  const int* perm, int nbc, Status* st) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbc) return;
  const int c = perm[t];
  if (!stepped(G, recs[list[first[c]]].b)) return;
  constexpr int nc = NC<CL>::v;
  double acc[nc];
#pragma unroll
  for (int v = 0; v < nc; ++v) acc[v] = 0.0;
  for (int rr = first[c]; rr < first[c + 1]; ++rr) {
    const DRec& r = recs[list[rr]];
    double fl[nc];
    if (r.type == 200 && CL == MK) continue;
    if (r.type == 101 || r.type == 201) {
#pragma unroll
      for (int v = 0; v < nc; ++v) { double x = F.connF[(long long)r.cf * nc + v]; fl[v] = r.owner ? x : -x; }
    } else {
      if (record_flux<CL, RS, LIM, R>(G, F, r, fl, nullptr)) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_BAD_RECON);
    }
#pragma unroll
    for (int v = 0; v < nc; ++v) acc[v] = acc[v] + fl[v];
  }
#pragma unroll
  for (int v = 0; v < nc; ++v) F.Rbw[(long long)c * nc + v] = acc[v];
}

// ------------------------------------------------------------------ the stage

// compute_source (Mod_Sources.f90:19-72): the source of every cell of one family, from the state
// at the start of the stage and the frozen gas; written to S (and tau, on the last stage), which
// the stage kernel adds to the residual. Its own kernel, so that the iterative closures do not
// share the stencil kernel's registers.
template <int CL, typename R>
__global__ void __launch_bounds__(256, 4) k_source(Geo G, FamDev F) {
  constexpr int nc = NC<CL>::v;
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G.NI) return;
  const int bq = find_block(G.blk, G.nb, q);
  if (!stepped(G, bq)) return;
  const DBlock& B = G.blk[bq];
  const unsigned l = (unsigned)(q - B.ioff), ni = (unsigned)B.ni, nj = (unsigned)B.nj;   // < 2^31 cells a block
  const unsigned i = l % ni, jk = l / ni, j = jk % nj, k = jk / nj;
  const long long g = gidx(B, (int)i, (int)j, (int)k);
  R p[nc], gas[5], s[nc];
#pragma unroll
  for (int v = 0; v < nc; ++v) p[v] = (R)F.Up[(long long)v * G.NG + g];
  R gr[9];
#pragma unroll
  for (int v = 0; v < 9; ++v) gr[v] = sizeof(R) == 4 ? (R)G.gasf[(long long)v * G.NI + q] : (R)G.gas[(long long)v * G.NI + q];
#pragma unroll
  for (int v = 0; v < 5; ++v) gas[v] = gr[v];
  R tau = cell_source<CL, R>(p, gas, gr[5], gr[6], gr[7], gr[8], F.mat, F.drag, F.heat, F.blow, s);
  if constexpr (sizeof(R) == 4) {
#pragma unroll
    for (int v = 0; v < nc; ++v) F.Sf[(long long)v * G.NI + q] = (F.frozen_mask & (1u << v)) ? 0.f : s[v];
  } else {
#pragma unroll
    for (int v = 0; v < nc; ++v) F.S[(long long)v * G.NI + q] = (F.frozen_mask & (1u << v)) ? 0.0 : (double)s[v];
  }
  if (F.write_tau) F.tau[q] = (double)tau;
}

// The stage kernel. One CTA of TX x TY threads (256) owns a column tile of one block and marches
// up a chunk of KZ planes. On each plane every thread computes exactly one x face (the face below
// its cell), one y face and one z face (the face above its cell; the one below comes from the
// plane before, or is computed once at the chunk's first plane) into shared memory, so the work is
// the same for every thread; then each cell of the tile's (TX-1) x (TY-1) interior takes its two
// faces per direction in the reference's odd-then-even order (Mod_Fluxes.f90:470-506), adds the
// source, forms R = (R/vol + S) dt, and applies the RK stage in conservative variables with the
// reference's floors and checks (Lib_Newstate.f90:198-219).
#ifndef ICE_STAGE_MINB
#define ICE_STAGE_MINB 1      // resident CTAs per SM the register allocation is held to
#endif
template <int CL, int RS, int LIM, typename R>
__global__ void __launch_bounds__(256, ICE_STAGE_MINB)
k_stage(Geo G, FamDev F, const Tile* tiles, int TX, int TY, int KZ, int write_r, Status* st) {
  constexpr int nc = NC<CL>::v;
  extern __shared__ double smem[];
  const int NT = TX * TY;
  double* Fx = smem;                  // [nc][NT]
  double* Fy = smem + nc * NT;
  double* Fz0 = smem + 2 * nc * NT;
  double* Fz1 = smem + 3 * nc * NT;
  const Tile t = tiles[blockIdx.x];
  const DBlock& B = G.blk[t.b];
  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int i = t.i0 + tx, j = t.j0 + ty;
  const bool ax = B.ni >= 2, ay = B.nj >= 2, az = B.nk >= 2;
  const bool col = i < B.ni && j < B.nj;
  const bool owner = col && (ax ? tx < TX - 1 : tx == 0) && (ay ? ty < TY - 1 : ty == 0);
  const int k1 = min(t.k0 + KZ, B.nk);
  bool bad = false;
  double* flo = Fz0;
  double* fhi = Fz1;
  if (az && col && t.k0 >= 1) {       // the face below the chunk's first plane
    R fl[nc];
    bad |= face_flux<CL, RS, LIM, R>(G, F, B, 2, i, j, t.k0 - 1, fl);
#pragma unroll
    for (int v = 0; v < nc; ++v) flo[v * NT + tid] = (double)fl[v];
  }
  for (int k = t.k0; k < k1; ++k) {
    if (ax && col && i >= 1) {        // x face below (i,j,k)
      R fl[nc];
      bad |= face_flux<CL, RS, LIM, R>(G, F, B, 0, i - 1, j, k, fl);
#pragma unroll
      for (int v = 0; v < nc; ++v) Fx[v * NT + tid] = (double)fl[v];
    }
    if (ay && col && j >= 1) {        // y face below (i,j,k)
      R fl[nc];
      bad |= face_flux<CL, RS, LIM, R>(G, F, B, 1, i, j - 1, k, fl);
#pragma unroll
      for (int v = 0; v < nc; ++v) Fy[v * NT + tid] = (double)fl[v];
    }
    if (az && col && k <= B.nk - 2) { // z face above (i,j,k)
      R fl[nc];
      bad |= face_flux<CL, RS, LIM, R>(G, F, B, 2, i, j, k, fl);
#pragma unroll
      for (int v = 0; v < nc; ++v) fhi[v * NT + tid] = (double)fl[v];
    }
    __syncthreads();
    if (owner) {
      const long long q = iidx(B, i, j, k);
      const int bc = F.bmap[q];
      double r[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v) r[v] = bc >= 0 ? F.Rb[(long long)bc * nc + v] : 0.0;
      // direction 1: face tid+1 is the cell's upper face, face tid its lower one
      if (ax) {
        const int ci = i + 1, n = B.ni;
        if (ci % 2 == 1) {
          if (ci < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - Fx[v * NT + tid + 1];
          }
          if (ci > 1) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] + Fx[v * NT + tid];
          }
        } else {
#pragma unroll
          for (int v = 0; v < nc; ++v) r[v] = r[v] + Fx[v * NT + tid];
          if (ci < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - Fx[v * NT + tid + 1];
          }
        }
      }
      if (ay) {
        const int cj = j + 1, n = B.nj;
        if (cj % 2 == 1) {
          if (cj < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - Fy[v * NT + tid + TX];
          }
          if (cj > 1) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] + Fy[v * NT + tid];
          }
        } else {
#pragma unroll
          for (int v = 0; v < nc; ++v) r[v] = r[v] + Fy[v * NT + tid];
          if (cj < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - Fy[v * NT + tid + TX];
          }
        }
      }
      if (az) {
        const int ck = k + 1, n = B.nk;
        if (ck % 2 == 1) {
          if (ck < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - fhi[v * NT + tid];
          }
          if (ck > 1) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] + flo[v * NT + tid];
          }
        } else {
#pragma unroll
          for (int v = 0; v < nc; ++v) r[v] = r[v] + flo[v * NT + tid];
          if (ck < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - fhi[v * NT + tid];
          }
        }
      }
      const long long g = gidx(B, i, j, k);
      double p[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v) p[v] = F.Up[(long long)v * G.NG + g];
      double s[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v)
        s[v] = !F.coupled ? 0.0 : F.Sf ? (double)F.Sf[(long long)v * G.NI + q] : F.S[(long long)v * G.NI + q];
      if (F.xstep) accumulate_source<CL>(F.xstep, G.NI, q, s, F.xfirst, F.rk);
      const double dt = F.dt ? F.dt[q] : *F.dtg;
      const double vol = G.vol[q];
#pragma unroll
      for (int v = 0; v < nc; ++v) r[v] = (r[v]/vol + s[v]) * dt;
      if (F.imports) {                          // add_births (Lib_Residual.f90:164-210): the coupler's rates
#pragma unroll
        for (int v = 0; v < nc; ++v) r[v] = r[v] + F.imports[(long long)v * G.NI + q] * dt;
      }
#pragma unroll
      for (int v = 0; v < nc; ++v) if (F.frozen_mask & (1u << v)) r[v] = 0.0;
      if (write_r) {
#pragma unroll
        for (int v = 0; v < nc; ++v) F.resid[(long long)v * G.NI + q] = r[v];
      } else {
        double po[nc], co[nc], cn[nc];
#pragma unroll
        for (int v = 0; v < nc; ++v) po[v] = F.U0[(long long)v * G.NG + g];
        prim2cons<CL, double>(po, co, F.mat.cp);
        prim2cons<CL, double>(p, cn, F.mat.cp);
#pragma unroll
        for (int v = 0; v < nc; ++v) { double rr = (cn[v] - co[v] + r[v]) * F.rk; cn[v] = co[v] + rr; }
        if (cn[0] < 0.0) atomicAdd(&st->nfloored, 1ULL);
        cons2prim<CL>(cn, p, F.mat.cp);
        if constexpr (sizeof(R) == 4) {
          if (F.realize && realize<CL>(p)) atomicAdd(&st->nrealized, 1ULL);
        }
        if (!check_prim<CL, double>(p)) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_NAN_STATE);
#pragma unroll
        for (int v = 0; v < nc; ++v) F.Uo[(long long)v * G.NG + g] = p[v];
      }
    }
    __syncthreads();
    double* tmp = flo; flo = fhi; fhi = tmp;
  }
  if (bad) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_BAD_RECON);
}

// ------------------------------------------------------------------ IRS and the separate update
template <int CL>
__global__ void k_update(Geo G, FamDev F, Status* st) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G.NI) return;
  constexpr int nc = NC<CL>::v;
  const DBlock& B = G.blk[find_block(G.blk, G.nb, q)];
  int i, j, k; decode(B, q, i, j, k);
  long long g = gidx(B, i, j, k);
  double p[nc], po[nc], co[nc], cn[nc];
#pragma unroll
  for (int v = 0; v < nc; ++v) { p[v] = F.Up[(long long)v * G.NG + g]; po[v] = F.U0[(long long)v * G.NG + g]; }
  prim2cons<CL, double>(po, co, F.mat.cp);
  prim2cons<CL, double>(p, cn, F.mat.cp);
#pragma unroll
  for (int v = 0; v < nc; ++v) { double rr = (cn[v] - co[v] + F.resid[(long long)v * G.NI + q]) * F.rk; cn[v] = co[v] + rr; }
  if (cn[0] < 0.0) atomicAdd(&st->nfloored, 1ULL);
  cons2prim<CL>(cn, p, F.mat.cp);
  if (!check_prim<CL, double>(p)) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_NAN_STATE);
#pragma unroll
  for (int v = 0; v < nc; ++v) F.Uo[(long long)v * G.NG + g] = p[v];
}


__global__ void k_begin(Status* st) {
  st->iter += 1;
  st->iter_from_call += 1;
  double d = (double)1e+5f;
  st->dtbits = (unsigned long long)__double_as_longlong(d);
}

__global__ void k_time(Status* st, int time_accurate) {
  double d = __longlong_as_double((long long)st->dtbits);
  st->dtglobal = d;
  if (time_accurate) st->time = st->time + d;
}


// ------------------------------------------------------------------ sensor
__global__ void k_beta(Geo G, FamDev F) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G.NI) return;
  const DBlock& B = G.blk[find_block(G.blk, G.nb, q)];
  int i, j, k; decode(B, q, i, j, k);
  const double* P = F.Up;   // variable 0: density
  F.betaw[q] = sd_rho<double>(P[gidx(B, i, j, k)], P[gidx(B, i - 1, j, k)], P[gidx(B, i + 1, j, k)],
                      P[gidx(B, i, j - 1, k)], P[gidx(B, i, j + 1, k)],
                      P[gidx(B, i, j, k - 1)], P[gidx(B, i, j, k + 1)]);
}


// One Jacobi sweep of direction d (Lib_IRS.f90:278-293): out = (R + b (star_{-1} + star_{+1}))/(1+2b),
// with the ghost values of star fixed to the first and last cell of R (zero gradient).
__global__ void k_irs(Geo G, int nc, const double* R0, const double* star, double* out, int d, double beta) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G.NI) return;
  const DBlock& B = G.blk[find_block(G.blk, G.nb, q)];
  int i, j, k; decode(B, q, i, j, k);
  int c = d == 0 ? i : d == 1 ? j : k;
  int n = d == 0 ? B.ni : d == 1 ? B.nj : B.nk;
  long long st = d == 0 ? 1 : d == 1 ? B.ni : (long long)B.ni * B.nj;
  long long qm = c > 0 ? q - st : q;         // ghost 0 = cell 1 of the original residual
  long long qp = c < n - 1 ? q + st : q;
  for (int v = 0; v < nc; ++v) {
    const double* S = (c > 0 ? star : R0) + (long long)v * G.NI;
    const double* Sp = (c < n - 1 ? star : R0) + (long long)v * G.NI;
    out[(long long)v * G.NI + q] = (R0[(long long)v * G.NI + q] + beta*(S[qm] + Sp[qp])) / (1.0 + 2.0*beta);
  }
}


// ------------------------------------------------------------------ residual norm
// residual_sq (Mod_Diagnostic.f90:106-130): per CTA, sums of (new - old)^2 of rho, u, v, w, T
// over a contiguous range of one block's cells, reduced in a fixed order.

__global__ void k_norm(Geo G, const double* Un, const double* Uo, int iT, const NormChunk* ch, double* part) {
  const NormChunk c = ch[blockIdx.x];
  const DBlock& B = G.blk[c.b];
  double acc[5] = {0, 0, 0, 0, 0};
  for (long long q = c.q0 + threadIdx.x; q < c.q1; q += blockDim.x) {
    int i, j, k; decode(B, q, i, j, k);
    long long g = gidx(B, i, j, k);
    int vs[5] = {0, 1, 2, 3, iT};
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      double d = fabs(Un[(long long)vs[m] * G.NG + g] - Uo[(long long)vs[m] * G.NG + g]);
      acc[m] = acc[m] + d*d;
    }
  }
  __shared__ double red[5][256];
#pragma unroll
  for (int m = 0; m < 5; ++m) red[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
#pragma unroll
      for (int m = 0; m < 5; ++m) red[m][threadIdx.x] = red[m][threadIdx.x] + red[m][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int m = 0; m < 5; ++m) part[(long long)blockIdx.x * 5 + m] = red[m][0];
  }
}


}  // namespace
}  // namespace ice
