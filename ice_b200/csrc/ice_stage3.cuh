// ice_stage3.cuh -- the stage kernel of 2-D and 3-D runs: the state planes staged in shared memory
// by TMA, a z-march over a column tile, every face flux of the tile computed once, the residual
// gathered per cell in the reference's order, the cell source, R = (R/vol + S) dt and the RK stage
// fused in one launch per family and stage.
//
// One CTA of NT threads owns a tile of w x h cells of one block (w h <= NT; the host picks each
// block's tile shape so that its tiles cut the block evenly, see tile_shape3 in ice_gpu.cu) and
// marches up a chunk of planes. Thread t < w h owns the cell (t % w, t / w) of the tile. Each plane of
// the family's state U_{k-1} (every variable, two halo cells on either side in x and y) arrives by one
// 4-D TMA load (x, y, z, variable) into an FP64 staging buffer, issued one plane ahead; the CTA
// converts it into a ring of three planes of the reconstruction type R (float in the FP32-flux form,
// double in the plain form). On each plane:
//  - z: the limited slope of the cell above (the slope the reference's state_reconstruction computes
//    for both faces of a cell, Lib_Reconstruction.f90:17-78) from planes k, k+1, k+2, kept in
//    registers, and the z face above the cell from the two cells' slopes: the same operations on the
//    same operands as the reference's per-face reconstruction, so the plain form keeps its bits;
//  - x and y: each thread the face below its own cell, then the w + h faces above the tile's last
//    column and last row as a short list of extra tasks (face_flux, Mod_Fluxes.f90:599-685), every
//    interior face of the tile once. The plain form reconstructs each face from its four-cell stencil;
//    the FP32-flux form first computes every cell's limited x and y slope once (the value the
//    per-face reconstruction computes twice, for the two faces of the cell) into the staging buffer,
//    and each face forms its two states from its cells' slopes; that form issues the next plane's
//    copy only after the faces, when the buffer is free again;
//  - each owned cell adds its boundary-record fluxes, then its two faces per direction in the
//    odd-then-even order of tile_sweep (Mod_Fluxes.f90:470-506), evaluates its source
//    (Mod_Sources.f90:465-622), forms R = (R/vol + S) dt (Lib_Residual.f90:147-156) and applies the
//    RK stage in conservative variables with the reference's floors (Lib_Newstate.f90:198-219).
#pragma once
#include "ice_kernels.cuh"
#include "ice_tma.cuh"

namespace ice {

constexpr int ST_KZ = 32;                       // planes per tile chunk at most

// The tile limits of a closure: NT threads, so w h <= NT owned cells; at most MAXW owned columns and
// MAXH owned rows; a staged plane of at most MAXBOX positions per variable (bx by, bx = w + 5 rounded
// up to even: two halo columns on either side and one for the even x start of the TMA box; by = h + 4).
// AG's twelve variables take 192 threads, so that two CTAs fit an SM; MK and IG take 256.
template <int CL> struct Shape {
  static constexpr int NT = CL == AG ? 192 : 256;
  static constexpr int MAXW = CL == AG ? 32 : 64;
  static constexpr int MAXH = CL == AG ? 24 : 64;
  static constexpr int MAXBOX = CL == AG ? 360 : 560;
  static constexpr int FX = NT + MAXH;          // x-face slots: h (w + 1)
  static constexpr int FY = NT + MAXW;          // y-face slots: (h + 1) w
  static constexpr int SXC = NT + 2 * MAXH;     // x-slope slots: h (w + 2), the FP32-flux form's cell slopes
  static constexpr int SYC = NT + 2 * MAXW;     // y-slope slots: (h + 2) w
};
__host__ __device__ constexpr int st_box_x(int w) { return (w + 6) & ~1; }

__host__ __device__ constexpr size_t st_align(size_t n) { return (n + 127) & ~(size_t)127; }

template <int CL, typename R> struct StageSmem {
  static constexpr int nc = NC<CL>::v, P = Shape<CL>::MAXBOX;
  static constexpr size_t stg = 0;                                          // double [nc][bx by]
  static constexpr size_t ring = st_align(stg + sizeof(double) * nc * P);  // R [3][nc][P]
  static constexpr size_t fx = st_align(ring + sizeof(R) * 3 * nc * P);    // R [nc][FX]
  static constexpr size_t fy = st_align(fx + sizeof(R) * nc * Shape<CL>::FX);   // R [nc][FY]
  static constexpr size_t bt = st_align(fy + sizeof(R) * nc * Shape<CL>::FY);   // R [2][P]: beta of planes k, k+1
  static constexpr size_t bar = st_align(bt + sizeof(R) * 2 * P);          // mbarrier
  static constexpr size_t bytes = bar + 16 + 128;   // + the alignment of the base to 128 bytes
  // the FP32-flux form's cell slopes of a plane live in the staging buffer while no copy is in flight:
  // R [nc][SXC] x slopes, R [nc][SYC] y slopes, R [SXC + SYC] half lengths, u8 [SXC + SYC] first-order flags
  static constexpr int SXC = Shape<CL>::SXC, SYC = Shape<CL>::SYC;
  static constexpr size_t slope_bytes = (sizeof(R) * (nc + 1) + 1) * (size_t)(SXC + SYC);
  static_assert(sizeof(R) == 8 || slope_bytes <= sizeof(double) * nc * P, "the cell slopes must fit the staging buffer");
};

// The limited slope of cell c along one direction, before the face's limval: q(s, v) reads the cells
// c-1, c, c+1 (s = 0, 1, 2); lm, l0, lp are their lengths after the injection rule. It is the `sl`
// that state_reconstruction computes for the left state of the face above c and the `sr` it
// computes for the right state of the face below c (the two are the same expression). `first` is
// the first-order test of either side (density at or below rho_empty in one of the three cells).
template <int CL, int LIM, typename R, typename Q>
__device__ __forceinline__ void cell_slope(int lim, const Q& q, R lm, R l0, R lp, R* s, R& dlc, bool& first) {
  constexpr int nc = NC<CL>::v;
  const R dlb = (R)0.5*(lm + l0), dlf = (R)0.5*(l0 + lp);
  dlc = (R)0.5*l0;
  R cx, cy;
  if (dlc > (R)0) { cx = dlf/dlc; cy = dlb/dlc; } else { cx = (R)2; cy = (R)2; }
  const R re = (R)kRhoEmpty;
  first = q(0, 0) <= re || q(1, 0) <= re || q(2, 0) <= re;
  R ib = (R)1, iff = (R)1;        // FP32-flux form: reciprocals of the two lengths once per cell
  if constexpr (sizeof(R) == 4) { ib = rcp_fast(dlb); iff = rcp_fast(dlf); }
#pragma unroll
  for (int v = 0; v < nc; ++v) {
    const R a = q(1, v);
    const R sf = sizeof(R) == 4 ? (q(2, v) - a) * iff : (q(2, v) - a) / dlf;
    const R sb = sizeof(R) == 4 ? (a - q(0, v)) * ib : (a - q(0, v)) / dlb;
    s[v] = first ? (R)0 : limiter<LIM>(lim, sf, sb, cx, cy);
  }
}

// The two states of a face from its cells' limited slopes, with state_reconstruction's fallback:
// the weight halves until both states are physical, and the first-order states are taken below
// 1e-18 (Lib_Reconstruction.f90:40-76). Returns true when the first-order states are unphysical.
template <int CL, typename R, typename QL, typename QR>
__device__ __forceinline__ bool states_from_slopes(const QL& ql, const R* sl, R dll, bool fl,
                                                   const QR& qr, const R* sr, R dlr, bool fr, R beta,
                                                   R* pl, R* pr) {
  constexpr int nc = NC<CL>::v;
  R limval = beta;
#pragma unroll
  for (int v = 0; v < nc; ++v) { pl[v] = ql[v]; pr[v] = qr[v]; }
  bool st_l = fl, st_r = fr;
  for (int pass = 0; (!st_l || !st_r) && pass < 256; ++pass) {
    if (pass == 255) limval = (R)0;
#pragma unroll
    for (int v = 0; v < nc; ++v) {
      if (!fl) pl[v] = ql[v] + (sl[v]*limval)*dll;
      if (!fr) pr[v] = qr[v] - (sr[v]*limval)*dlr;
    }
    if (!fl) st_l = check_prim<CL>(pl);
    if (!fr) st_r = check_prim<CL>(pr);
    limval = (R)0.5*limval;
    if (limval < (R)1e-18 && !(st_l && st_r)) {
#pragma unroll
      for (int v = 0; v < nc; ++v) { pl[v] = ql[v]; pr[v] = qr[v]; }
      if (!(check_prim<CL>(pl) && check_prim<CL>(pr))) return true;
      break;
    }
  }
  return false;
}

template <typename S> struct SmemStencil {     // q(s, v): stencil cell s of a staged plane, np positions a variable
  const S* P; int base, st, np;
  __device__ __forceinline__ S operator()(int s, int v) const { return P[v * np + base + s * st]; }
};

template <typename S> struct SmemCell {        // c[v]: one cell of a staged plane
  const S* P; int pos, np;
  __device__ __forceinline__ S operator[](int v) const { return P[v * np + pos]; }
};

// One interior face along d (0: x, 1: y) between the 0-based cells (i,j,k) and its upper neighbour,
// its four-cell stencil from a staged plane (base = the position of cell c - 1), bf the smaller of the
// two cells' Jameson weights: face_flux + compute_flux_ (Mod_Fluxes.f90:599-685).
template <int CL, int RS, int LIM, typename R>
__device__ __forceinline__ bool face_flux_staged(const Geo& G, const FamDev& F, const DBlock& B, int d,
                                                 int i, int j, int k, const R* P, int np, int base, int st, R bf,
                                                 R* flux) {
  constexpr int nc = NC<CL>::v;
  const int c = d == 0 ? i : j;
  const int n = d == 0 ? B.ni : B.nj;
  const long long r0 = ridx(B, i, j, k);
  const long long rs = d == 0 ? 1LL : (long long)(B.ni + 2);
  R l0, l1, l2, l3;
  if constexpr (sizeof(R) == 4) {
    const float* dl = G.dlf + (long long)d * G.NR;
    l0 = dl[r0 - rs]; l1 = dl[r0]; l2 = dl[r0 + rs]; l3 = dl[r0 + 2 * rs];
  } else {
    const double* dl = G.dl + (long long)d * G.NR;
    l0 = dl[r0 - rs]; l1 = dl[r0]; l2 = dl[r0 + rs]; l3 = dl[r0 + 2 * rs];
  }
  if (c == 0 || c == n - 2) {
    const long long gs = gstride(B, d);
    const long long g0 = gidx(B, i, j, k) - gs;
    if (c == 0 && F.inj[g0]) l0 = (R)0;
    if (c == n - 2 && F.inj[g0 + 3 * gs]) l3 = (R)0;
  }
  R dl0 = (R)0.5*(l0 + l1), dl1 = (R)0.5*(l1 + l2), dl2 = (R)0.5*(l2 + l3);
  R dll = (R)0.5*l1, dlr = (R)0.5*l2;
  R pl[nc], pr[nc], fl[nc];
  SmemStencil<R> q{P, base, st, np};
  const bool bad = reconstruct<CL, LIM, R>(F.limiter, q, dl0, dl1, dl2, dll, dlr, pl, pr, bf);
  const long long fi = fidx(B, d, i, j, k, c + 1);
  R nrm[3], area;
  face_geometry<R>(G, d, fi, nrm, area);
  riemann<CL, RS, R>(pl, pr, nrm, fl, (R)F.mat.cp);
#pragma unroll
  for (int v = 0; v < nc; ++v) flux[v] = fl[v] * area;
  return bad;
}

// A hint to bring the cache line of p (a valid address of global memory) into L1; nothing waits on it.
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" :: "l"((unsigned long long)__cvta_generic_to_global(p)));
}

// The stage kernel (see the head of this file). write_r: store R instead of updating (IRS runs).
template <int CL, int RS, int LIM, typename R>
__global__ void __launch_bounds__(Shape<CL>::NT, (sizeof(R) == 4) ? 2 : 1)
k_stage3(Geo G, FamDev F, const CUtensorMap* __restrict__ maps, const Tile* __restrict__ tiles, int write_r,
         Status* st) {
  constexpr int nc = NC<CL>::v;
  constexpr int NT = Shape<CL>::NT, RSLOT = nc * Shape<CL>::MAXBOX;
  constexpr int FX = Shape<CL>::FX, FY = Shape<CL>::FY;
  using L = StageSmem<CL, R>;
  extern __shared__ __align__(128) unsigned char smdyn[];
  // the TMA destination must sit on a 128-byte boundary: align the base explicitly
  unsigned char* smraw = smdyn + ((128u - (smem_u32(smdyn) & 127u)) & 127u);
  double* stg = (double*)(smraw + L::stg);
  R* ring = (R*)(smraw + L::ring);
  R* Fx = (R*)(smraw + L::fx);
  R* Fy = (R*)(smraw + L::fy);
  R* BT = (R*)(smraw + L::bt);
  uint64_t* bar = (uint64_t*)(smraw + L::bar);

  const Tile t = tiles[blockIdx.x];
  const DBlock B = G.blk[t.b];
  const CUtensorMap* map = maps + t.b;
  const int tid = threadIdx.x;
  const int w = t.w, h = t.h, bx = t.bx, np = t.bx * t.by;   // owned columns and rows; staged row and plane
  const bool ax = B.ni >= 2, ay = B.nj >= 2, az = B.nk >= 2;
  const bool own = tid < w * h;
  const int tx = own ? tid % w : 0, ty = own ? tid / w : 0;
  const int i = t.i0 + tx, j = t.j0 + ty;
  const int xa = t.i0 & ~1;                      // staged box start (ghost-inclusive x of cell i0 - 2, made even)
  const int sh = t.i0 - xa;
  auto spos = [&](int cx, int cy) { return (cy + 2) * bx + cx + 2 + sh; };   // tile cell (cx, cy) in a plane
  const int pos = spos(tx, ty);
  const int k0 = t.k0, k1 = t.k0 + t.nkz;
  const bool u0p = F.U0 == F.Up;                // the first RK stage: U_0 is the stencil state itself
  const uint32_t box_bytes = (uint32_t)(sizeof(double) * nc * np);

  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    prefetch_tmap(map);
  }
  __syncthreads();
  uint32_t parity = 0;
  auto issue = [&](int kp) {                    // plane kp (cell index) into the staging buffer
    if (tid == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(bar, box_bytes);
      tma_load_4d(stg, map, bar, xa, t.j0, kp + 2, 0);
    }
  };
  // Waits for the staged plane and converts it into a ring slot. False, for every thread of the CTA,
  // when a wait gave up: the threads that gave up wait once more (bounded) for the copy in flight,
  // and the caller leaves the tile with the timeout bit set.
  auto land = [&](int slot) -> bool {
    const bool ok = mbar_wait(bar, parity);
    if (__syncthreads_or(!ok)) {
      if (!ok) mbar_wait(bar, parity);
      return false;
    }
    parity ^= 1u;
    R* dst = ring + slot * RSLOT;
    for (int q = tid; q < nc * np; q += NT) dst[q] = (R)stg[q];
    __syncthreads();
    return true;
  };
  auto stall = [&]() { if (tid == 0) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_TIMEOUT); };
  auto plane = [&](int slot) { return (const R*)(ring + slot * RSLOT); };

  // The Jameson sensor from the staged densities (compute_beta, Mod_Fluxes.f90:366-389): the weight of
  // the tile cell (cx, cy) on the plane of ring slot s0, with the planes below and above in slots sm
  // and sp; in 2-D runs (no z march) the planes below and above are the ghost planes, read from
  // global memory.
  auto rho_at = [&](int slot, int cx, int cy) { return plane(slot)[spos(cx, cy)]; };
  auto beta_at = [&](int sm, int s0, int sp, int cx, int cy, int kc) -> R {
    R zm, zp;
    if (az) { zm = rho_at(sm, cx, cy); zp = rho_at(sp, cx, cy); }
    else {
      const long long gc = gidx(B, t.i0 + cx, t.j0 + cy, kc);
      zm = (R)F.Up[gc - B.pxy]; zp = (R)F.Up[gc + B.pxy];
    }
    return sd_rho<R>(rho_at(s0, cx, cy), rho_at(s0, cx - 1, cy), rho_at(s0, cx + 1, cy),
                     rho_at(s0, cx, cy - 1), rho_at(s0, cx, cy + 1), zm, zp);
  };
  // the weights of a whole plane's face cells (columns -1..w, rows -1..h) into BT[b]
  const int nbx = w + 2, nb = (w + 2) * (h + 2);
  auto beta_plane = [&](int b, int sm, int s0, int sp, int kc) {
    if (!F.sd) return;
    for (int e = tid; e < nb; e += NT) BT[b * Shape<CL>::MAXBOX + e] = beta_at(sm, s0, sp, e % nbx - 1, e / nbx - 1, kc);
  };
  auto beta_of = [&](int b, int cx, int cy) {
    return F.sd ? BT[b * Shape<CL>::MAXBOX + (cy + 1) * nbx + cx + 1] : (R)1;
  };
  int bcur = 0;

  // z: slope of the thread's cell at plane c from three ring slots (c-1, c, c+1)
  R sz[nc], flo[nc], fhi[nc];
  R dlz = (R)0;
  bool fz = true;
  bool bad = false;
  auto zslope = [&](int sm, int s0, int sp, int c, R* s, R& dlc, bool& first) {
    const long long r0 = ridx(B, i, j, c);
    const long long rs = (long long)(B.ni + 2) * (B.nj + 2);
    R lm, l0, lp;
    if constexpr (sizeof(R) == 4) {
      const float* dl = G.dlf + 2 * G.NR;
      lm = dl[r0 - rs]; l0 = dl[r0]; lp = dl[r0 + rs];
    } else {
      const double* dl = G.dl + 2 * G.NR;
      lm = dl[r0 - rs]; l0 = dl[r0]; lp = dl[r0 + rs];
    }
    const long long g = gidx(B, i, j, c);
    if (c == 0 && F.inj[g - B.pxy]) lm = (R)0;
    if (c == B.nk - 1 && F.inj[g + B.pxy]) lp = (R)0;
    const R* Pm = plane(sm); const R* P0 = plane(s0); const R* Pp = plane(sp);
    auto q = [&](int s, int v) { return (s == 0 ? Pm : s == 1 ? P0 : Pp)[v * np + pos]; };
    cell_slope<CL, LIM, R>(F.limiter, q, lm, l0, lp, s, dlc, first);
  };
  // z face between c and c + 1 from the ring slots of the two cells and their slopes
  auto zface = [&](int sl, int sr, int c, const R* sa, R da, bool fa, const R* sb, R db, bool fb, R bf, R* out) {
    R pl[nc], pr[nc];
    const long long fi = fidx(B, 2, i, j, c, c + 1);
    R nrm[3], area;
    face_geometry<R>(G, 2, fi, nrm, area);
    const SmemCell<R> ql{plane(sl), pos, np}, qr{plane(sr), pos, np};
    bad |= states_from_slopes<CL, R>(ql, sa, da, fa, qr, sb, db, fb, bf, pl, pr);
    R fl[nc];
    riemann<CL, RS, R>(pl, pr, nrm, fl, (R)F.mat.cp);
#pragma unroll
    for (int v = 0; v < nc; ++v) out[v] = fl[v] * area;
  };

  // prologue: the ring holds planes k0, k0+1, k0+2; sz the slope at k0; flo the face below k0
  // (z work is done for the owned cells only: no other thread reads a z face)
  int cur, nx1, nx2;
  if (!az) {
    issue(k0);
    if (!land(0)) { stall(); return; }
    cur = 0; nx1 = 1; nx2 = 2;
    beta_plane(bcur, 0, 0, 0, k0);
    __syncthreads();
  } else if (k0 >= 1) {
    issue(k0 - 2);
    if (!land(0)) { stall(); return; }
    issue(k0 - 1);
    if (!land(1)) { stall(); return; }
    issue(k0);
    if (!land(2)) { stall(); return; }
    R sm1[nc]; R dm1 = (R)0; bool fm1 = true;
    R bm1 = (R)1;
    if (own) {
      zslope(0, 1, 2, k0 - 1, sm1, dm1, fm1);
      if (F.sd) bm1 = beta_at(0, 1, 2, tx, ty, k0 - 1);
    }
    issue(k0 + 1);
    __syncthreads();                            // slot 0 (plane k0-2) is read by every thread before reuse
    if (!land(0)) { stall(); return; }
    beta_plane(bcur, 1, 2, 0, k0);
    if (own) {
      zslope(1, 2, 0, k0, sz, dlz, fz);
      const R b0 = F.sd ? beta_at(1, 2, 0, tx, ty, k0) : (R)1;
      zface(1, 2, k0 - 1, sm1, dm1, fm1, sz, dlz, fz, mn(bm1, b0), flo);
    }
    issue(k0 + 2);
    __syncthreads();
    if (!land(1)) { stall(); return; }
    cur = 2; nx1 = 0; nx2 = 1;
  } else {
    issue(-1);
    if (!land(0)) { stall(); return; }
    issue(0);
    if (!land(1)) { stall(); return; }
    issue(1);
    if (!land(2)) { stall(); return; }
    if (own) zslope(0, 1, 2, 0, sz, dlz, fz);
    beta_plane(bcur, 0, 1, 2, 0);
    issue(2);
    __syncthreads();
    if (!land(0)) { stall(); return; }
    cur = 1; nx1 = 2; nx2 = 0;
  }

  // the extra face tasks of a plane: the x faces above the last column (rows 0..h-1), then the y faces
  // above the last row (columns 0..w-1), where they are interior faces of the block
  const int nhx = (ax && t.i0 + w < B.ni) ? h : 0;
  const int nhy = (ay && t.j0 + h < B.nj) ? w : 0;
  // the face tasks: x and y faces below the owned cells (none along a direction with one cell), extras
  const int nxo = ax ? w * h : 0, nyo = ay ? w * h : 0;
  const int nfx = nxo + nyo + nhx + nhy;
  // face task e: the face below tile cell (cx, cy) along d; false for a face on the block's boundary
  auto face_task = [&](int e, int& d, int& cx, int& cy) -> bool {
    if (e < nxo + nyo) {
      d = e >= nxo;
      const int c = e - (d ? nxo : 0);
      cx = c % w; cy = c / w;
      return d == 0 ? t.i0 + cx != 0 : t.j0 + cy != 0;
    }
    if (e < nxo + nyo + nhx) { d = 0; cx = w; cy = e - nxo - nyo; }
    else { d = 1; cx = e - nxo - nyo - nhx; cy = h; }
    return true;
  };

  // The FP32-flux form computes each cell's limited x and y slopes once per plane (the slope that
  // state_reconstruction computes for the left state of the face above the cell and for the right
  // state of the face below it: the same operands and operations, so the same values) into the
  // staging buffer, and the faces form their states from them; the next plane's copy into that buffer
  // is then issued once the faces are done. The plain form reconstructs each face from its stencil.
  constexpr bool SL = sizeof(R) == 4;
  constexpr int SXC = Shape<CL>::SXC, SYC = Shape<CL>::SYC;
  R* SX = (R*)stg;                              // [nc][SXC]: tile cell (cx, cy), cx in -1..w: cy (w + 2) + cx + 1
  R* SY = SX + nc * SXC;                        // [nc][SYC]: cy in -1..h: (cy + 1) w + cx
  R* DX = SY + nc * SYC;                        // the cells' half lengths along x, then along y
  R* DY = DX + SXC;
  unsigned char* QX = (unsigned char*)(DY + SYC);   // the first-order flags along x, then along y
  unsigned char* QY = QX + SXC;
  const int sxw = w + 2;
  const int nsx = ax ? sxw * h : 0, nsy = ay ? w * (h + 2) : 0;

  for (int k = k0; k < k1; ++k) {
    const bool more = k + 1 < k1;
    if constexpr (!SL) {
      if (more) issue(k + 3);                   // lands at the end of this plane, into the slot of k
    }
    const R* P = plane(cur);
    if (own) {
      // the global operands of this plane's update and z face into L1 while the plane's slopes and faces
      // are computed: the kernel waits on global loads more than on anything else
      const long long gq = gidx(B, i, j, k), qq = iidx(B, i, j, k);
#pragma unroll
      for (int v = 0; v < nc; ++v) {
        prefetch_l1(F.Up + (long long)v * G.NG + gq);
        if (!u0p) prefetch_l1(F.U0 + (long long)v * G.NG + gq);
      }
      if (F.coupled && F.src_ready) {
        if (F.Sf) { for (int v = 0; v < nc; ++v) prefetch_l1(F.Sf + (long long)v * G.NI + qq); }
      } else if (F.coupled) {
        if constexpr (sizeof(R) == 4) { for (int v = 0; v < 9; ++v) prefetch_l1(G.gasf + (long long)v * G.NI + qq); }
      }
      prefetch_l1(G.vol + qq); prefetch_l1(F.bmap + qq);
      if constexpr (sizeof(R) == 4) {
        if (az && k <= B.nk - 2) {
          const long long r1 = ridx(B, i, j, k + 1), rs = (long long)(B.ni + 2) * (B.nj + 2);
          prefetch_l1(G.dlf + 2 * G.NR + r1 + rs);
          prefetch_l1(G.ff[2] + fidx(B, 2, i, j, k, k + 1));
        }
      }
    }
    if constexpr (SL) {
      // the cell slopes of this plane: along x for the columns -1..w, along y for the rows -1..h, of
      // the cells inside the block (the others border no interior face of the tile)
      for (int e = tid; e < nsx + nsy; e += NT) {
        int d, cx, cy, idx;
        if (e < nsx) { d = 0; cx = e % sxw - 1; cy = e / sxw; idx = e; }
        else { d = 1; idx = e - nsx; cx = idx % w; cy = idx / w - 1; }
        const int ci = d == 0 ? t.i0 + cx : t.j0 + cy, n = d == 0 ? B.ni : B.nj;
        if (ci < 0 || ci >= n) continue;
        const int ic = t.i0 + cx, jc = t.j0 + cy;
        const long long r0 = ridx(B, ic, jc, k);
        const long long rs = d == 0 ? 1LL : (long long)(B.ni + 2);
        const float* dl = G.dlf + (long long)d * G.NR;
        R lm = dl[r0 - rs], l0 = dl[r0], lp = dl[r0 + rs];
        if (ci == 0 || ci == n - 1) {
          const long long g = gidx(B, ic, jc, k), gs = gstride(B, d);
          if (ci == 0 && F.inj[g - gs]) lm = (R)0;
          if (ci == n - 1 && F.inj[g + gs]) lp = (R)0;
        }
        const int st1 = d == 0 ? 1 : bx;
        const SmemStencil<R> q{P, spos(cx, cy) - st1, st1, np};
        R s[nc], dlc; bool first;
        cell_slope<CL, LIM, R>(F.limiter, q, lm, l0, lp, s, dlc, first);
        R* S = d == 0 ? SX : SY;
        const int cap = d == 0 ? SXC : SYC;
#pragma unroll
        for (int v = 0; v < nc; ++v) S[v * cap + idx] = s[v];
        (d == 0 ? DX : DY)[idx] = dlc;
        (d == 0 ? QX : QY)[idx] = first ? 1 : 0;
      }
      // and the next plane's Jameson weights (planes k, k+1, k+2 are in the ring), which the z face reads
      // after this barrier
      if (az && k <= B.nk - 2) beta_plane(bcur ^ 1, cur, nx1, nx2, k + 1);
      __syncthreads();
    }
    // the x and y faces of this plane, each once, as one list of tasks dealt out to the threads in turn:
    // the x face below every owned cell, the y face below every owned cell, then the x faces above the
    // last column and the y faces above the last row (a face on the block's boundary is its records')
    for (int e = tid; e < nfx; e += NT) {
      int d, cx, cy;
      if (!face_task(e, d, cx, cy)) continue;
      // the face below tile cell (cx, cy) along d: its lower cell, stencil and the two cells' weights
      const int lx = cx - (d == 0), ly = cy - (d == 1);
      const int sst = d == 0 ? 1 : bx;
      const R bf = mn(beta_of(bcur, lx, ly), beta_of(bcur, cx, cy));
      R fl[nc];
      if constexpr (SL) {
        // the states from the two cells' slopes, then the flux
        const int il = d == 0 ? cy * sxw + cx : cy * w + cx, iu = il + (d == 0 ? 1 : w);
        const R* S = d == 0 ? SX : SY;
        const int cap = d == 0 ? SXC : SYC;
        const R* D = d == 0 ? DX : DY;
        const unsigned char* Q = d == 0 ? QX : QY;
        R sl[nc], sr[nc], pl[nc], pr[nc];
#pragma unroll
        for (int v = 0; v < nc; ++v) { sl[v] = S[v * cap + il]; sr[v] = S[v * cap + iu]; }
        const int c = d == 0 ? t.i0 + lx : t.j0 + ly;
        const long long fi = fidx(B, d, t.i0 + lx, t.j0 + ly, k, c + 1);
        R nrm[3], area;
        face_geometry<R>(G, d, fi, nrm, area);
        const SmemCell<R> ql{P, spos(lx, ly), np}, qr{P, spos(cx, cy), np};
        bad |= states_from_slopes<CL, R>(ql, sl, D[il], Q[il] != 0, qr, sr, D[iu], Q[iu] != 0, bf, pl, pr);
        riemann<CL, RS, R>(pl, pr, nrm, fl, (R)F.mat.cp);
#pragma unroll
        for (int v = 0; v < nc; ++v) fl[v] = fl[v] * area;
      } else {
        bad |= face_flux_staged<CL, RS, LIM, R>(G, F, B, d, t.i0 + lx, t.j0 + ly, k, P, np, spos(cx, cy) - 2 * sst,
                                                sst, bf, fl);
      }
      R* dst = d == 0 ? Fx + cy * (w + 1) + cx : Fy + cy * w + cx;
      const int vs = d == 0 ? FX : FY;
#pragma unroll
      for (int v = 0; v < nc; ++v) dst[v * vs] = fl[v];
    }
    // z: the face above the cell, from the slopes at k (carried) and k + 1
    R szn[nc]; R dlzn = (R)0; bool fzn = true;
    if (az && own && k <= B.nk - 2) {
      zslope(cur, nx1, nx2, k + 1, szn, dlzn, fzn);
      const R b1 = SL ? beta_of(bcur ^ 1, tx, ty) : (F.sd ? beta_at(cur, nx1, nx2, tx, ty, k + 1) : (R)1);
      zface(cur, nx1, k, sz, dlz, fz, szn, dlzn, fzn, mn(beta_of(bcur, tx, ty), b1), fhi);
    }
    // the next plane's weights (its planes below and above are in the ring now), read after a barrier
    if (!SL && az && more) beta_plane(bcur ^ 1, cur, nx1, nx2, k + 1);
    if constexpr (SL) fence_proxy_async_smem();   // this thread's slope accesses before the copy that overwrites them
    __syncthreads();
    if constexpr (SL) {
      if (more) issue(k + 3);                   // lands at the end of this plane, into the slot of k
    }
    if (own) {
      const long long q = iidx(B, i, j, k);
      const int bc = F.bmap[q];
      // the cell's residual, summed in the reference's order: in FP64 in the plain form, in FP32
      // (the type of the fluxes) in the FP32-flux form
      using A = R;
      A r[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v) r[v] = bc >= 0 ? (A)F.Rb[(long long)bc * nc + v] : (A)0;
      if (ax) {
        const int ci = i + 1, n = B.ni;
        const int lo = ty * (w + 1) + tx;
        if (ci % 2 == 1) {
          if (ci < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - (A)Fx[v * FX + lo + 1];
          }
          if (ci > 1) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] + (A)Fx[v * FX + lo];
          }
        } else {
#pragma unroll
          for (int v = 0; v < nc; ++v) r[v] = r[v] + (A)Fx[v * FX + lo];
          if (ci < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - (A)Fx[v * FX + lo + 1];
          }
        }
      }
      if (ay) {
        const int cj = j + 1, n = B.nj;
        const int lo = ty * w + tx;
        if (cj % 2 == 1) {
          if (cj < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - (A)Fy[v * FY + lo + w];
          }
          if (cj > 1) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] + (A)Fy[v * FY + lo];
          }
        } else {
#pragma unroll
          for (int v = 0; v < nc; ++v) r[v] = r[v] + (A)Fy[v * FY + lo];
          if (cj < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - (A)Fy[v * FY + lo + w];
          }
        }
      }
      if (az) {
        const int ck = k + 1, n = B.nk;
        if (ck % 2 == 1) {
          if (ck < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - (A)fhi[v];
          }
          if (ck > 1) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] + (A)flo[v];
          }
        } else {
#pragma unroll
          for (int v = 0; v < nc; ++v) r[v] = r[v] + (A)flo[v];
          if (ck < n) {
#pragma unroll
            for (int v = 0; v < nc; ++v) r[v] = r[v] - (A)fhi[v];
          }
        }
      }
      const long long g = gidx(B, i, j, k);
      double p[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v) p[v] = F.Up[(long long)v * G.NG + g];
      double s[nc];
#pragma unroll
      for (int v = 0; v < nc; ++v) s[v] = 0.0;
      if (F.coupled && F.src_ready) {           // a source kernel ran first (evaporating family or surrogate)
#pragma unroll
        for (int v = 0; v < nc; ++v) s[v] = F.Sf ? (double)F.Sf[(long long)v * G.NI + q] : F.S[(long long)v * G.NI + q];
      } else if (F.coupled) {                   // compute_source_ on the stage's state
        R pr_[nc], gas[5], sr[nc];
#pragma unroll
        for (int v = 0; v < nc; ++v) pr_[v] = (R)p[v];
#pragma unroll
        R gr[9];
#pragma unroll
        for (int v = 0; v < 9; ++v) gr[v] = sizeof(R) == 4 ? (R)G.gasf[(long long)v * G.NI + q] : (R)G.gas[(long long)v * G.NI + q];
#pragma unroll
        for (int v = 0; v < 5; ++v) gas[v] = gr[v];
        R tau = cell_source<CL, R>(pr_, gas, gr[5], gr[6], gr[7], gr[8], F.mat, F.drag, F.heat, F.blow, sr);
#pragma unroll
        for (int v = 0; v < nc; ++v) s[v] = (F.frozen_mask & (1u << v)) ? 0.0 : (double)sr[v];
        if (F.write_tau) F.tau[q] = (double)tau;
      }
      if (F.xstep) accumulate_source<CL>(F.xstep, G.NI, q, s, F.xfirst, F.rk);
      const double dt = F.dt ? F.dt[q] : *F.dtg;
      const double vol = G.vol[q];
      double rd[nc];
      if constexpr (sizeof(R) == 8) {
#pragma unroll
        for (int v = 0; v < nc; ++v) rd[v] = (r[v]/vol + s[v]) * dt;
      } else {
        const double ivol = 1.0 / vol;
#pragma unroll
        for (int v = 0; v < nc; ++v) rd[v] = ((double)r[v]*ivol + s[v]) * dt;
      }
      if (F.imports) {                          // add_births (Lib_Residual.f90:164-210): the coupler's rates
#pragma unroll
        for (int v = 0; v < nc; ++v) rd[v] = rd[v] + F.imports[(long long)v * G.NI + q] * dt;
      }
#pragma unroll
      for (int v = 0; v < nc; ++v) if (F.frozen_mask & (1u << v)) rd[v] = 0.0;
      if (write_r) {
#pragma unroll
        for (int v = 0; v < nc; ++v) F.resid[(long long)v * G.NI + q] = rd[v];
      } else {
        double po[nc], co[nc], cn[nc];
#pragma unroll
        for (int v = 0; v < nc; ++v) po[v] = u0p ? p[v] : F.U0[(long long)v * G.NG + g];
        prim2cons<CL, double>(po, co, F.mat.cp);
        prim2cons<CL, double>(p, cn, F.mat.cp);
#pragma unroll
        for (int v = 0; v < nc; ++v) { double rr = (cn[v] - co[v] + rd[v]) * F.rk; cn[v] = co[v] + rr; }
        if (cn[0] < 0.0) atomicAdd(&st->nfloored, 1ULL);
        cons2prim<CL, sizeof(R) == 4>(cn, p, F.mat.cp);
        if constexpr (sizeof(R) == 4) {
          if (F.realize && realize<CL>(p)) atomicAdd(&st->nrealized, 1ULL);
        }
        if (!check_prim<CL, double>(p)) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_NAN_STATE);
#pragma unroll
        for (int v = 0; v < nc; ++v) F.Uo[(long long)v * G.NG + g] = p[v];
      }
    }
    if (!more) break;
    // plane k + 3 replaces plane k in the ring: nothing reads plane k after the barrier above, so
    // each thread converts its share as soon as its own update is done; one barrier then both
    // publishes the slot and agrees on a wait that gave up (the next plane's faces overwrite Fx and
    // Fy only after it, when every owner has gathered its fluxes).
    {
      const bool ok = mbar_wait(bar, parity);
      if (ok) {
        R* dst = ring + cur * RSLOT;
        for (int e = tid; e < nc * np; e += NT) dst[e] = (R)stg[e];
      }
      if (__syncthreads_or(!ok)) {
        if (!ok) mbar_wait(bar, parity);
        stall();
        break;
      }
      parity ^= 1u;
    }
    const int o = cur; cur = nx1; nx1 = nx2; nx2 = o;
    bcur ^= 1;
#pragma unroll
    for (int v = 0; v < nc; ++v) { flo[v] = fhi[v]; sz[v] = szn[v]; }
    dlz = dlzn; fz = fzn;
  }
  if (bad) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_BAD_RECON);
}

}  // namespace ice
