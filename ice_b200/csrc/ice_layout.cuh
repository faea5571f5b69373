// ice_layout.cuh -- the device layout of the solve stage: blocks, geometry, records, status,
// the per-family view the kernels read, and the launch interface of the per-closure units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include "ice_physics.cuh"

namespace ice {


// ------------------------------------------------------------------ device layout
struct DBlock {
  int ni, nj, nk;
  int px;             // row pitch of the ghost-cell pools: ni + 4 rounded up to even, so that every row,
                      // plane and block starts on a 16-byte boundary (the TMA tensor maps need it)
  long long pxy;      // plane pitch, px * (nj + 4)
  long long goff;     // ghost-cell pools (1-gc:n+gc)^3
  long long ioff;     // interior pools
  long long roff;     // ring pools (0:n+1)^3
  long long foff[3];  // face pools of each direction
};

struct Geo {                 // geometry shared by the families
  const DBlock* blk;
  int nb;
  long long NG, NI, NR, NF[3];
  const double* face[3];     // 4 SoA components (nx, ny, nz, A) of NF[d] each
  const double* vol;         // NI
  const double* dl;          // 3 SoA components of NR
  const double* M;           // 9 SoA components of NI (column-major c(3,3))
  const double* gas;         // 9 SoA components of NI: rho u v w T R gam k mu
  // the FP32-flux form's copies of the face geometry (nx, ny, nz, A of a face in one 16-byte word) and
  // of the cell lengths, rounded once from the FP64 arrays above (null in the plain form)
  const float4* ff[3];
  const float* dlf;
  const float* gasf;         // the FP32-flux form's copy of the frozen gas (coupled runs), rounded once
  // a split run (ice_gpu_set_partition): per block, whether this rank steps it; null when it steps all
  const unsigned char* owned;
};
__device__ __forceinline__ bool stepped(const Geo& G, int b) { return !G.owned || G.owned[b]; }


struct DRec {                // one boundary record, 0-based cells
  int b, i, j, k, f, type;
  int bs, is, js, ks, fs;
  int owner, cf;             // cf 0-based (-1 when none)
  int pb, pi, pj, pk;        // the partner's cell (connections)
  int normal_dir;
  double massflux, velocity, alpha, beta, temperature, radius, gfixed;
  // host-computed once per record (the platform libm of the driver's host, as the
  // reference's ghost_record evaluates them): cos/sin of the inlet angles and 4/3 pi r^3
  double ca, sa, cb, sb, vol_p;
  // chimera (102): donors cd0 .. cd0 + cn1 - 1 of ghost layer 1, then cn2 of layer 2, in the family's
  // donor arrays (FamDev::cdon, cw)
  int cd0, cn1, cn2;
};

struct Status {
  unsigned int flags;
  unsigned int pad;
  unsigned long long nfloored;
  unsigned long long dtbits;  // running min of dt as the bits of a positive double
  double dtglobal;
  double time;
  int iter;
  int iter_from_call;
  unsigned long long sur_cells, sur_env, sur_res;   // surrogate: cells, envelope and check fallbacks
  unsigned long long nrealized;  // cells the chosen form's realizability correction changed
};

__device__ __forceinline__ long long gidx(const DBlock& B, int i, int j, int k) {
  return B.goff + (long long)(k + 2) * B.pxy + (long long)(j + 2) * B.px + (i + 2);
}
__device__ __forceinline__ long long iidx(const DBlock& B, int i, int j, int k) {
  return B.ioff + ((long long)k * B.nj + j) * B.ni + i;
}
__device__ __forceinline__ long long ridx(const DBlock& B, int i, int j, int k) {
  return B.roff + ((long long)(k + 1) * (B.nj + 2) + (j + 1)) * (B.ni + 2) + (i + 1);
}
// face d with Fortran index F (the 1-based index of the cell below it along d), other indices 0-based
__device__ __forceinline__ long long fidx(const DBlock& B, int d, int i, int j, int k, int F) {
  if (d == 0) return B.foff[0] + ((long long)k * B.nj + j) * (B.ni + 1) + F;
  if (d == 1) return B.foff[1] + ((long long)k * (B.nj + 1) + F) * B.ni + i;
  return B.foff[2] + ((long long)F * B.nj + j) * B.ni + i;
}
__device__ __forceinline__ long long gstride(const DBlock& B, int d) {
  return d == 0 ? 1LL : d == 1 ? (long long)B.px : B.pxy;
}

struct FamDev {              // what the kernels of one family read
  int closure, riemann, nc, limiter, sd, coupled, drag, heat, blow;
  unsigned int frozen_mask;  // bit v: slot v+1 frozen
  Mat mat;
  const double* U0;          // pointwise U_0
  const double* Up;          // stencil U_{k-1}
  double* Uo;                // U_k
  double* Ug;                // buffer whose ghosts the ghost kernels fill (== Up)
  unsigned char* inj;
  const double* beta;        // NI, or null (1)
  double* betaw;
  const double* dt;          // NI (steady) or null
  const double* dtg;         // &status->dtglobal (time-accurate)
  double* tau;               // NI
  double* S;                 // [v][NI]: the stage's source (coupled runs)
  float* Sf;                 // the FP32-flux form's source, [v][NI] floats in the same buffer (else null)
  const int* bmap;           // NI: boundary-cell index or -1
  const double* Rb;          // [nbcell][nc]
  double* Rbw;
  double* connF;             // [ncf][nc]
  const int4* cdon;          // chimera donors: 0-based block, i, j, k
  const double* cw;          // chimera donor weights
  const double* imports;     // [v][NI]: the coupler's rates into the cells, or null
  double* xstep;             // [5][NI]: the step's weighted source in slots 1-4 and the energy slot, or null
  int xfirst;                // this stage starts the running sum (stage 1)
  double* resid;             // IRS: [v][NI]
  double rk;
  int write_tau;
  int src_ready;             // S holds this stage's source already (its own kernel or the surrogate's ran)
  int realize;               // the FP32-flux form's realizability correction is on
};

// bound_empty_dt's reductions over one family's cells, as the bits of non-negative doubles (which
// order as their bits): the smallest step of an occupied cell, the smallest step of a source, the
// largest speed per axis, and whether a source fills anything.
struct EmptyScan {
  unsigned long long floor_bits, src_bits, umax_bits[3];
  unsigned int filled, pad;
};

// A column tile of a block and its chunk of nkz planes. The staged stage kernel's tiles also carry
// their owned columns and rows (w, h) and the staged box of their block (bx, by: the TMA box's x and y).
struct Tile { int b, i0, j0, k0, nkz; short w, h, bx, by; };
struct MlpNorm;
struct NormChunk { int b; long long q0, q1; };

// Everything one family's stage needs, for the launcher of its closure's translation unit.
struct LaunchArgs {
  Geo G;
  FamDev F;
  const DRec* recs; int nrec;
  const DRec* grecs;                                 // the records in the ghost kernel's order
  int ghost_split;                                   // a record's second layer reads another's first
  const int* own; int nown;
  const int* bfirst; const int* blist; int nbc;
  const int* bperm;                                  // the boundary cells in the boundary kernel's thread order
  const Tile* tiles; int ntile; int TX, TY, KZ;     // the 1-D stage kernel's tiles
  const Tile* tiles3; int ntile3;                    // the staged stage kernel's tiles (2-D and 3-D runs)
  const CUtensorMap* maps;                           // per block: the TMA map of U_{k-1} (the stencil buffer)
  const unsigned char* mlp_img;                      // the family's surrogate network (null: the plain closure)
  const MlpNorm* mlp_norm;
  int ndir, sd, irs, precision;
  double irs_beta;
  double* resid; double* resid2; double* resid3;
  Status* st;
  cudaStream_t s;
  void (*tick)(void*, int, cudaStream_t);
  void* tick_ctx;
  // a split run: the exchange of one kind (ICE_GPU_HALO_CELLS, BETA, FLUX) of this family at its point
  // of the stage, called on every rank whatever its local work (null when every block is stepped here)
  void (*xchg)(const struct LaunchArgs&, int kind);
  int fam;                                           // 0-based family
};

enum { KC_DT = 0, KC_GHOST, KC_BETA, KC_BOUND, KC_STAGE, KC_IRS, KC_NORM, KC_SOURCE, KC_N };

// the boundary and ghost kernels of a family's stage (ice_fam_<closure>.cu), which call the stage
// kernel of its closure and precision (ice_stage_<closure>_<f64|f32>.cu)
void launch_family_mk(const LaunchArgs& a);
void launch_family_ig(const LaunchArgs& a);
void launch_family_ag(const LaunchArgs& a);
void launch_source_mk_f64(const LaunchArgs& a);
void launch_source_mk_f32(const LaunchArgs& a);
void launch_source_ig_f64(const LaunchArgs& a);
void launch_source_ig_f32(const LaunchArgs& a);
void launch_source_ag_f64(const LaunchArgs& a);
void launch_source_ag_f32(const LaunchArgs& a);
void launch_bound_mk_f64(const LaunchArgs& a);
void launch_bound_mk_f32(const LaunchArgs& a);
void launch_bound_ig_f64(const LaunchArgs& a);
void launch_bound_ig_f32(const LaunchArgs& a);
void launch_bound_ag_f64(const LaunchArgs& a);
void launch_bound_ag_f32(const LaunchArgs& a);
void launch_pack_beta_mk_f64(const LaunchArgs& a, const int4* e, int n, double* out);
void launch_pack_beta_mk_f32(const LaunchArgs& a, const int4* e, int n, double* out);
void launch_pack_beta_ig_f64(const LaunchArgs& a, const int4* e, int n, double* out);
void launch_pack_beta_ig_f32(const LaunchArgs& a, const int4* e, int n, double* out);
void launch_pack_beta_ag_f64(const LaunchArgs& a, const int4* e, int n, double* out);
void launch_pack_beta_ag_f32(const LaunchArgs& a, const int4* e, int n, double* out);
void launch_stage_mk_f64(const LaunchArgs& a, bool write_r);
void launch_stage_mk_f32(const LaunchArgs& a, bool write_r);
void launch_stage_ig_f64(const LaunchArgs& a, bool write_r);
void launch_stage_ig_f32(const LaunchArgs& a, bool write_r);
void launch_stage_ag_f64(const LaunchArgs& a, bool write_r);
void launch_stage_ag_f32(const LaunchArgs& a, bool write_r);

}  // namespace ice
