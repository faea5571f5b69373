// ice_gpu.cu -- the B200 (sm_100a) solve stage of ICE's Eulerian dispersed-phase time step,
// behind the C ABI of include/ice_gpu.h.
//
// One call of ice_gpu_step replaces `call Explicit_Step(grid)` (src/lib/driver/Wrap_Solve.f90:26;
// numerics/time/explicit/Mod_Explicit.f90:11-245). Every array is resident in HBM; a step is a
// CUDA graph of:
//   k_begin        iteration counters, dt reset                      (Mod_Explicit.f90:40-44)
//   k_dt_all       per-cell CFL dt of every family + global min (FP64)  (Mod_dt.f90:11-112,256-275)
//   (k_empty_scan, k_empty_apply for a family with the coupler's imports: Mod_dt.f90:134-242)
//   k_time         dtglobal, time += dt                               (Mod_Explicit.f90:67-73)
//   per family, per RK stage:
//     k_source     the source of an evaporating family (or a 1-D run), or the surrogate's
//                  k_source_mlp                                        (Mod_Sources.f90:465-622)
//     k_ghost      both ghost layers from the record list (two launches, layer 1 then
//                  layer 2, where a block is one cell deep along a record's face), block
//                  connections as on-device copies in one HBM pool    (Lib_Ghost.f90:29-387)
//     k_beta       Jameson sensor (when on; 1-D runs only)            (Mod_Fluxes.f90:366-389)
//     k_conn       connection-face fluxes by their owner records      (Mod_BC_Fluxes.f90:151-170)
//     k_bound      boundary cells, records summed in face order        (Mod_BC_Fluxes.f90:105-144)
//     k_stage3     (k_stage in 1-D runs) interior face fluxes of a tile in shared memory, gathered
//                  per cell in the odd-then-even order (Mod_Fluxes.f90:421-521), fused with the
//                  source of a family without evaporation (Mod_Sources.f90:465-622), the residual
//                  with the coupler's imports (Lib_Residual.f90:147-210) and the RK update with
//                  cons<->prim and the state checks (Lib_Newstate.f90:198-219)
//     (k_irs, k_update when implicit residual smoothing is on: Lib_IRS.f90:34-86)
//
// The state is stored structure-of-arrays, one contiguous array per variable over every block
// of a family (ghost layers included), in three buffers that rotate over the RK stages: the
// stage reads U_{k-1} (stencil) and U_0 (pointwise) and writes U_k, so no state copy
// (state_copy, Lib_Newstate.f90:65-106) and no zeroing of the residual (Lib_Residual.f90:13-41)
// remain: the residual lives in registers.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdarg>
#include <cmath>
#include <vector>
#include <string>
#include <algorithm>
#include <memory>
#include <queue>
#include <functional>
#include "ice_kernels.cuh"
#include "ice_stage3.cuh"
#include "ice_mlp.cuh"
#include "ice_tune.h"
#include "../../include/ice_gpu.h"

using namespace ice;

namespace {

constexpr int kMaxF = ICE_GPU_MAX_FAMILIES;
constexpr int kMaxNC = 12;     // variables of the largest closure (AG)

// ------------------------------------------------------------------ host side
struct HRec {
  int b, i, j, k, f, type, p, bs, is, js, ks, fs, partner, owner, cf;
  double massflux, velocity, alpha, beta, temperature, radius, gfixed, normal_dir;
};

template <typename T> struct DevBuf {
  T* p = nullptr; size_t n = 0;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t count) {
    if (p) { cudaFree(p); p = nullptr; }
    n = count;
    if (count == 0) return cudaSuccess;
    return cudaMalloc((void**)&p, count * sizeof(T));
  }
};

struct FamHost {
  int closure, riemann, nc;
  DevBuf<double> S[3];
  DevBuf<unsigned char> inj;
  DevBuf<double> dt, tau, beta;
  DevBuf<int> bmap;
  DevBuf<double> Rb, connF, resid, resid2, resid3, src;
  DevBuf<DRec> recs;
  DevBuf<DRec> grecs;                        // the same records ordered for the ghost kernel (upload_recs)
  bool ghost_split = false;                  // the ghost layers in two launches (upload_recs)
  DevBuf<int> bfirst, blist, own;
  DevBuf<int> bperm;                         // the boundary cells in the boundary kernel's thread order
  DevBuf<CUtensorMap> maps[3];               // per state buffer, per block: the staged kernel's TMA maps
  DevBuf<Tile> tiles3;                       // the staged kernel's tiles
  int ntile3 = 0;
  std::vector<Tile> shape3;                  // per block: the staged kernel's tile shape (w, h, bx, by)
  // the evaporation surrogate (FP32-flux form): the network's BF16 image, its standardisation and
  // envelope, its FP32 parameters; on = the stage's source comes from the surrogate source kernel
  DevBuf<unsigned char> mlp_img;
  MlpNorm mlp_norm;
  std::vector<float> mlp_w;
  bool sur_on = false;
  int nrec = 0, nbc = 0, nown = 0, ncf = 0;
  std::vector<int> h_first, h_list, h_own;   // 0-based record numbers of the whole table
  std::vector<int> h_grp;                    // the family's records: their numbers in the table
  std::vector<DRec> h_recs;                  // the device records, kept to attach chimera donors
  DevBuf<int4> cdon;                         // chimera donors (0-based block, i, j, k) and weights
  DevBuf<double> cw;
  DevBuf<double> imp;                        // the coupler's imports [v][NI] (ice_gpu_set_imports)
  DevBuf<EmptyScan> escan;                   // bound_empty_dt's reductions
  bool have_imp = false;
  DevBuf<double> xstep;                      // the step's weighted source, slots 1-4 and energy [5][NI]
};


}  // namespace

struct ice_gpu_ctx {
  ice_gpu_params P;
  int nb = 0;
  std::vector<int> dims;
  std::vector<DBlock> hblk;
  long long NG = 0, NI = 0, NR = 0, NF[3] = {0, 0, 0};
  DevBuf<DBlock> blk;
  DevBuf<double> face[3], vol, dl, M, gas;
  DevBuf<float4> facef[3];  // the FP32-flux form's geometry (Geo::ff, dlf), rounded from the FP64 arrays
  DevBuf<float> dlf;
  DevBuf<float> gasf;       // the FP32-flux form's copy of the gas (Geo::gasf)
  bool geo32_ok = false;
  bool have_gas = false;
  std::vector<bool> have_block;
  std::vector<bool> gas_set;     // per block: ice_gpu_set_gas was called
  bool have_records = false;
  bool exchange = false;  // two-way coupling: the step's weighted source is kept for the gas
  int nchim = 0;          // 102 records of the table
  bool have_chimera = true;   // their donors are set (ice_gpu_set_chimera)
  FamHost fam[kMaxF];
  std::vector<HRec> recs;
  DevBuf<Tile> tiles;
  int ntile = 0, TX = 0, TY = 0, KZ = 0;
  bool staged = false;    // 2-D and 3-D runs: the staged stage kernel (ice_stage3.cuh)
  DevBuf<NormChunk> chunks;
  DevBuf<double> npart;
  int nchunk = 0;
  std::vector<int> chunk_block;
  DevBuf<Status> st;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  // ice_gpu_step_host: the step cut into its dt part and one graph per family (per buffer phase), two
  // copy streams, the caller's arrays staged in one device buffer, one event per family
  cudaGraphExec_t graph_pre[3] = {nullptr, nullptr, nullptr};
  cudaGraphExec_t graph_fam[3][kMaxF] = {};
  cudaStream_t s_up = nullptr, s_down = nullptr;
  cudaEvent_t ev_up = nullptr, ev_fam[kMaxF] = {};
  DevBuf<double> xall;
  int phase = 0;          // buffer holding the current state
  int prev_phase = -1;    // buffer holding the state before the last step
  double res_reference = 0.0;  // the first non-zero density residual of a steady run (0: none yet)
  bool res_end = false;        // the last step ended the run on res-threshold
  double last_norm[5] = {0, 0, 0, 0, 0};
  bool profiling = false;
  double kms[KC_N] = {0};
  // the block split (ice_gpu_set_partition, _set_halo, _set_exchange_hook): the blocks this rank steps
  // (empty: all), on the device too; per kind and family the entries sent and received (0-based int4:
  // block, i, j, k; or the connection face in x); the hook and its pinned host buffers
  std::vector<unsigned char> owned;
  DevBuf<unsigned char> owned_dev;
  std::vector<int4> hs[3][kMaxF], hr[3][kMaxF];
  DevBuf<int4> hs_dev[3][kMaxF], hr_dev[3][kMaxF];
  ice_gpu_exchange_fn hook = nullptr;
  void* hook_user = nullptr;
  DevBuf<double> xdev;
  double* xhost = nullptr;
  size_t xhost_n = 0;
  int xerr = 0;                  // the first failure of an exchange of the running call
  unsigned long long xbits = 0;  // the reduced dt on its way back to the device
  long long nlaunch = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevBuf<double> xfer;    // one block of one family in the caller's layout (upload/download)
  long long ng_max = 0;
  std::string err;
};

static std::string g_create_err;

static bool sur_active(const ice_gpu_ctx* c, int p) {
  const FamHost& H = c->fam[p];
  return H.sur_on && H.mlp_img.p && c->P.coupled && c->P.precision == ICE_PREC_FP32FLUX && !c->P.irs;
}

// The caller's prim(nc, -1:ni+2, -1:nj+2, -1:nk+2) (variable fastest) <-> one block of the SoA pool,
// whose rows are px long (the row padding is never read).
__device__ __forceinline__ long long pool_of(long long q, int ni4, int nj4, int px) {
  long long x = q % ni4, r = q / ni4;
  return (r / nj4) * ((long long)px * nj4) + (r % nj4) * px + x;
}
__global__ void k_aos2soa(const double* __restrict__ a, double* __restrict__ s, long long NG, long long n, int nc,
                          int ni4, int nj4, int px) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    long long d = pool_of(q, ni4, nj4, px);
    for (int v = 0; v < nc; ++v) s[(long long)v * NG + d] = a[(long long)nc * q + v];
  }
}
__global__ void k_soa2aos(const double* __restrict__ s, double* __restrict__ a, long long NG, long long n, int nc,
                          int ni4, int nj4, int px) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    long long d = pool_of(q, ni4, nj4, px);
    for (int v = 0; v < nc; ++v) a[(long long)nc * q + v] = s[(long long)v * NG + d];
  }
}
__global__ void k_inj2pool(const unsigned char* __restrict__ a, unsigned char* __restrict__ s, long long n,
                           int ni4, int nj4, int px) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    s[pool_of(q, ni4, nj4, px)] = a[q];
}
static unsigned grid_of(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16); }

static int fail(ice_gpu_ctx* c, int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap; va_start(ap, fmt); vsnprintf(buf, sizeof buf, fmt, ap); va_end(ap);
  if (c) c->err = buf; else g_create_err = buf;
  return code;
}

#define CK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
  return fail(c, ICE_GPU_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); } while (0)

static int nbase_of(int cl) { return cl == ICE_CLOSURE_MK ? 6 : cl == ICE_CLOSURE_IG ? 7 : 12; }

static void free_graphs(ice_gpu_ctx* c) {
  for (auto& g : c->graph) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto& g : c->graph_pre) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto& row : c->graph_fam) for (auto& g : row) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

// The surrogate source runs for family p: on, trained, a coupled run in the FP32-flux form.
static bool sur_active(const ice_gpu_ctx* c, int p);

// The buffer stage srk reads as its stencil (U_{k-1}) when the step starts from buffer `phase`.
static int stencil_buffer(const ice_gpu_ctx*, int srk, int phase) {
  return srk == 1 ? phase : srk == 2 ? (phase + 1) % 3 : (phase + 2) % 3;
}

static FamDev make_famdev(ice_gpu_ctx* c, int p, int srk, int phase) {
  FamHost& H = c->fam[p];
  const ice_gpu_family& pf = c->P.fam[p];
  FamDev F;
  memset(&F, 0, sizeof F);
  F.closure = H.closure; F.riemann = H.riemann; F.nc = H.nc;
  F.limiter = c->P.limiter; F.sd = c->P.shock_detector; F.coupled = c->P.coupled;
  F.realize = c->P.precision == ICE_PREC_FP32FLUX && !c->P.no_realize;
  F.drag = c->P.drag; F.heat = c->P.heat; F.blow = c->P.blow;
  F.frozen_mask = 0;
  for (int q = 0; q < pf.nfrozen; ++q) F.frozen_mask |= 1u << (pf.frozen[q] - 1);
  F.mat.rho = pf.rho_al; F.mat.cp = pf.cs_al; F.mat.lv = pf.lv_al; F.mat.emiss = pf.emiss;
  F.mat.evap = pf.evap; F.mat.intf = pf.intf;
  for (int q = 0; q < ICE_GPU_NEP; ++q) F.mat.ep[q] = pf.ep[q];
  // buffer roles (see the rotation in step_graph)
  int a = phase, b = (phase + 1) % 3;
  int up = stencil_buffer(c, srk, phase);
  int out = srk == 1 ? b : srk == 2 ? (phase + 2) % 3 : b;
  F.U0 = H.S[a].p; F.Up = H.S[up].p; F.Ug = H.S[up].p; F.Uo = H.S[out].p;
  F.inj = H.inj.p;
  F.beta = c->P.shock_detector ? H.beta.p : nullptr;
  F.betaw = H.beta.p;
  F.dt = c->P.time_accurate ? nullptr : H.dt.p;
  F.dtg = &c->st.p->dtglobal;
  F.tau = H.tau.p;
  F.S = H.src.p;
  F.Sf = c->P.precision == ICE_PREC_FP32FLUX ? (float*)H.src.p : nullptr;
  F.bmap = H.bmap.p;
  F.Rb = H.Rb.p; F.Rbw = H.Rb.p;
  F.connF = H.connF.p;
  F.cdon = H.cdon.p; F.cw = H.cw.p;
  F.imports = H.have_imp ? H.imp.p : nullptr;
  F.xstep = (c->exchange && c->P.coupled) ? H.xstep.p : nullptr;
  F.xfirst = srk == 1;
  F.resid = H.resid.p;
  static const double RKC[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.50, 0.0}, {1.0, 0.25, 2.0/3.0}};
  F.rk = RKC[c->P.nrk - 1][srk - 1];
  F.write_tau = srk == c->P.nrk;
  F.src_ready = (sur_active(c, p) || (c->staged && c->P.coupled && pf.evap != 0)) ? 1 : 0;
  return F;
}

static Geo make_geo(ice_gpu_ctx* c) {
  Geo G;
  G.blk = c->blk.p; G.nb = c->nb;
  G.NG = c->NG; G.NI = c->NI; G.NR = c->NR;
  for (int d = 0; d < 3; ++d) { G.NF[d] = c->NF[d]; G.face[d] = c->face[d].p; }
  G.vol = c->vol.p; G.dl = c->dl.p; G.M = c->M.p; G.gas = c->gas.p;
  for (int d = 0; d < 3; ++d) G.ff[d] = c->facef[d].p;
  G.dlf = c->dlf.p;
  G.gasf = c->gasf.p;
  G.owned = c->owned.empty() ? nullptr : c->owned_dev.p;
  return G;
}

__global__ void k_face32(const double* f, long long NF, float4* out) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < NF; q += (long long)gridDim.x * blockDim.x)
    out[q] = make_float4((float)f[q], (float)f[NF + q], (float)f[2 * NF + q], (float)f[3 * NF + q]);
}

__global__ void k_dl32(const double* dl, long long n, float* out) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    out[q] = (float)dl[q];
}

// The FP32-flux form's geometry: the face normals and areas packed per face and the cell lengths in
// single precision, rounded as the kernels rounded each value on reading (allocated once, so that
// captured graphs keep their pointers; converted again after any ice_gpu_set_block).
static int build_geo32(ice_gpu_ctx* c) {
  if (c->P.precision != ICE_PREC_FP32FLUX || c->geo32_ok) return 0;
  bool fresh = false;
  for (int d = 0; d < 3; ++d) {
    if (!c->facef[d].p && c->NF[d] > 0) { CK(c->facef[d].alloc((size_t)c->NF[d])); fresh = true; }
    if (c->NF[d] > 0) {
      k_face32<<<grid_of(c->NF[d]), 256, 0, c->stream>>>(c->face[d].p, c->NF[d], c->facef[d].p);
      CK(cudaGetLastError());
    }
  }
  if (!c->dlf.p) { CK(c->dlf.alloc((size_t)3 * c->NR)); fresh = true; }
  k_dl32<<<grid_of(3 * c->NR), 256, 0, c->stream>>>(c->dl.p, 3 * c->NR, c->dlf.p);
  CK(cudaGetLastError());
  if (c->P.coupled && c->gas.p) {
    if (!c->gasf.p) { CK(c->gasf.alloc((size_t)9 * c->NI)); fresh = true; }
    k_dl32<<<grid_of(9 * c->NI), 256, 0, c->stream>>>(c->gas.p, 9 * c->NI, c->gasf.p);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->stream));
  if (fresh) free_graphs(c);          // graphs captured before the buffers existed hold null pointers
  c->geo32_ok = true;
  return 0;
}

// ---------------------------------------------------------------- kernel dispatch
#define GRID(n, t) ((unsigned)(((n) + (t) - 1) / (t)))

// ---------------------------------------------------------------- the block split's exchanges
// Pack and unpack of the exchange lists (0-based int4 entries: block, i, j, k; a connection face in x).
__global__ void k_pack_cells(Geo G, const double* __restrict__ U, int nc, const int4* __restrict__ e, int n,
                             double* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int4 x = e[q];
  const long long g = gidx(G.blk[x.x], x.y, x.z, x.w);
  for (int v = 0; v < nc; ++v) out[(long long)q * nc + v] = U[(long long)v * G.NG + g];
}
__global__ void k_unpack_cells(Geo G, double* __restrict__ U, int nc, const int4* __restrict__ e, int n,
                               const double* __restrict__ in) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int4 x = e[q];
  const long long g = gidx(G.blk[x.x], x.y, x.z, x.w);
  for (int v = 0; v < nc; ++v) U[(long long)v * G.NG + g] = in[(long long)q * nc + v];
}
__global__ void k_unpack_beta(Geo G, double* __restrict__ beta, const int4* __restrict__ e, int n,
                              const double* __restrict__ in) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int4 x = e[q];
  beta[iidx(G.blk[x.x], x.y, x.z, x.w)] = in[q];
}
__global__ void k_pack_flux(const double* __restrict__ F, int nc, const int4* __restrict__ e, int n,
                            double* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  for (int v = 0; v < nc; ++v) out[(long long)q * nc + v] = F[(long long)e[q].x * nc + v];
}
__global__ void k_unpack_flux(double* __restrict__ F, int nc, const int4* __restrict__ e, int n,
                              const double* __restrict__ in) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  for (int v = 0; v < nc; ++v) F[(long long)e[q].x * nc + v] = in[(long long)q * nc + v];
}

static int ensure_xbuf(ice_gpu_ctx* c, size_t n, cudaStream_t s) {
  if (c->xdev.n >= n && c->xhost_n >= n) return 0;
  CK(cudaStreamSynchronize(s));                    // the last exchange's copy and unpack read the buffers
  if (c->xdev.n < n) CK(c->xdev.alloc(n));
  if (c->xhost_n < n) {
    if (c->xhost) cudaFreeHost(c->xhost);
    c->xhost = nullptr; c->xhost_n = 0;
    CK(cudaMallocHost((void**)&c->xhost, n * sizeof(double)));
    c->xhost_n = n;
  }
  return 0;
}

// One exchange of a split step (Mod_GhostExchange.f90:737-800 for the cells), at its point of the
// family's stage: pack on the device, copy to the host, the hook, copy back, unpack. The stream is
// drained before the hook, so the hook sees this stage's data and no kernel waits on another rank.
// The first failure is kept (xerr) and reported by the step; later exchanges of the call are skipped.
static void halo_xchg(const LaunchArgs& a, int kind) {
  ice_gpu_ctx* c = (ice_gpu_ctx*)a.tick_ctx;
  if (c->xerr) return;
  const int p = a.fam, nc = c->fam[p].nc, w = kind == ICE_GPU_HALO_BETA ? 1 : nc;
  const int ns = (int)c->hs[kind][p].size(), nr = (int)c->hr[kind][p].size();
  const size_t ls = (size_t)ns * w, lr = (size_t)nr * w;
  if (ensure_xbuf(c, ls + lr + 1, a.s)) { c->xerr = ICE_GPU_ECUDA; return; }
  double* ds = c->xdev.p; double* dr = c->xdev.p + ls;
  const int4* es = c->hs_dev[kind][p].p; const int4* er = c->hr_dev[kind][p].p;
  if (ns > 0) {
    if (kind == ICE_GPU_HALO_CELLS) k_pack_cells<<<GRID(ns, 128), 128, 0, a.s>>>(a.G, a.F.Up, nc, es, ns, ds);
    else if (kind == ICE_GPU_HALO_FLUX) k_pack_flux<<<GRID(ns, 128), 128, 0, a.s>>>(a.F.connF, nc, es, ns, ds);
    else {
      // in the translation unit of the closure's connection kernel, compiled as it is, for its bits
      const int cl = c->fam[p].closure;
      const bool f32 = a.precision == ICE_PREC_FP32FLUX;
      if (cl == ICE_CLOSURE_MK) (f32 ? launch_pack_beta_mk_f32 : launch_pack_beta_mk_f64)(a, es, ns, ds);
      else if (cl == ICE_CLOSURE_IG) (f32 ? launch_pack_beta_ig_f32 : launch_pack_beta_ig_f64)(a, es, ns, ds);
      else (f32 ? launch_pack_beta_ag_f32 : launch_pack_beta_ag_f64)(a, es, ns, ds);
    }
    cudaMemcpyAsync(c->xhost, ds, ls * sizeof(double), cudaMemcpyDeviceToHost, a.s);
  }
  if (cudaStreamSynchronize(a.s) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    c->xerr = ICE_GPU_ECUDA; fail(c, ICE_GPU_ECUDA, "split exchange: a CUDA error before the hook");
    return;
  }
  if (!c->hook) { c->xerr = ICE_GPU_ENOTREADY; fail(c, ICE_GPU_ENOTREADY, "a split run needs its exchange hook"); return; }
  if (c->hook(c->hook_user, kind, p + 1, (int64_t)ls, c->xhost, (int64_t)lr, c->xhost + ls) != 0) {
    c->xerr = ICE_GPU_EEXCH; fail(c, ICE_GPU_EEXCH, "the exchange hook failed (kind %d, family %d)", kind, p + 1);
    return;
  }
  if (nr > 0) {
    cudaMemcpyAsync(dr, c->xhost + ls, lr * sizeof(double), cudaMemcpyHostToDevice, a.s);
    if (kind == ICE_GPU_HALO_CELLS) k_unpack_cells<<<GRID(nr, 128), 128, 0, a.s>>>(a.G, a.F.Ug, nc, er, nr, dr);
    else if (kind == ICE_GPU_HALO_FLUX) k_unpack_flux<<<GRID(nr, 128), 128, 0, a.s>>>(a.F.connF, nc, er, nr, dr);
    else k_unpack_beta<<<GRID(nr, 128), 128, 0, a.s>>>(a.G, a.F.betaw, er, nr, dr);
  }
}

// The reductions of a split run: the minimum (DT) or the sum (NORM) over the ranks of n doubles.
static int halo_reduce(ice_gpu_ctx* c, int kind, double* x, long long n) {
  if (c->owned.empty()) return 0;
  if (!c->hook) return fail(c, ICE_GPU_ENOTREADY, "a split run needs its exchange hook (ice_gpu_set_exchange_hook)");
  std::vector<double> in(x, x + n);
  if (c->hook(c->hook_user, kind, 0, n, in.data(), n, x) != 0)
    return fail(c, ICE_GPU_EEXCH, "the exchange hook failed (kind %d)", kind);
  return 0;
}

static void launch_family(ice_gpu_ctx* c, int p, int srk, int phase, cudaStream_t s,
                          void (*tick)(void*, int, cudaStream_t)) {
  FamHost& H = c->fam[p];
  LaunchArgs a;
  a.G = make_geo(c);
  a.F = make_famdev(c, p, srk, phase);
  a.recs = H.recs.p; a.nrec = H.nrec; a.grecs = H.grecs.p; a.ghost_split = H.ghost_split;
  a.own = H.own.p; a.nown = H.nown;
  a.bfirst = H.bfirst.p; a.blist = H.blist.p; a.nbc = H.nbc; a.bperm = H.bperm.p;
  a.tiles = c->tiles.p; a.ntile = c->ntile; a.TX = c->TX; a.TY = c->TY; a.KZ = c->KZ;
  a.tiles3 = H.tiles3.p; a.ntile3 = H.ntile3;
  a.maps = H.maps[stencil_buffer(c, srk, phase)].p;
  a.mlp_img = sur_active(c, p) ? H.mlp_img.p : nullptr;
  a.mlp_norm = &H.mlp_norm;
  a.ndir = c->P.ndir; a.sd = c->P.shock_detector; a.irs = c->P.irs; a.precision = c->P.precision;
  a.irs_beta = c->P.irs_beta;
  a.resid = H.resid.p; a.resid2 = H.resid2.p; a.resid3 = H.resid3.p;
  a.st = c->st.p;
  a.s = s;
  a.tick = tick; a.tick_ctx = c;
  a.xchg = c->owned.empty() ? nullptr : halo_xchg;
  a.fam = p;
  if (H.closure == ICE_CLOSURE_MK) launch_family_mk(a);
  else if (H.closure == ICE_CLOSURE_IG) launch_family_ig(a);
  else launch_family_ag(a);
}

// A family the coupler feeds or drains: bound_empty_dt and bound_removal_dt (Mod_Explicit.f90:57-60),
// after every family's compute_dt (k_dt_all).
static void launch_dt_bounds(ice_gpu_ctx* c, int p, int phase, cudaStream_t s) {
  if (!c->fam[p].have_imp) return;
  Geo G = make_geo(c);
  FamDev F = make_famdev(c, p, 1, phase);
  double* dto = c->P.time_accurate ? nullptr : c->fam[p].dt.p;
  unsigned g = GRID(c->NI, 256);
  EmptyScan* e = c->fam[p].escan.p;
  k_empty_init<<<1, 1, 0, s>>>(e);
  switch (c->fam[p].closure) {
    case ICE_CLOSURE_MK:
      k_empty_scan<MK><<<g, 256, 0, s>>>(G, F, dto, c->P.cfl, c->P.ndir, e);
      k_empty_apply<MK><<<g, 256, 0, s>>>(G, F, dto, c->P.cfl, c->P.ndir, e, c->st.p);
      break;
    case ICE_CLOSURE_IG:
      k_empty_scan<IG><<<g, 256, 0, s>>>(G, F, dto, c->P.cfl, c->P.ndir, e);
      k_empty_apply<IG><<<g, 256, 0, s>>>(G, F, dto, c->P.cfl, c->P.ndir, e, c->st.p);
      break;
    default:
      k_empty_scan<AG><<<g, 256, 0, s>>>(G, F, dto, c->P.cfl, c->P.ndir, e);
      k_empty_apply<AG><<<g, 256, 0, s>>>(G, F, dto, c->P.cfl, c->P.ndir, e, c->st.p);
      break;
  }
}

static int next_phase(const ice_gpu_ctx* c, int phase) {
  return c->P.nrk == 2 ? (phase + 2) % 3 : (phase + 1) % 3;
}

// One Explicit_Step on stream s starting from buffer `phase`: the step's dt over every family, then
// each family's RK stages (the families are independent of one another within a step).
static void enqueue_step_dt(ice_gpu_ctx* c, int phase, cudaStream_t s, void (*tick)(void*, int, cudaStream_t)) {
  k_begin<<<1, 1, 0, s>>>(c->st.p);
  {
    DtArgs a;
    memset(&a, 0, sizeof a);
    a.nf = c->P.nfam; a.ramp = c->P.cfl_ramp_iter; a.ndir = c->P.ndir;
    a.cfl = c->P.cfl; a.dt_max = c->P.dt_max; a.tau_factor = c->P.tau_factor;
    for (int p = 0; p < c->P.nfam; ++p) {
      FamDev F = make_famdev(c, p, 1, phase);
      a.f[p].Up = F.Up; a.f[p].tau = F.tau; a.f[p].coupled = F.coupled; a.f[p].closure = c->fam[p].closure;
      a.f[p].dt_out = c->P.time_accurate ? nullptr : c->fam[p].dt.p;
    }
    k_dt_all<<<GRID(c->NI, 256), 256, 0, s>>>(make_geo(c), a, c->st.p);
  }
  for (int p = 0; p < c->P.nfam; ++p) launch_dt_bounds(c, p, phase, s);
  if (!c->owned.empty() && !c->xerr) {
    // a split run: the step's dt is the smallest over every rank (Mod_Explicit.f90:67-73)
    unsigned long long bits = 0;
    if (cudaMemcpyAsync(&bits, &c->st.p->dtbits, sizeof bits, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      c->xerr = ICE_GPU_ECUDA; fail(c, ICE_GPU_ECUDA, "split exchange: reading the dt");
    } else {
      double d;
      memcpy(&d, &bits, sizeof d);
      if (halo_reduce(c, ICE_GPU_HALO_DT, &d, 1)) c->xerr = ICE_GPU_EEXCH;
      memcpy(&bits, &d, sizeof d);
      c->xbits = bits;
      cudaMemcpyAsync(&c->st.p->dtbits, &c->xbits, sizeof bits, cudaMemcpyHostToDevice, s);
      cudaStreamSynchronize(s);
    }
  }
  k_time<<<1, 1, 0, s>>>(c->st.p, c->P.time_accurate);
  if (tick) tick(c, KC_DT, s);
}

static void enqueue_step_family(ice_gpu_ctx* c, int p, int phase, cudaStream_t s,
                                void (*tick)(void*, int, cudaStream_t)) {
  for (int srk = 1; srk <= c->P.nrk; ++srk) launch_family(c, p, srk, phase, s, tick);
}

// The step: its dt over every family, then the families' RK stages one family after the other. (Run
// side by side on forked streams, the families' stage kernels shared the SMs with one another's
// differently sized CTAs and the 48-block step took 4.6 % longer, 139.9 ms against 133.7 ms.)
static void enqueue_step(ice_gpu_ctx* c, int phase, cudaStream_t s, void (*tick)(void*, int, cudaStream_t)) {
  enqueue_step_dt(c, phase, s, tick);
  for (int p = 0; p < c->P.nfam; ++p) enqueue_step_family(c, p, phase, s, tick);
}

static void prof_tick(void* vc, int cls, cudaStream_t s) {
  ice_gpu_ctx* c = (ice_gpu_ctx*)vc;
  cudaEventRecord(c->ev1, s);
  cudaEventSynchronize(c->ev1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->kms[cls] += ms;
  cudaEventRecord(c->ev0, s);
}

static long long launches_per_step(const ice_gpu_ctx* c) {
  long long n = 3;
  for (int p = 0; p < c->P.nfam; ++p) n += c->fam[p].have_imp ? 3 : 0;
  for (int p = 0; p < c->P.nfam; ++p) {
    const FamHost& H = c->fam[p];
    long long per = (H.nrec > 0 ? (H.ghost_split ? 2 : 1) : 0) + (c->P.shock_detector && !c->staged ? 1 : 0) + (H.nown > 0) + (H.nbc > 0) +
                    (c->P.coupled && (!c->staged || sur_active(c, p) || c->P.fam[p].evap != 0) ? 1 : 0);
    per += c->P.irs ? (2 + 2 * c->P.ndir) : 1;
    n += per * c->P.nrk;
  }
  return n;
}

// ---------------------------------------------------------------- set-up helpers
// The stage kernel's tiles: TX x TY columns of a block (x faces of TX - 1 cells and y faces of
// TY - 1 cells per tile, the last column and row being the next tile's), KZ planes per tile.
static void tile_shape(int ndir, int& TX, int& TY, int& KZ) {
  if (ndir == 1) { TX = 256; TY = 1; KZ = 1; }
  else if (ndir == 2) { TX = 32; TY = 8; KZ = 1; }
  else { TX = 16; TY = 16; KZ = 32; }
  if (const char* e = getenv("ICE_GPU_TILE")) {        // "TXxTYxKZ", for the tile tuner
    int a, b, k;
    if (sscanf(e, "%dx%dx%d", &a, &b, &k) == 3 && a * b == 256 && a >= 2 && k >= 1) { TX = a; TY = b; KZ = k; }
  }
}

// The staged kernel's limits for a closure (Shape<CL> of ice_stage3.cuh).
static void shape_limits(int closure, int& NT, int& MW, int& MH, int& MB, int& FX, int& FY, int& SXC, int& SYC) {
  if (closure == ICE_CLOSURE_AG) {
    NT = Shape<AG>::NT; MW = Shape<AG>::MAXW; MH = Shape<AG>::MAXH; MB = Shape<AG>::MAXBOX;
    FX = Shape<AG>::FX; FY = Shape<AG>::FY; SXC = Shape<AG>::SXC; SYC = Shape<AG>::SYC;
  } else {
    NT = Shape<MK>::NT; MW = Shape<MK>::MAXW; MH = Shape<MK>::MAXH; MB = Shape<MK>::MAXBOX;
    FX = Shape<MK>::FX; FY = Shape<MK>::FY; SXC = Shape<MK>::SXC; SYC = Shape<MK>::SYC;
  }
}

// The staged kernel's tile shape of a block of ni x nj columns: of the shapes W x H that fit the
// closure's limits (W H <= NT threads, the staged box, the face buffers), the one whose tiles, cut
// evenly from the block (ceil(ni / W) tiles of ceil(ni / nx) columns, likewise rows), take the fewest
// passes of the CTA per plane over the whole block: the face tasks (x and y faces below the owned
// cells, the faces above the last column and row) dealt out to the NT threads, then the z face and
// the update (zpass of the tuned schedule); at most wcap columns; among equals, the fewest tiles.
// Returns w, h (the even cut) and the box.
// The schedule of a closure: its row of the tuned table (ice_tune.h), or ICE_GPU_TUNE="kz,zpass,wcap".
static TuneRow tune_of(int closure) {
  TuneRow r = kTune[std::min(std::max(closure, 1), 3) - 1];
  if (const char* e = getenv("ICE_GPU_TUNE")) {
    int kz, zp, wc;
    if (sscanf(e, "%d,%d,%d", &kz, &zp, &wc) == 3 && kz >= 1 && kz <= ST_KZ && zp >= 0 && wc >= 1) r = TuneRow{kz, zp, wc};
  }
  return r;
}

static Tile tile_shape3(int ni, int nj, int closure) {
  int NT, MW, MH, MB, FX, FY, SXC, SYC;
  shape_limits(closure, NT, MW, MH, MB, FX, FY, SXC, SYC);
  (void)MW;
  const TuneRow tr = tune_of(closure);
  Tile best{};
  long long best_cost = -1, best_tiles = 0;
  const bool ax = ni >= 2, ay = nj >= 2;
  const int wmax = ax ? std::min(std::min(ni, NT), tr.wcap) : 1;
  for (int W = 1; W <= wmax; ++W) {
    if (st_box_x(W) > 256) break;                 // a TMA box is at most 256 elements along each axis
    const int hmax = std::min(std::min(nj, MH), NT / W);
    for (int H = 1; H <= hmax; ++H) {
      if (st_box_x(W) * (H + 4) > MB || H * (W + 1) > FX || (H + 1) * W > FY) break;
      if (H * (W + 2) > SXC || (H + 2) * W > SYC) break;   // the FP32-flux form's cell slopes
      const int nx = (ni + W - 1) / W, ny = (nj + H - 1) / H;
      const int w = (ni + nx - 1) / nx, h = (nj + ny - 1) / ny;
      const int tasks = (ax ? w * h + h : 0) + (ay ? w * h + w : 0);
      const long long tiles = (long long)nx * ny;
      const long long cost = tiles * ((tasks + NT - 1) / NT + tr.zpass);
      if (best_cost < 0 || cost < best_cost || (cost == best_cost && tiles < best_tiles)) {
        best_cost = cost; best_tiles = tiles;
        best = Tile{0, 0, 0, 0, 0, (short)w, (short)h, (short)st_box_x(w), (short)(h + 4)};
      }
    }
  }
  return best;
}

// The chunk height of the staged kernel's tiles for one family: of a few candidates up to the tuned
// kz planes, the one whose tiles, handed longest first to the least-loaded of the GPU's resident CTA
// slots (as the block scheduler hands them out), finish soonest; a tile costs its planes plus the
// three its prologue loads. Small grids get shorter chunks and more tiles, so that the last wave is
// not left half empty; large ones keep the largest (a change must gain more than 1 %).
static int choose_kz(const ice_gpu_ctx* c, const FamHost& H, int slots) {
  static const int cand[] = {ST_KZ, 28, 24, 20, 16, 12, 8, 4};
  const int kzmax = tune_of(H.closure).kz;
  int best = 0;
  double best_t = 0.0;
  for (int kz : cand) {
    if (kz > kzmax) continue;
    std::vector<int> cost;
    for (int b = 0; b < c->nb; ++b) {
      int ni = c->dims[3 * b], nj = c->dims[3 * b + 1], nk = c->dims[3 * b + 2];
      const Tile& sp = H.shape3[b];
      long long ncol = (long long)((ni + sp.w - 1) / sp.w) * ((nj + sp.h - 1) / sp.h);
      int nch = (nk + kz - 1) / kz, base = nk / nch, extra = nk % nch;
      for (int ch = 0; ch < nch; ++ch)
        for (long long q = 0; q < ncol; ++q) cost.push_back(base + (ch < extra ? 1 : 0) + 3);
    }
    std::sort(cost.begin(), cost.end(), std::greater<int>());
    std::priority_queue<long long, std::vector<long long>, std::greater<long long>> load;
    for (int q = 0; q < slots; ++q) load.push(0);
    long long span = 0;
    for (int x : cost) {
      long long l = load.top() + x;
      load.pop(); load.push(l);
      span = std::max(span, l);
    }
    if (best == 0 || (double)span < 0.99 * best_t) { best = kz; best_t = (double)span; }
  }
  return best;
}

static int build_tiles(ice_gpu_ctx* c) {
  tile_shape(c->P.ndir, c->TX, c->TY, c->KZ);
  std::vector<Tile> t;
  if (c->P.ndir == 1) {
    for (int b = 0; b < c->nb; ++b) {
      if (!c->owned.empty() && !c->owned[b]) continue;       // a split run steps its own blocks
      int ni = c->dims[3 * b], nj = c->dims[3 * b + 1], nk = c->dims[3 * b + 2];
      int sx = ni >= 2 ? c->TX - 1 : 1, sy = nj >= 2 ? std::max(c->TY - 1, 1) : 1;
      for (int k = 0; k < nk; k += c->KZ)
        for (int j = 0; j < nj; j += sy)
          for (int i = 0; i < ni; i += sx) t.push_back(Tile{b, i, j, k, std::min(c->KZ, nk - k)});
    }
    c->ntile = (int)t.size();
    CK(c->tiles.alloc(t.size()));
    CK(cudaMemcpy(c->tiles.p, t.data(), t.size() * sizeof(Tile), cudaMemcpyHostToDevice));
  } else {
    // the staged kernel: column tiles of each block's shape (tile_shape3), each block's height cut
    // into equal chunks of at most kz planes (choose_kz); the longest first
    c->staged = true;
    int nsm = 148;
    {
      int dev = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    }
    const int slots = nsm * (c->P.precision == ICE_PREC_FP32FLUX ? 2 : 1);   // the kernel's launch bounds
    for (int p = 0; p < c->P.nfam; ++p) {
      FamHost& H = c->fam[p];
      t.clear();
      H.shape3.resize(c->nb);
      for (int b = 0; b < c->nb; ++b) H.shape3[b] = tile_shape3(c->dims[3 * b], c->dims[3 * b + 1], H.closure);
      const int kz = choose_kz(c, H, slots);
      for (int b = 0; b < c->nb; ++b) {
        if (!c->owned.empty() && !c->owned[b]) continue;     // a split run steps its own blocks
        int ni = c->dims[3 * b], nj = c->dims[3 * b + 1], nk = c->dims[3 * b + 2];
        const Tile& sp = H.shape3[b];
        int nch = (nk + kz - 1) / kz, base = nk / nch, extra = nk % nch;
        for (int ch = 0, k = 0; ch < nch; ++ch) {
          int hz = base + (ch < extra ? 1 : 0);
          for (int j = 0; j < nj; j += sp.h)
            for (int i = 0; i < ni; i += sp.w)
              t.push_back(Tile{b, i, j, k, hz, (short)std::min((int)sp.w, ni - i), (short)std::min((int)sp.h, nj - j),
                               sp.bx, sp.by});
          k += hz;
        }
      }
      std::stable_sort(t.begin(), t.end(), [](const Tile& x, const Tile& y) { return x.nkz > y.nkz; });
      H.ntile3 = (int)t.size();
      CK(H.tiles3.alloc(t.size()));
      CK(cudaMemcpy(H.tiles3.p, t.data(), t.size() * sizeof(Tile), cudaMemcpyHostToDevice));
    }
  }
  // norm chunks: 2048 cells of one block each
  std::vector<NormChunk> ch;
  c->chunk_block.clear();
  for (int b = 0; b < c->nb; ++b) {
    long long n = (long long)c->dims[3 * b] * c->dims[3 * b + 1] * c->dims[3 * b + 2];
    for (long long q = 0; q < n; q += 2048) {
      ch.push_back(NormChunk{b, c->hblk[b].ioff + q, c->hblk[b].ioff + std::min(n, q + 2048)});
      c->chunk_block.push_back(b);
    }
  }
  c->nchunk = (int)ch.size();
  CK(c->chunks.alloc(ch.size()));
  CK(cudaMemcpy(c->chunks.p, ch.data(), ch.size() * sizeof(NormChunk), cudaMemcpyHostToDevice));
  CK(c->npart.alloc((size_t)c->nchunk * 5));
  return 0;
}

// The staged stage kernel's TMA maps: per family, state buffer and block, a 4-D view (x, y, z,
// variable) of the block's ghost-cell pool, strides row px, plane pxy and variable NG (all multiples
// of 16 bytes by the padding of the layout), box bx x by x 1 x nc of the block's tile shape.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)f;
  }
  return fn;
}

static int build_maps(ice_gpu_ctx* c) {
  if (!c->staged) return 0;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return fail(c, ICE_GPU_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
  std::vector<CUtensorMap> h(c->nb);
  for (int p = 0; p < c->P.nfam; ++p) {
    FamHost& H = c->fam[p];
    for (int buf = 0; buf < 3; ++buf) {
      for (int b = 0; b < c->nb; ++b) {
        const DBlock& B = c->hblk[b];
        cuuint64_t dims[4] = {(cuuint64_t)B.px, (cuuint64_t)(B.nj + 4), (cuuint64_t)(B.nk + 4), (cuuint64_t)H.nc};
        cuuint64_t strides[3] = {(cuuint64_t)B.px * 8, (cuuint64_t)B.pxy * 8, (cuuint64_t)c->NG * 8};
        cuuint32_t box[4] = {(cuuint32_t)H.shape3[b].bx, (cuuint32_t)H.shape3[b].by, 1, (cuuint32_t)H.nc};
        cuuint32_t es[4] = {1, 1, 1, 1};
        CUresult r = enc(&h[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)(H.S[buf].p + B.goff), dims, strides, box,
                         es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(c, ICE_GPU_ECUDA, "cuTensorMapEncodeTiled: error %d (family %d, block %d)",
                                           (int)r, p + 1, b + 1);
      }
      CK(H.maps[buf].alloc(c->nb));
      CK(cudaMemcpy(H.maps[buf].p, h.data(), c->nb * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    }
  }
  return 0;
}

extern "C" {

int ice_gpu_create(const ice_gpu_params* P, int32_t nblocks, const int32_t* dims, ice_gpu_ctx** out) {
  ice_gpu_ctx* c = nullptr;
  if (!P || !dims || !out || nblocks < 1) return fail(nullptr, ICE_GPU_EINVAL, "create: null argument or no block");
  if (P->nfam < 1 || P->nfam > kMaxF) return fail(nullptr, ICE_GPU_EINVAL, "create: nfam %d out of 1..%d", P->nfam, kMaxF);
  if (P->nrk < 1 || P->nrk > 3) return fail(nullptr, ICE_GPU_EINVAL, "create: nrk %d", P->nrk);
  if (P->ndir < 1 || P->ndir > 3) return fail(nullptr, ICE_GPU_EINVAL, "create: ndir %d", P->ndir);
  for (int p = 0; p < P->nfam; ++p) {
    const ice_gpu_family& f = P->fam[p];
    if (f.closure < 1 || f.closure > 3) return fail(nullptr, ICE_GPU_EINVAL, "family %d: closure %d", p + 1, f.closure);
    if (f.riemann == ICE_RIEMANN_SAUREL && f.closure != ICE_CLOSURE_MK)
      return fail(nullptr, ICE_GPU_EINVAL, "family %d: riemann-solver = Saurel is specific to the MK closure; use Rusanov or HLLE", p + 1);
    if (f.liq != 0 || f.boil != 0)
      return fail(nullptr, ICE_GPU_EINVAL, "family %d: liquid-conduction P2T and boiling ZGR are not supported", p + 1);
  }
  if (P->irs && P->time_accurate)
    return fail(nullptr, ICE_GPU_EINVAL, "irs = true needs time-accurate = false (Assign_Setup.f90:79-83)");
  std::unique_ptr<ice_gpu_ctx> u(new ice_gpu_ctx);
  c = u.get();
  c->P = *P;
  c->nb = nblocks;
  c->dims.assign(dims, dims + 3 * nblocks);
  c->have_block.assign(nblocks, false);
  c->gas_set.assign(nblocks, false);
  long long G = 0, I = 0, R = 0, F0 = 0, F1 = 0, F2 = 0;
  for (int b = 0; b < nblocks; ++b) {
    int ni = dims[3 * b], nj = dims[3 * b + 1], nk = dims[3 * b + 2];
    if (ni < 1 || nj < 1 || nk < 1) return fail(nullptr, ICE_GPU_EINVAL, "block %d: dims %d %d %d", b + 1, ni, nj, nk);
    if ((long long)ni * nj * nk >= (1LL << 31))
      return fail(nullptr, ICE_GPU_EINVAL, "block %d: %lld cells, at most 2^31 - 1 per block", b + 1, (long long)ni * nj * nk);
    DBlock B;
    B.ni = ni; B.nj = nj; B.nk = nk;
    B.px = (ni + 4 + 1) & ~1;
    B.pxy = (long long)B.px * (nj + 4);
    B.goff = G; B.ioff = I; B.roff = R; B.foff[0] = F0; B.foff[1] = F1; B.foff[2] = F2;
    G += B.pxy * (nk + 4);
    c->ng_max = std::max(c->ng_max, (long long)(ni + 4) * (nj + 4) * (nk + 4));
    I += (long long)ni * nj * nk;
    R += (long long)(ni + 2) * (nj + 2) * (nk + 2);
    F0 += (long long)(ni + 1) * nj * nk; F1 += (long long)ni * (nj + 1) * nk; F2 += (long long)ni * nj * (nk + 1);
    c->hblk.push_back(B);
  }
  c->NG = G; c->NI = I; c->NR = R; c->NF[0] = F0; c->NF[1] = F1; c->NF[2] = F2;
  cudaError_t e;
#define CKC(call) do { e = (call); if (e != cudaSuccess) return fail(nullptr, ICE_GPU_ECUDA, "%s: %s", #call, cudaGetErrorString(e)); } while (0)
  CKC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CKC(c->blk.alloc(nblocks));
  CKC(cudaMemcpy(c->blk.p, c->hblk.data(), nblocks * sizeof(DBlock), cudaMemcpyHostToDevice));
  for (int d = 0; d < 3; ++d) CKC(c->face[d].alloc((size_t)4 * c->NF[d]));
  CKC(c->vol.alloc(I));
  CKC(c->dl.alloc((size_t)3 * R));
  CKC(c->M.alloc((size_t)9 * I));
  if (P->coupled) CKC(c->gas.alloc((size_t)9 * I));
  for (int p = 0; p < P->nfam; ++p) {
    FamHost& H = c->fam[p];
    H.closure = P->fam[p].closure; H.riemann = P->fam[p].riemann; H.nc = nbase_of(H.closure);
    for (int s = 0; s < 3; ++s) {
      CKC(H.S[s].alloc((size_t)H.nc * G));
      // poison: a ghost cell no record fills stays NaN, as Allocate_Block leaves it
      CKC(cudaMemset(H.S[s].p, 0xFF, sizeof(double) * H.nc * G));
    }
    CKC(H.inj.alloc(G)); CKC(cudaMemset(H.inj.p, 0, G));
    CKC(H.dt.alloc(I));
    CKC(H.tau.alloc(I));
    std::vector<double> inf(I, INFINITY);
    CKC(cudaMemcpy(H.tau.p, inf.data(), I * sizeof(double), cudaMemcpyHostToDevice));
    CKC(H.beta.alloc(I));
    std::vector<double> one(I, 1.0);
    CKC(cudaMemcpy(H.beta.p, one.data(), I * sizeof(double), cudaMemcpyHostToDevice));
    CKC(H.bmap.alloc(I)); CKC(cudaMemset(H.bmap.p, 0xFF, I * sizeof(int)));
    if (P->coupled) CKC(H.src.alloc((size_t)H.nc * I));
    if (P->irs) { CKC(H.resid.alloc((size_t)H.nc * I)); CKC(H.resid2.alloc((size_t)H.nc * I)); CKC(H.resid3.alloc((size_t)H.nc * I)); }
  }
  CKC(c->st.alloc(1));
  Status s0; memset(&s0, 0, sizeof s0);
  CKC(cudaMemcpy(c->st.p, &s0, sizeof s0, cudaMemcpyHostToDevice));
  CKC(cudaEventCreate(&c->ev0)); CKC(cudaEventCreate(&c->ev1));
#undef CKC
  if (build_tiles(c)) { g_create_err = c->err; return ICE_GPU_ECUDA; }
  if (build_maps(c)) { g_create_err = c->err; return ICE_GPU_ECUDA; }
  *out = u.release();
  return 0;
}

int ice_gpu_destroy(ice_gpu_ctx* c) {
  if (!c) return 0;
  cudaStreamSynchronize(c->stream);
  free_graphs(c);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->s_up) { cudaStreamSynchronize(c->s_up); cudaStreamDestroy(c->s_up); }
  if (c->s_down) { cudaStreamSynchronize(c->s_down); cudaStreamDestroy(c->s_down); }
  if (c->ev_up) cudaEventDestroy(c->ev_up);
  if (c->xhost) cudaFreeHost(c->xhost);
  for (auto& e : c->ev_fam) if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int ice_gpu_last_error(const ice_gpu_ctx* c, char* buf, int32_t n) {
  if (!buf || n <= 0) return ICE_GPU_EINVAL;
  const std::string& s = c ? c->err : g_create_err;
  strncpy(buf, s.c_str(), n - 1); buf[n - 1] = 0;
  return 0;
}

int ice_gpu_set_block(ice_gpu_ctx* c, int32_t b1, const double* f1, const double* f2, const double* f3,
                      const double* vol, const double* dl, const double* M) {
  if (!c) return ICE_GPU_EINVAL;
  if (b1 < 1 || b1 > c->nb) return fail(c, ICE_GPU_EINVAL, "set_block: block %d out of range", b1);
  if (!f1 || !f2 || !f3 || !vol || !dl || !M) return fail(c, ICE_GPU_EINVAL, "set_block: null array");
  const DBlock& B = c->hblk[b1 - 1];
  int ni = B.ni, nj = B.nj, nk = B.nk;
  const double* fs[3] = {f1, f2, f3};
  long long nf[3] = {(long long)(ni + 1) * nj * nk, (long long)ni * (nj + 1) * nk, (long long)ni * nj * (nk + 1)};
  std::vector<double> tmp;
  for (int d = 0; d < 3; ++d) {
    tmp.resize(nf[d]);
    for (int comp = 0; comp < 4; ++comp) {
      for (long long q = 0; q < nf[d]; ++q) tmp[q] = fs[d][4 * q + comp];
      CK(cudaMemcpy(c->face[d].p + (long long)comp * c->NF[d] + B.foff[d], tmp.data(), nf[d] * sizeof(double), cudaMemcpyHostToDevice));
    }
  }
  long long ncell = (long long)ni * nj * nk, nring = (long long)(ni + 2) * (nj + 2) * (nk + 2);
  CK(cudaMemcpy(c->vol.p + B.ioff, vol, ncell * sizeof(double), cudaMemcpyHostToDevice));
  tmp.resize(nring);
  for (int comp = 0; comp < 3; ++comp) {
    for (long long q = 0; q < nring; ++q) tmp[q] = dl[3 * q + comp];
    CK(cudaMemcpy(c->dl.p + (long long)comp * c->NR + B.roff, tmp.data(), nring * sizeof(double), cudaMemcpyHostToDevice));
  }
  // M on the interior cells only (compute_dt reads nothing else)
  tmp.resize(ncell);
  for (int comp = 0; comp < 9; ++comp) {
    for (int k = 0; k < nk; ++k) for (int j = 0; j < nj; ++j) for (int i = 0; i < ni; ++i) {
      long long r = ((long long)(k + 1) * (nj + 2) + (j + 1)) * (ni + 2) + (i + 1);
      tmp[((long long)k * nj + j) * ni + i] = M[9 * r + comp];
    }
    CK(cudaMemcpy(c->M.p + (long long)comp * c->NI + B.ioff, tmp.data(), ncell * sizeof(double), cudaMemcpyHostToDevice));
  }
  c->have_block[b1 - 1] = true;
  c->geo32_ok = false;
  return 0;
}

int ice_gpu_set_gas(ice_gpu_ctx* c, int32_t b1, const double* prim5, const double* R, const double* gam,
                    const double* k, const double* mu) {
  if (!c) return ICE_GPU_EINVAL;
  if (!c->P.coupled) return fail(c, ICE_GPU_EINVAL, "set_gas: the run is not coupled");
  if (b1 < 1 || b1 > c->nb) return fail(c, ICE_GPU_EINVAL, "set_gas: block %d out of range", b1);
  const DBlock& B = c->hblk[b1 - 1];
  long long n = (long long)B.ni * B.nj * B.nk;
  std::vector<double> tmp(n);
  for (int comp = 0; comp < 5; ++comp) {
    for (long long q = 0; q < n; ++q) tmp[q] = prim5[5 * q + comp];
    CK(cudaMemcpy(c->gas.p + (long long)comp * c->NI + B.ioff, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  }
  const double* rest[4] = {R, gam, k, mu};
  for (int comp = 0; comp < 4; ++comp)
    CK(cudaMemcpy(c->gas.p + (long long)(5 + comp) * c->NI + B.ioff, rest[comp], n * sizeof(double), cudaMemcpyHostToDevice));
  c->gas_set[b1 - 1] = true;
  c->geo32_ok = false;                 // the FP32-flux form's copy of the gas is made again
  c->have_gas = std::all_of(c->gas_set.begin(), c->gas_set.end(), [](bool x) { return x; });
  return 0;
}

int ice_gpu_upload_state(ice_gpu_ctx* c, int32_t b1, int32_t p1, const double* prim, const uint8_t* inj) {
  if (!c) return ICE_GPU_EINVAL;
  if (b1 < 1 || b1 > c->nb || p1 < 1 || p1 > c->P.nfam) return fail(c, ICE_GPU_EINVAL, "upload_state: bad block/family");
  if (!prim) return fail(c, ICE_GPU_EINVAL, "upload_state: null prim");
  const DBlock& B = c->hblk[b1 - 1];
  FamHost& H = c->fam[p1 - 1];
  long long ng = (long long)(B.ni + 4) * (B.nj + 4) * (B.nk + 4);
  if (!c->xfer.p) CK(c->xfer.alloc((size_t)c->ng_max * kMaxNC));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpyAsync(c->xfer.p, prim, (size_t)ng * H.nc * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  k_aos2soa<<<grid_of(ng), 256, 0, c->stream>>>(c->xfer.p, H.S[c->phase].p + B.goff, c->NG, ng, H.nc,
                                                 B.ni + 4, B.nj + 4, B.px);
  CK(cudaGetLastError());
  if (inj) {
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpyAsync(c->xfer.p, inj, ng, cudaMemcpyHostToDevice, c->stream));
    k_inj2pool<<<grid_of(ng), 256, 0, c->stream>>>((const unsigned char*)c->xfer.p, H.inj.p + B.goff, ng,
                                                   B.ni + 4, B.nj + 4, B.px);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->stream));
  c->prev_phase = -1;
  return 0;
}

int ice_gpu_download_state(ice_gpu_ctx* c, int32_t b1, int32_t p1, double* prim) {
  if (!c) return ICE_GPU_EINVAL;
  if (b1 < 1 || b1 > c->nb || p1 < 1 || p1 > c->P.nfam) return fail(c, ICE_GPU_EINVAL, "download_state: bad block/family");
  const DBlock& B = c->hblk[b1 - 1];
  FamHost& H = c->fam[p1 - 1];
  long long ng = (long long)(B.ni + 4) * (B.nj + 4) * (B.nk + 4);
  if (!prim) return fail(c, ICE_GPU_EINVAL, "download_state: null prim");
  if (!c->xfer.p) CK(c->xfer.alloc((size_t)c->ng_max * kMaxNC));
  k_soa2aos<<<grid_of(ng), 256, 0, c->stream>>>(H.S[c->phase].p + B.goff, c->xfer.p, c->NG, ng, H.nc,
                                                 B.ni + 4, B.nj + 4, B.px);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(prim, c->xfer.p, (size_t)ng * H.nc * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int ice_gpu_set_time(ice_gpu_ctx* c, double time, int32_t iter, int32_t iter_from_call) {
  if (!c) return ICE_GPU_EINVAL;
  Status s;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(&s, c->st.p, sizeof s, cudaMemcpyDeviceToHost));
  s.time = time; s.iter = iter; s.iter_from_call = iter_from_call;
  CK(cudaMemcpy(c->st.p, &s, sizeof s, cudaMemcpyHostToDevice));
  return 0;
}

int ice_gpu_set_res_reference(ice_gpu_ctx* c, double ref) {
  if (!c) return ICE_GPU_EINVAL;
  c->res_reference = ref;
  return 0;
}

int ice_gpu_get_res_reference(ice_gpu_ctx* c, double* ref) {
  if (!c) return ICE_GPU_EINVAL;
  if (!ref) return fail(c, ICE_GPU_EINVAL, "get_res_reference: null pointer");
  *ref = c->res_reference;
  return 0;
}

int ice_gpu_update_params(ice_gpu_ctx* c, const ice_gpu_params* P) {
  if (!c || !P) return ICE_GPU_EINVAL;
  if (P->nfam != c->P.nfam || P->ndir != c->P.ndir) return fail(c, ICE_GPU_EINVAL, "update_params: nfam and ndir may not change");
  for (int p = 0; p < P->nfam; ++p) {
    if (P->fam[p].closure != c->P.fam[p].closure) return fail(c, ICE_GPU_EINVAL, "update_params: closures may not change");
    if (P->fam[p].riemann == ICE_RIEMANN_SAUREL && P->fam[p].closure != ICE_CLOSURE_MK)
      return fail(c, ICE_GPU_EINVAL, "update_params: Saurel is specific to MK");
  }
  if (P->irs && P->time_accurate) return fail(c, ICE_GPU_EINVAL, "update_params: irs needs a steady run");
  if (P->irs && !c->P.irs) {
    for (int p = 0; p < c->P.nfam; ++p) {
      FamHost& H = c->fam[p];
      CK(H.resid.alloc((size_t)H.nc * c->NI)); CK(H.resid2.alloc((size_t)H.nc * c->NI)); CK(H.resid3.alloc((size_t)H.nc * c->NI));
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  c->P = *P;
  for (int p = 0; p < c->P.nfam; ++p) c->fam[p].riemann = P->fam[p].riemann;
  free_graphs(c);
  return 0;
}

// The family's device records (table order, which the boundary and connection kernels index), and a
// copy for the ghost kernel ordered by block, face and cell with the first index fastest, so that the
// threads of a warp fill neighbouring ghost cells of one face (a record's ghosts are its own, so the
// order of the fills does not change a value). ghost_split: some record's block (or, for a connection,
// its source block) is one cell deep along the record's face direction, so that record's second ghost
// layer reads the first layer of the opposite face's record; the ghost kernel then runs as two launches.
static int upload_recs(ice_gpu_ctx* c, FamHost& H) {
  const std::vector<DRec>& dr = H.h_recs;
  CK(H.recs.alloc(dr.size()));
  CK(H.grecs.alloc(dr.size()));
  H.ghost_split = false;
  for (const DRec& r : dr) {
    if (r.type == 0 || r.type == 102) continue;
    if (c->dims[3 * r.b + (r.f - 1) / 2] == 1) H.ghost_split = true;
    if ((r.type == 101 || r.type == 201) && c->dims[3 * r.bs + (r.fs - 1) / 2] == 1) H.ghost_split = true;
  }
  if (dr.empty()) return 0;
  CK(cudaMemcpy(H.recs.p, dr.data(), dr.size() * sizeof(DRec), cudaMemcpyHostToDevice));
  std::vector<int> ord(dr.size());
  for (size_t q = 0; q < ord.size(); ++q) ord[q] = (int)q;
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
    const DRec& a = dr[x]; const DRec& b = dr[y];
    if (a.b != b.b) return a.b < b.b;
    if (a.f != b.f) return a.f < b.f;
    if (a.k != b.k) return a.k < b.k;
    if (a.j != b.j) return a.j < b.j;
    return a.i < b.i;
  });
  std::vector<DRec> g(dr.size());
  for (size_t q = 0; q < ord.size(); ++q) g[q] = dr[ord[q]];
  CK(cudaMemcpy(H.grecs.p, g.data(), g.size() * sizeof(DRec), cudaMemcpyHostToDevice));
  return 0;
}

// build_local_bc_index + collect_boundary_cells + collect_owner_records
// (parallel/Mod_GhostExchange.f90:103-360) for a device that owns every block.
int ice_gpu_set_records(ice_gpu_ctx* c, int32_t nrec, const int32_t* ri, const double* rr) {
  if (!c) return ICE_GPU_EINVAL;
  if (nrec < 0 || (nrec > 0 && (!ri || !rr))) return fail(c, ICE_GPU_EINVAL, "set_records: bad arguments");
  c->recs.resize(nrec);
  for (int n = 0; n < nrec; ++n) {
    const int32_t* q = ri + (long long)n * ICE_GPU_REC_INTS;
    const double* x = rr + (long long)n * ICE_GPU_REC_REALS;
    HRec& r = c->recs[n];
    r.b = q[0]; r.i = q[1]; r.j = q[2]; r.k = q[3]; r.f = q[4]; r.type = q[5]; r.p = q[6];
    r.bs = q[7]; r.is = q[8]; r.js = q[9]; r.ks = q[10]; r.fs = q[11]; r.partner = q[12]; r.owner = q[13]; r.cf = q[14];
    r.massflux = x[0]; r.velocity = x[1]; r.alpha = x[2]; r.beta = x[3]; r.temperature = x[4]; r.radius = x[5];
    r.gfixed = x[6]; r.normal_dir = x[7];
    if (r.b < 1 || r.b > c->nb || r.p < 1 || r.p > c->P.nfam || r.f < 1 || r.f > 6)
      return fail(c, ICE_GPU_EINVAL, "record %d: bad block, family or face", n + 1);
    const int* d = &c->dims[3 * (r.b - 1)];
    if (r.i < 1 || r.i > d[0] || r.j < 1 || r.j > d[1] || r.k < 1 || r.k > d[2])
      return fail(c, ICE_GPU_EINVAL, "record %d: cell %d %d %d outside block %d", n + 1, r.i, r.j, r.k, r.b);
    {
      const int ijk[3] = {r.i, r.j, r.k};
      int dd = (r.f - 1) / 2;
      if (ijk[dd] != (r.f % 2 == 1 ? 1 : d[dd]))
        return fail(c, ICE_GPU_EINVAL, "record %d: cell %d %d %d is off its face %d", n + 1, r.i, r.j, r.k, r.f);
    }
    int t = r.type;
    bool known = t == 0 || t == 101 || t == 201 || t == 102 || t == 200 || t == 300 || t == 301 || t == 400 ||
                 (t >= 401 && t <= 403);
    if (!known) return fail(c, ICE_GPU_EINVAL, "record %d: boundary code %d is not supported on the device", n + 1, t);
    if (t == 101 || t == 201) {
      if (r.bs < 1 || r.bs > c->nb) return fail(c, ICE_GPU_EINVAL, "record %d: source block %d", n + 1, r.bs);
      if (r.fs < 1 || r.fs > 6) return fail(c, ICE_GPU_EINVAL, "record %d: source face %d", n + 1, r.fs);
      const int* ds = &c->dims[3 * (r.bs - 1)];
      int g0 = (r.fs == 1) - (r.fs == 2), g1 = (r.fs == 3) - (r.fs == 4), g2 = (r.fs == 5) - (r.fs == 6);
      int s1[3] = {r.is, r.js, r.ks}, s2[3] = {r.is + g0, r.js + g1, r.ks + g2};
      for (int a = 0; a < 3; ++a)
        if (s1[a] < 1 || s1[a] > ds[a] || s2[a] < 1 || s2[a] > ds[a])
          return fail(c, ICE_GPU_EINVAL, "record %d: the two source cells of its ghosts are not inside block %d", n + 1, r.bs);
      if (r.partner < 1 || r.partner > nrec || r.cf < 1) return fail(c, ICE_GPU_EINVAL, "record %d: connection not paired", n + 1);
    }
    // read_bc (io/IO_BC.f90:264-271): a 401 or 403 inlet that injects (non-zero mass flux) reads the gas
    // speed; a run without a gas phase refuses it while the table is read. A zero-flux inlet mirrors
    // (ghost_rule, Lib_Ghost.f90:409) and reads no gas.
    if ((t == 401 || t == 403) && r.massflux != 0.0 && !c->P.coupled)
      return fail(c, ICE_GPU_EINVAL, "record %d: inlet %d takes its speed from the gas, and the run has no gas", n + 1, t);
  }
  for (int p = 0; p < c->P.nfam; ++p) {
    FamHost& H = c->fam[p];
    // the family's records in table order
    std::vector<int> grp;
    for (int n = 0; n < nrec; ++n) if (c->recs[n].p == p + 1) grp.push_back(n);
    std::vector<int> pos(nrec, -1);
    for (size_t q = 0; q < grp.size(); ++q) pos[grp[q]] = (int)q;
    std::vector<DRec> dr(grp.size());
    int ncf = 0;
    for (size_t q = 0; q < grp.size(); ++q) {
      const HRec& r = c->recs[grp[q]];
      DRec& d = dr[q];
      d.b = r.b - 1; d.i = r.i - 1; d.j = r.j - 1; d.k = r.k - 1; d.f = r.f; d.type = r.type;
      d.bs = r.bs - 1; d.is = r.is - 1; d.js = r.js - 1; d.ks = r.ks - 1; d.fs = r.fs;
      d.owner = r.owner; d.cf = r.cf - 1;
      if (r.type == 101 || r.type == 201) {
        const HRec& q2 = c->recs[r.partner - 1];
        d.pb = q2.b - 1; d.pi = q2.i - 1; d.pj = q2.j - 1; d.pk = q2.k - 1;
        ncf = std::max(ncf, r.cf);
      } else { d.pb = d.pi = d.pj = d.pk = 0; }
      d.normal_dir = r.normal_dir != 0.0;
      d.massflux = r.massflux; d.velocity = r.velocity; d.alpha = r.alpha; d.beta = r.beta;
      d.temperature = r.temperature; d.radius = r.radius; d.gfixed = r.gfixed;
      d.ca = cos(r.alpha); d.sa = sin(r.alpha); d.cb = cos(r.beta); d.sb = sin(r.beta);
      d.vol_p = 4.0/3.0*kPi*pow(r.radius, 3.0);
      d.cd0 = d.cn1 = d.cn2 = 0;
    }
    H.nrec = (int)grp.size();
    H.h_grp = grp;
    H.h_recs = dr;
    if (int rc = upload_recs(c, H)) return rc;
    // boundary cells: block by block in cell order, the records of a cell by face (stable)
    H.h_first.clear(); H.h_list.clear();
    std::vector<int> bmap(c->NI, -1);
    for (int b = 0; b < c->nb; ++b) {
      const DBlock& B = c->hblk[b];
      long long ncell = (long long)B.ni * B.nj * B.nk;
      std::vector<int> head(ncell, -1), tail(ncell, -1), next(nrec, -1);
      for (int n : grp) {
        const HRec& r = c->recs[n];
        if (r.b != b + 1 || r.type == 0) continue;
        long long q = ((long long)(r.k - 1) * B.nj + (r.j - 1)) * B.ni + (r.i - 1);
        if (head[q] < 0) head[q] = n; else next[tail[q]] = n;
        tail[q] = n;
      }
      for (long long q = 0; q < ncell; ++q) {
        if (head[q] < 0) continue;
        bmap[B.ioff + q] = (int)H.h_first.size();
        int s0 = (int)H.h_list.size();
        H.h_first.push_back(s0);
        for (int n = head[q]; n >= 0; n = next[n]) H.h_list.push_back(n);
        for (size_t m = s0 + 1; m < H.h_list.size(); ++m) {
          int n = H.h_list[m]; long long l = (long long)m - 1;
          while (l >= s0 && c->recs[H.h_list[l]].f > c->recs[n].f) { H.h_list[l + 1] = H.h_list[l]; --l; }
          H.h_list[l + 1] = n;
        }
      }
    }
    H.nbc = (int)H.h_first.size();
    H.h_first.push_back((int)H.h_list.size());
    std::vector<int> dlist(H.h_list.size());
    for (size_t q = 0; q < H.h_list.size(); ++q) dlist[q] = pos[H.h_list[q]];
    CK(H.bfirst.alloc(H.h_first.size()));
    CK(cudaMemcpy(H.bfirst.p, H.h_first.data(), H.h_first.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(H.blist.alloc(std::max<size_t>(dlist.size(), 1)));
    if (!dlist.empty()) CK(cudaMemcpy(H.blist.p, dlist.data(), dlist.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(H.bmap.p, bmap.data(), c->NI * sizeof(int), cudaMemcpyHostToDevice));
    CK(H.Rb.alloc((size_t)std::max(H.nbc, 1) * H.nc));
    // the boundary kernel's thread order: the cells grouped by block, by the face of their first record
    // and by whether it is a connection, in cell order within a group, so that the threads of a warp take
    // the same branches (each cell's sum and its slot of Rb are the same in any order)
    {
      std::vector<int> perm(H.nbc);
      for (int q = 0; q < H.nbc; ++q) perm[q] = q;
      auto key = [&](int q) {
        const HRec& r = c->recs[H.h_list[H.h_first[q]]];
        const int conn = (r.type == 101 || r.type == 201) ? 1 : 0;
        return ((long long)r.b * 8 + r.f) * 2 + conn;
      };
      std::stable_sort(perm.begin(), perm.end(), [&](int x, int y) { return key(x) < key(y); });
      CK(H.bperm.alloc(std::max<size_t>(perm.size(), 1)));
      if (!perm.empty()) CK(cudaMemcpy(H.bperm.p, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    // connection owners, table order
    H.h_own.clear();
    for (int n : grp) {
      const HRec& r = c->recs[n];
      if ((r.type == 101 || r.type == 201) && r.owner) H.h_own.push_back(n);
    }
    H.nown = (int)H.h_own.size();
    H.ncf = ncf;
    std::vector<int> down(H.h_own.size());
    for (size_t q = 0; q < H.h_own.size(); ++q) down[q] = pos[H.h_own[q]];
    CK(H.own.alloc(std::max<size_t>(down.size(), 1)));
    if (!down.empty()) CK(cudaMemcpy(H.own.p, down.data(), down.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(H.connF.alloc((size_t)std::max(ncf, 1) * H.nc));
  }
  c->nchim = 0;
  for (const HRec& r : c->recs) c->nchim += r.type == 102;
  c->have_chimera = c->nchim == 0;
  c->have_records = true;
  free_graphs(c);
  return 0;
}

// The donors of the table's chimera records (ICE_bc_type%ni, donorID, volume_fraction,
// base/Advanced_Types_m.f90:29-31, as read_bc reads them, io/IO_BC.f90:209-236), attached to the
// family record lists that ice_gpu_set_records built.
int ice_gpu_set_chimera(ice_gpu_ctx* c, int32_t nrec, const int32_t* nchi, const int32_t* donor, const double* weight) {
  if (!c) return ICE_GPU_EINVAL;
  if (!c->have_records) return fail(c, ICE_GPU_ENOTREADY, "set_chimera: set the boundary table first");
  if (nrec != (int32_t)c->recs.size() || (nrec > 0 && !nchi))
    return fail(c, ICE_GPU_EINVAL, "set_chimera: %d records given, the table has %d", nrec, (int)c->recs.size());
  std::vector<long long> off(nrec + 1, 0);
  for (int n = 0; n < nrec; ++n) {
    const int n1 = nchi[2 * n], n2 = nchi[2 * n + 1];
    if (n1 < 0 || n2 < 0) return fail(c, ICE_GPU_EINVAL, "record %d: negative donor count", n + 1);
    if (c->recs[n].type != 102 && (n1 || n2))
      return fail(c, ICE_GPU_EINVAL, "record %d: donors given to a record of code %d", n + 1, c->recs[n].type);
    if (c->recs[n].type == 102 && (n1 < 1 || n2 < 1))
      return fail(c, ICE_GPU_EINVAL, "record %d: a chimera record needs donors for both ghost layers", n + 1);
    off[n + 1] = off[n] + n1 + n2;
  }
  if (off[nrec] > 0 && (!donor || !weight)) return fail(c, ICE_GPU_EINVAL, "set_chimera: null donor arrays");
  if (off[nrec] > (1LL << 30)) return fail(c, ICE_GPU_EINVAL, "set_chimera: %lld donors", off[nrec]);
  for (long long s = 0; s < off[nrec]; ++s) {
    const int32_t* d = donor + 4 * s;
    if (d[0] < 1 || d[0] > c->nb) return fail(c, ICE_GPU_EINVAL, "donor %lld: block %d", s + 1, d[0]);
    const int* dm = &c->dims[3 * (d[0] - 1)];
    if (d[1] < 1 || d[1] > dm[0] || d[2] < 1 || d[2] > dm[1] || d[3] < 1 || d[3] > dm[2])
      return fail(c, ICE_GPU_EINVAL, "donor %lld: cell %d %d %d is not an interior cell of block %d", s + 1, d[1], d[2],
                  d[3], d[0]);
    if (!std::isfinite(weight[s])) return fail(c, ICE_GPU_EINVAL, "donor %lld: weight is not finite", s + 1);
  }
  for (int p = 0; p < c->P.nfam; ++p) {
    FamHost& H = c->fam[p];
    std::vector<int4> dn;
    std::vector<double> dw;
    for (size_t q = 0; q < H.h_grp.size(); ++q) {
      const int n = H.h_grp[q];
      DRec& d = H.h_recs[q];
      d.cd0 = (int)dn.size(); d.cn1 = nchi[2 * n]; d.cn2 = nchi[2 * n + 1];
      for (long long s = off[n]; s < off[n + 1]; ++s) {
        const int32_t* x = donor + 4 * s;
        dn.push_back(make_int4(x[0] - 1, x[1] - 1, x[2] - 1, x[3] - 1));
        dw.push_back(weight[s]);
      }
    }
    if (int rc = upload_recs(c, H)) return rc;
    CK(H.cdon.alloc(std::max<size_t>(dn.size(), 1)));
    CK(H.cw.alloc(std::max<size_t>(dw.size(), 1)));
    if (!dn.empty()) {
      CK(cudaMemcpy(H.cdon.p, dn.data(), dn.size() * sizeof(int4), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(H.cw.p, dw.data(), dw.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
  }
  c->have_chimera = true;
  free_graphs(c);
  return 0;
}

// The coupler's imports into family p of block b (ICE_cond_phase_type%imports, which the coupler's
// add_birth_rate, add_absorption_rate and add_removal_rate accumulate: coupling/Mod_Exchange.f90:270-390),
// (ncond, ni, nj, nk) in the driver's layout; NULL sets the block's to zero. The first call for a family
// allocates them (zero elsewhere), and from then on the family's steps add them to the residual and
// bound its steps as bound_empty_dt and bound_removal_dt do.
int ice_gpu_set_imports(ice_gpu_ctx* c, int32_t b1, int32_t p1, const double* imports) {
  if (!c) return ICE_GPU_EINVAL;
  if (b1 < 1 || b1 > c->nb || p1 < 1 || p1 > c->P.nfam) return fail(c, ICE_GPU_EINVAL, "set_imports: bad block/family");
  FamHost& H = c->fam[p1 - 1];
  const DBlock& B = c->hblk[b1 - 1];
  const long long n = (long long)B.ni * B.nj * B.nk;
  if (imports)
    for (long long q = 0; q < n * H.nc; ++q)
      if (!std::isfinite(imports[q])) return fail(c, ICE_GPU_EINVAL, "set_imports: a rate is not finite");
  CK(cudaStreamSynchronize(c->stream));
  if (!H.have_imp) {
    CK(H.imp.alloc((size_t)c->NI * H.nc));
    CK(cudaMemset(H.imp.p, 0, (size_t)c->NI * H.nc * sizeof(double)));
    CK(H.escan.alloc(1));
    H.have_imp = true;
    free_graphs(c);
  }
  std::vector<double> col((size_t)n);
  for (int v = 0; v < H.nc; ++v) {
    for (long long q = 0; q < n; ++q) col[(size_t)q] = imports ? imports[q * H.nc + v] : 0.0;
    CK(cudaMemcpy(H.imp.p + (long long)v * c->NI + B.ioff, col.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
  }
  return 0;
}

// Two-way coupling (twcoupled): every stage adds its source to the step's running sum
// (add_stage_source, Mod_Explicit.f90:257-280), which the gas reads after the step as exchange_rate.
int ice_gpu_set_exchange(ice_gpu_ctx* c, int32_t on) {
  if (!c) return ICE_GPU_EINVAL;
  if (on && !c->P.coupled) return fail(c, ICE_GPU_EINVAL, "set_exchange: the run is not coupled to a gas");
  CK(cudaStreamSynchronize(c->stream));
  if (on && !c->exchange)
    for (int p = 0; p < c->P.nfam; ++p) {
      FamHost& H = c->fam[p];
      CK(H.xstep.alloc((size_t)5 * c->NI));
      CK(cudaMemset(H.xstep.p, 0, (size_t)5 * c->NI * sizeof(double)));
    }
  c->exchange = on != 0;
  free_graphs(c);
  return 0;
}

// exchange_rate (coupling/Mod_Exchange.f90:60-78) of every cell of family p in block b over the last step,
// (5, ni, nj, nk): the mass, momentum and energy the gas receives per unit volume and time, the
// negated step source of the family (no burning family: nothing generated, no heat of reaction).
int ice_gpu_exchange_rate(ice_gpu_ctx* c, int32_t b1, int32_t p1, double* x) {
  if (!c) return ICE_GPU_EINVAL;
  if (b1 < 1 || b1 > c->nb || p1 < 1 || p1 > c->P.nfam || !x) return fail(c, ICE_GPU_EINVAL, "exchange_rate: bad arguments");
  if (!c->exchange) return fail(c, ICE_GPU_ENOTREADY, "exchange_rate: exchange is off (ice_gpu_set_exchange)");
  const DBlock& B = c->hblk[b1 - 1];
  const long long n = (long long)B.ni * B.nj * B.nk;
  std::vector<double> col((size_t)n);
  CK(cudaStreamSynchronize(c->stream));
  for (int m = 0; m < 5; ++m) {
    CK(cudaMemcpy(col.data(), c->fam[p1 - 1].xstep.p + (long long)m * c->NI + B.ioff, (size_t)n * sizeof(double),
                  cudaMemcpyDeviceToHost));
    for (long long q = 0; q < n; ++q) x[q * 5 + m] = -col[(size_t)q];
  }
  return 0;
}

int ice_gpu_index_maps(const ice_gpu_ctx* c, int32_t p1, int32_t* nbcell, int32_t* first, int32_t* nrecs,
                       int32_t* recs, int32_t* nown, int32_t* own) {
  if (!c || p1 < 1 || p1 > c->P.nfam || !nbcell || !nrecs || !nown) return ICE_GPU_EINVAL;
  const FamHost& H = c->fam[p1 - 1];
  *nbcell = H.nbc; *nrecs = (int)H.h_list.size(); *nown = H.nown;
  if (first) for (size_t q = 0; q < H.h_first.size(); ++q) first[q] = H.h_first[q] + 1;
  if (recs) for (size_t q = 0; q < H.h_list.size(); ++q) recs[q] = H.h_list[q] + 1;
  if (own) for (size_t q = 0; q < H.h_own.size(); ++q) own[q] = H.h_own[q] + 1;
  return 0;
}

static int check_ready(ice_gpu_ctx* c) {
  for (int b = 0; b < c->nb; ++b) if (!c->have_block[b]) return fail(c, ICE_GPU_ENOTREADY, "block %d has no metrics", b + 1);
  if (!c->have_records) return fail(c, ICE_GPU_ENOTREADY, "no boundary table");
  if (!c->have_chimera)
    return fail(c, ICE_GPU_ENOTREADY, "%d chimera records have no donors (ice_gpu_set_chimera)", c->nchim);
  // the sources of a coupled run and the ghosts of its 401 and 403 inlets read the gas of their block:
  // refused here, before any launch, where a block has none (an uncoupled run's injecting 401 or 403
  // inlets were refused by ice_gpu_set_records)
  if (c->P.coupled && !c->have_gas) return fail(c, ICE_GPU_ENOTREADY, "a coupled run needs the gas of every block");
  return 0;
}

static int finish_step(ice_gpu_ctx* c, ice_gpu_step_out* out, float dms);

int ice_gpu_step(ice_gpu_ctx* c, int32_t nsteps, ice_gpu_step_out* out) {
  if (!c) return ICE_GPU_EINVAL;
  if (int rc = check_ready(c)) return rc;
  if (int rc = build_geo32(c)) return rc;
  if (nsteps < 0) return fail(c, ICE_GPU_EINVAL, "step: nsteps %d", nsteps);
  cudaStream_t s = c->stream;
  if (c->profiling) {
    for (double& x : c->kms) x = 0.0;
    c->nlaunch = 0;
  }
  // res-threshold ends a steady run once its density residual has fallen by res_threshold from the
  // first non-zero one (Mod_Explicit.f90:193-240): such a run takes the norm after every step and the
  // call ends at the step that meets it
  const bool res_stop = !c->P.time_accurate && c->P.res_threshold > 0.0;
  c->res_end = false;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  CK(cudaEventCreate(&t0)); CK(cudaEventCreate(&t1));
  CK(cudaEventRecord(t0, s));
  for (int n = 0; n < nsteps && !c->res_end; ++n) {
    int ph = c->phase;
    if (c->profiling) {
      CK(cudaEventRecord(c->ev0, s));
      enqueue_step(c, ph, s, prof_tick);
      c->nlaunch += launches_per_step(c);
    } else if (!c->owned.empty()) {
      // a split run: launched as it goes, the stream drained at each exchange for the hook
      c->xerr = 0;
      enqueue_step(c, ph, s, nullptr);
      if (c->xerr) {
        cudaStreamSynchronize(s);
        cudaEventDestroy(t0); cudaEventDestroy(t1);
        return c->xerr;
      }
    } else {
      if (!c->graph[ph]) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        enqueue_step(c, ph, s, nullptr);
        CK(cudaStreamEndCapture(s, &g));
        CK(cudaGraphInstantiate(&c->graph[ph], g, 0));
        cudaGraphDestroy(g);
      }
      CK(cudaGraphLaunch(c->graph[ph], s));
    }
    c->prev_phase = ph;
    c->phase = next_phase(c, ph);
    if (res_stop) {
      if (int rc = ice_gpu_residual_norm(c, c->last_norm, nullptr)) {
        cudaEventDestroy(t0); cudaEventDestroy(t1);
        return rc;
      }
      if (c->res_reference == 0.0) c->res_reference = c->last_norm[0];
      c->res_end = c->res_reference > 0.0 && c->last_norm[0] <= c->P.res_threshold * c->res_reference;
    }
  }
  CK(cudaEventRecord(t1, s));
  CK(cudaStreamSynchronize(s));
  float dms = 0.f;
  CK(cudaEventElapsedTime(&dms, t0, t1));
  cudaEventDestroy(t0); cudaEventDestroy(t1);
  return finish_step(c, out, dms);
}

// The step's report from the device status (after the stream has drained).
static int finish_step(ice_gpu_ctx* c, ice_gpu_step_out* out, float dms) {
  CK(cudaGetLastError());
  Status h;
  CK(cudaMemcpy(&h, c->st.p, sizeof h, cudaMemcpyDeviceToHost));
  int rc = 0;
  if (out) {
    out->dtglobal = h.dtglobal; out->time = h.time; out->iter = h.iter; out->status = (int)h.flags;
    const bool res_stop = !c->P.time_accurate && c->P.res_threshold > 0.0;
    out->nfloored = (int64_t)h.nfloored; out->have_norm = res_stop ? 1 : 0;
    out->nrealized = (int64_t)h.nrealized;
    bool endsim = h.iter_from_call >= c->P.itermax || c->res_end || h.time >= c->P.time_threshold;
    bool iosim = c->P.sol_diter > 0 && h.iter % c->P.sol_diter == 0;
    out->todo = endsim ? 3 : iosim ? 2 : 1;
    for (int m = 0; m < 5; ++m) out->residual[m] = res_stop ? c->last_norm[m] : 0.0;
    out->device_ms = dms;
  }
  if (h.flags & (ICE_GPU_ST_NAN_STATE | ICE_GPU_ST_BAD_RECON)) {
    rc = fail(c, ICE_GPU_ESTATE, "%s", (h.flags & ICE_GPU_ST_NAN_STATE) ?
              "invalid state after the update (NaN or infinity)" : "unphysical state at first order on a face");
  }
  return rc;
}

// ice_gpu_step with the state on the host: upload every block and family, nsteps steps, download.
// The uploads run on their own stream into one staging buffer (converted to the pools as each
// block lands); the step waits for them (its dt is a minimum over every family); the last step runs
// one graph per family, converts each family's new state as soon as its own stages end, and its
// download runs on a third stream under the next family's stages. The largest families step first,
// so that the download left after the last stage is the smallest.
int ice_gpu_step_host(ice_gpu_ctx* c, int32_t nsteps, const double* const* prim_in, double* const* prim_out,
                      ice_gpu_step_out* out) {
  if (!c) return ICE_GPU_EINVAL;
  if (int rc = check_ready(c)) return rc;
  if (int rc = build_geo32(c)) return rc;
  if (nsteps < 1) return fail(c, ICE_GPU_EINVAL, "step_host: nsteps %d", nsteps);
  if (!prim_in || !prim_out) return fail(c, ICE_GPU_EINVAL, "step_host: null array list");
  if (!c->owned.empty()) return fail(c, ICE_GPU_EINVAL, "step_host: a split run steps through ice_gpu_step");
  const int nf = c->P.nfam;
  for (int q = 0; q < c->nb * nf; ++q)
    if (!prim_in[q] || !prim_out[q]) return fail(c, ICE_GPU_EINVAL, "step_host: null array for block %d family %d",
                                                 q / nf + 1, q % nf + 1);
  if (c->profiling || (!c->P.time_accurate && c->P.res_threshold > 0.0)) {
    // per-class timing, or a steady run that may end on res-threshold inside the call: the plain
    // calls, one after another
    for (int b = 0; b < c->nb; ++b)
      for (int p = 0; p < nf; ++p)
        if (int rc = ice_gpu_upload_state(c, b + 1, p + 1, prim_in[b * nf + p], nullptr)) return rc;
    if (int rc = ice_gpu_step(c, nsteps, out)) return rc;
    for (int b = 0; b < c->nb; ++b)
      for (int p = 0; p < nf; ++p)
        if (int rc = ice_gpu_download_state(c, b + 1, p + 1, prim_out[b * nf + p])) return rc;
    return 0;
  }
  // staging offsets: block-major, family within
  std::vector<long long> off((size_t)c->nb * nf + 1, 0);
  for (int b = 0; b < c->nb; ++b) {
    const DBlock& B = c->hblk[b];
    const long long ng = (long long)(B.ni + 4) * (B.nj + 4) * (B.nk + 4);
    for (int p = 0; p < nf; ++p) off[(size_t)b * nf + p + 1] = off[(size_t)b * nf + p] + ng * c->fam[p].nc;
  }
  if (c->xall.n < (size_t)off.back()) CK(c->xall.alloc((size_t)off.back()));
  if (!c->s_up) CK(cudaStreamCreateWithFlags(&c->s_up, cudaStreamNonBlocking));
  if (!c->s_down) CK(cudaStreamCreateWithFlags(&c->s_down, cudaStreamNonBlocking));
  if (!c->ev_up) CK(cudaEventCreateWithFlags(&c->ev_up, cudaEventDisableTiming));
  for (int p = 0; p < nf; ++p) if (!c->ev_fam[p]) CK(cudaEventCreateWithFlags(&c->ev_fam[p], cudaEventDisableTiming));
  cudaStream_t s = c->stream;
  CK(cudaStreamSynchronize(s));
  // families by size, largest first (their order within a step does not change any result)
  std::vector<int> order(nf);
  for (int p = 0; p < nf; ++p) order[p] = p;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return c->fam[a].nc > c->fam[b].nc; });
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  CK(cudaEventCreate(&t0)); CK(cudaEventCreate(&t1));
  CK(cudaEventRecord(t0, c->s_up));
  const int ph0 = c->phase;
  for (int p : order)
    for (int b = 0; b < c->nb; ++b) {
      const DBlock& B = c->hblk[b];
      const FamHost& H = c->fam[p];
      const long long ng = (long long)(B.ni + 4) * (B.nj + 4) * (B.nk + 4);
      double* x = c->xall.p + off[(size_t)b * nf + p];
      CK(cudaMemcpyAsync(x, prim_in[b * nf + p], (size_t)ng * H.nc * sizeof(double), cudaMemcpyHostToDevice, c->s_up));
      k_aos2soa<<<grid_of(ng), 256, 0, c->s_up>>>(x, H.S[ph0].p + B.goff, c->NG, ng, H.nc, B.ni + 4, B.nj + 4, B.px);
      CK(cudaGetLastError());
    }
  CK(cudaEventRecord(c->ev_up, c->s_up));
  CK(cudaStreamWaitEvent(s, c->ev_up, 0));
  for (int n = 0; n < nsteps; ++n) {
    const int ph = c->phase;
    if (!c->graph_pre[ph]) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      enqueue_step_dt(c, ph, s, nullptr);
      CK(cudaStreamEndCapture(s, &g));
      CK(cudaGraphInstantiate(&c->graph_pre[ph], g, 0));
      cudaGraphDestroy(g);
    }
    CK(cudaGraphLaunch(c->graph_pre[ph], s));
    const int phn = next_phase(c, ph);
    for (int p : order) {
      if (!c->graph_fam[ph][p]) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        enqueue_step_family(c, p, ph, s, nullptr);
        CK(cudaStreamEndCapture(s, &g));
        CK(cudaGraphInstantiate(&c->graph_fam[ph][p], g, 0));
        cudaGraphDestroy(g);
      }
      CK(cudaGraphLaunch(c->graph_fam[ph][p], s));
      if (n + 1 < nsteps) continue;
      // the family's new state is final: converted to the caller's layout in order on the step's stream
      // (a conversion kernel beside the stage kernels would wait for SM room), then downloaded on the
      // copy stream beside the next family's stages
      const FamHost& H = c->fam[p];
      for (int b = 0; b < c->nb; ++b) {
        const DBlock& B = c->hblk[b];
        const long long ng = (long long)(B.ni + 4) * (B.nj + 4) * (B.nk + 4);
        double* x = c->xall.p + off[(size_t)b * nf + p];
        k_soa2aos<<<grid_of(ng), 256, 0, s>>>(H.S[phn].p + B.goff, x, c->NG, ng, H.nc, B.ni + 4, B.nj + 4, B.px);
        CK(cudaGetLastError());
      }
      CK(cudaEventRecord(c->ev_fam[p], s));
      CK(cudaStreamWaitEvent(c->s_down, c->ev_fam[p], 0));
      for (int b = 0; b < c->nb; ++b) {
        const DBlock& B = c->hblk[b];
        const long long ng = (long long)(B.ni + 4) * (B.nj + 4) * (B.nk + 4);
        CK(cudaMemcpyAsync(prim_out[b * nf + p], c->xall.p + off[(size_t)b * nf + p],
                           (size_t)ng * H.nc * sizeof(double), cudaMemcpyDeviceToHost, c->s_down));
      }
    }
    c->prev_phase = ph;
    c->phase = phn;
  }
  CK(cudaEventRecord(t1, c->s_down));
  CK(cudaStreamSynchronize(c->s_down));
  CK(cudaStreamSynchronize(s));
  float dms = 0.f;
  CK(cudaEventElapsedTime(&dms, t0, t1));
  cudaEventDestroy(t0); cudaEventDestroy(t1);
  return finish_step(c, out, dms);
}

int ice_gpu_residual_norm(ice_gpu_ctx* c, double* total, double* fam) {
  if (!c || !total) return ICE_GPU_EINVAL;
  if (c->prev_phase < 0) return fail(c, ICE_GPU_ENOTREADY, "residual_norm: no step taken since the state was set");
  Geo G = make_geo(c);
  int nf = c->P.nfam;
  std::vector<double> part((size_t)c->nb * nf * 5, 0.0);
  std::vector<double> h((size_t)c->nchunk * 5);
  for (int p = 0; p < nf; ++p) {
    FamHost& H = c->fam[p];
    k_norm<<<c->nchunk, 256, 0, c->stream>>>(G, H.S[c->phase].p, H.S[c->prev_phase].p, nbase_of(H.closure) - 2,
                                             c->chunks.p, c->npart.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h.data(), c->npart.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int q = 0; q < c->nchunk; ++q) {
      if (!c->owned.empty() && !c->owned[c->chunk_block[q]]) continue;    // another rank's block
      double* a = &part[((size_t)c->chunk_block[q] * nf + p) * 5];
      for (int m = 0; m < 5; ++m) a[m] = a[m] + h[(size_t)q * 5 + m];
    }
  }
  // a split run: every block's partial sums come from the one rank that steps it (the others add
  // zeros), so the sums below keep the block order of an unsplit run
  if (int rc = halo_reduce(c, ICE_GPU_HALO_NORM, part.data(), (long long)part.size())) return rc;
  double tot[5] = {0, 0, 0, 0, 0};
  for (int b = 0; b < c->nb; ++b) for (int p = 0; p < nf; ++p) for (int m = 0; m < 5; ++m) tot[m] = tot[m] + part[((size_t)b * nf + p) * 5 + m];
  for (int m = 0; m < 5; ++m) total[m] = sqrt(tot[m]);
  if (fam) {
    for (int p = 0; p < nf; ++p) {
      double f[5] = {0, 0, 0, 0, 0};
      for (int b = 0; b < c->nb; ++b) for (int m = 0; m < 5; ++m) f[m] = f[m] + part[((size_t)b * nf + p) * 5 + m];
      for (int m = 0; m < 5; ++m) fam[p * 5 + m] = sqrt(f[m]);
    }
  }
  return 0;
}

// ---------------------------------------------------------------- the block split
int ice_gpu_set_partition(ice_gpu_ctx* c, const int32_t* owned) {
  if (!c) return ICE_GPU_EINVAL;
  if (!owned) {
    c->owned.clear();
  } else {
    if (c->P.irs) return fail(c, ICE_GPU_EINVAL, "set_partition: IRS is not supported in a split run");
    if (c->nchim > 0) return fail(c, ICE_GPU_EINVAL, "set_partition: chimera records are not supported in a split run");
    for (int p = 0; p < c->P.nfam; ++p)
      if (c->fam[p].have_imp) return fail(c, ICE_GPU_EINVAL, "set_partition: imports are not supported in a split run");
    std::vector<unsigned char> o(c->nb);
    int n = 0;
    for (int b = 0; b < c->nb; ++b) { o[b] = owned[b] != 0; n += o[b]; }
    if (n == 0) return fail(c, ICE_GPU_EINVAL, "set_partition: this rank steps no block");
    c->owned = o;
    CK(c->owned_dev.alloc(c->nb));
    CK(cudaMemcpy(c->owned_dev.p, o.data(), c->nb, cudaMemcpyHostToDevice));
  }
  CK(cudaStreamSynchronize(c->stream));
  free_graphs(c);
  if (build_tiles(c)) return ICE_GPU_ECUDA;
  return 0;
}

int ice_gpu_set_halo(ice_gpu_ctx* c, int32_t kind, int32_t p1, int32_t nsend, const int32_t* send, int32_t nrecv,
                     const int32_t* recv) {
  if (!c) return ICE_GPU_EINVAL;
  if (kind < 0 || kind > 2 || p1 < 1 || p1 > c->P.nfam || nsend < 0 || nrecv < 0 || (nsend > 0 && !send) ||
      (nrecv > 0 && !recv))
    return fail(c, ICE_GPU_EINVAL, "set_halo: bad arguments");
  const int p = p1 - 1;
  std::vector<int4> lists[2];
  for (int side = 0; side < 2; ++side) {
    const int n = side ? nrecv : nsend;
    const int32_t* e = side ? recv : send;
    for (int q = 0; q < n; ++q) {
      const int32_t* x = e + 4 * q;
      if (kind == ICE_GPU_HALO_FLUX) {
        if (x[0] < 1 || x[0] > c->fam[p].ncf) return fail(c, ICE_GPU_EINVAL, "set_halo: connection face %d", x[0]);
        lists[side].push_back(make_int4(x[0] - 1, 0, 0, 0));
        continue;
      }
      if (x[0] < 1 || x[0] > c->nb) return fail(c, ICE_GPU_EINVAL, "set_halo: block %d", x[0]);
      const int* d = &c->dims[3 * (x[0] - 1)];
      if (x[1] < 1 || x[1] > d[0] || x[2] < 1 || x[2] > d[1] || x[3] < 1 || x[3] > d[2])
        return fail(c, ICE_GPU_EINVAL, "set_halo: cell %d %d %d outside block %d", x[1], x[2], x[3], x[0]);
      lists[side].push_back(make_int4(x[0] - 1, x[1] - 1, x[2] - 1, x[3] - 1));
    }
  }
  c->hs[kind][p] = lists[0];
  c->hr[kind][p] = lists[1];
  CK(c->hs_dev[kind][p].alloc(lists[0].size()));
  CK(c->hr_dev[kind][p].alloc(lists[1].size()));
  if (!lists[0].empty())
    CK(cudaMemcpy(c->hs_dev[kind][p].p, lists[0].data(), lists[0].size() * sizeof(int4), cudaMemcpyHostToDevice));
  if (!lists[1].empty())
    CK(cudaMemcpy(c->hr_dev[kind][p].p, lists[1].data(), lists[1].size() * sizeof(int4), cudaMemcpyHostToDevice));
  return 0;
}

int ice_gpu_set_exchange_hook(ice_gpu_ctx* c, ice_gpu_exchange_fn fn, void* user) {
  if (!c) return ICE_GPU_EINVAL;
  c->hook = fn; c->hook_user = user;
  return 0;
}

int ice_gpu_set_profiling(ice_gpu_ctx* c, int32_t on) {
  if (!c) return ICE_GPU_EINVAL;
  c->profiling = on != 0;
  return 0;
}

int ice_gpu_kernel_times(const ice_gpu_ctx* c, double* ms, int32_t nclass, int64_t* nlaunch) {
  if (!c) return ICE_GPU_EINVAL;
  for (int q = 0; q < nclass && q < KC_N; ++q) ms[q] = c->kms[q];
  if (nlaunch) *nlaunch = c->profiling ? c->nlaunch : 0;
  return 0;
}

// ---------------------------------------------------------------- the evaporation surrogate
int ice_gpu_surrogate_train(ice_gpu_ctx* c, int32_t p1, const ice_gpu_surrogate_opts* o, ice_gpu_surrogate_report* rep) {
  if (!c || !o) return ICE_GPU_EINVAL;
  if (p1 < 1 || p1 > c->P.nfam) return fail(c, ICE_GPU_EINVAL, "surrogate_train: family %d out of range", p1);
  if (int rc = check_ready(c)) return rc;
  if (!c->P.coupled) return fail(c, ICE_GPU_EINVAL, "surrogate_train: the run is not coupled (no source to replace)");
  const ice_gpu_family& pf = c->P.fam[p1 - 1];
  if (pf.evap == 0) return fail(c, ICE_GPU_EINVAL, "surrogate_train: family %d has no evaporation", p1);
  if (o->nsamples < 1024 || o->nsamples > (1LL << 26) || o->epochs < 1 || o->batch < 64 || o->batch > 65536 ||
      !(o->lr > 0) || !(o->val_frac > 0 && o->val_frac < 0.5))
    return fail(c, ICE_GPU_EINVAL, "surrogate_train: options out of range");
  FamHost& H = c->fam[p1 - 1];
  DevBuf<float> X, T;
  CK(X.alloc((size_t)o->nsamples * MLP_IN));
  CK(T.alloc((size_t)o->nsamples * 2));
  FamDev F = make_famdev(c, p1 - 1, 1, c->phase);
  if (mlp_make_samples(H.closure, make_geo(c), F, c->P.drag, c->P.heat, c->P.blow, o->nsamples, o->seed, o->jitter,
                       X.p, T.p, c->stream))
    return fail(c, ICE_GPU_ECUDA, "surrogate_train: sample kernel: %s", cudaGetErrorString(cudaGetLastError()));
  MlpTrainOpts to{o->nsamples, o->epochs, o->batch, o->lr, o->jitter, o->seed, o->val_frac};
  MlpTrainReport tr{};
  std::string err;
  if (mlp_train(X.p, T.p, o->nsamples, to, H.mlp_w, H.mlp_norm, tr, c->stream, err))
    return fail(c, ICE_GPU_ECUDA, "%s: %s", err.c_str(), cudaGetErrorString(cudaGetLastError()));
  std::vector<unsigned char> img;
  mlp_image(H.mlp_w.data(), img);
  CK(H.mlp_img.alloc(img.size()));
  CK(cudaMemcpy(H.mlp_img.p, img.data(), img.size(), cudaMemcpyHostToDevice));
  H.sur_on = true;
  free_graphs(c);
  if (rep) {
    rep->train_loss = tr.train_loss; rep->val_loss = tr.val_loss;
    rep->mdot_rel_median = tr.mdot_rel_median; rep->mdot_rel_p99 = tr.mdot_rel_p99;
    rep->q_rel_median = tr.q_rel_median; rep->q_rel_p99 = tr.q_rel_p99;
    rep->seconds = tr.seconds; rep->nsamples = tr.nsamples; rep->steps = tr.steps;
    for (int a = 0; a < MLP_IN; ++a) { rep->env_lo[a] = H.mlp_norm.env_lo[a]; rep->env_hi[a] = H.mlp_norm.env_hi[a]; }
  }
  return 0;
}

int ice_gpu_surrogate_enable(ice_gpu_ctx* c, int32_t p1, int32_t on) {
  if (!c) return ICE_GPU_EINVAL;
  if (p1 < 1 || p1 > c->P.nfam) return fail(c, ICE_GPU_EINVAL, "surrogate_enable: family %d out of range", p1);
  FamHost& H = c->fam[p1 - 1];
  if (on && !H.mlp_img.p) return fail(c, ICE_GPU_ENOTREADY, "surrogate_enable: family %d has no trained network", p1);
  CK(cudaStreamSynchronize(c->stream));
  H.sur_on = on != 0;
  free_graphs(c);
  return 0;
}

int ice_gpu_surrogate_stats(const ice_gpu_ctx* c, int64_t* counts) {
  if (!c || !counts) return ICE_GPU_EINVAL;
  Status h;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess ||
      cudaMemcpy(&h, c->st.p, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return ICE_GPU_ECUDA;
  counts[0] = (int64_t)h.sur_cells; counts[1] = (int64_t)h.sur_env; counts[2] = (int64_t)h.sur_res;
  return 0;
}

int ice_gpu_mlp_grad(const float* w, const float* x, const float* t, int32_t n, float* grad, float* loss) {
  if (!w || !x || !t || !grad || !loss || n < 1 || n > 65536) return fail(nullptr, ICE_GPU_EINVAL, "mlp_grad: bad arguments");
  std::string err;
  if (mlp_grad_host(w, x, t, n, grad, loss, err)) return fail(nullptr, ICE_GPU_ECUDA, "%s", err.c_str());
  return 0;
}

int ice_gpu_mlp_infer(const float* w, const float* x, int32_t n, float* y) {
  if (!w || !x || !y || n < 1) return fail(nullptr, ICE_GPU_EINVAL, "mlp_infer: bad arguments");
  std::string err;
  if (mlp_infer_host(w, x, n, y, err)) return fail(nullptr, ICE_GPU_ECUDA, "%s", err.c_str());
  return 0;
}

// Pair_Connections (io/IO_BC.f90:360-510)
int ice_gpu_pair_connections(int32_t nb, const int32_t* dims, int32_t ngroups, int32_t nrec, int32_t* rec,
                             char* err, int32_t errlen) {
  auto R = [&](int n, int f) -> int32_t& { return rec[(long long)n * ICE_GPU_REC_INTS + f]; };
  enum { Fb, Fi, Fj, Fk, Ff, Ftype, Fp, Fbs, Fis, Fjs, Fks, Ffs, Fpartner, Fowner, Fcf };
  auto tang = [](int f, int i, int j, int k, int* t) {
    if (f <= 2) { t[0] = j; t[1] = k; } else if (f <= 4) { t[0] = i; t[1] = k; } else { t[0] = i; t[1] = j; }
  };
  auto msg = [&](const char* fmt, int a, int b2) {
    if (err && errlen > 0) snprintf(err, errlen, fmt, a, b2);
    return ICE_GPU_EINVAL;
  };
  if (nb < 1 || ngroups < 1 || nrec < 0 || !dims || (nrec > 0 && !rec)) return msg("bad arguments (%d %d)", nb, ngroups);
  for (int n = 0; n < nrec; ++n)
    if (R(n, Ftype) == 101 || R(n, Ftype) == 201) { R(n, Fpartner) = 0; R(n, Fowner) = 0; R(n, Fcf) = 0; }
  for (int p = 1; p <= ngroups; ++p) {
    std::vector<std::vector<int>> map((size_t)nb * 6);
    std::vector<int> mdim((size_t)nb * 12, 0);
    for (int n = p - 1; n < nrec; n += ngroups) {
      int ty = R(n, Ftype);
      if (ty != 101 && ty != 201) continue;
      int b = R(n, Fb), f = R(n, Ff), t[2], nt[2];
      if (b < 1 || b > nb || f < 1 || f > 6) return msg("record %d: bad block or face %d", n + 1, f);
      size_t key = (size_t)(b - 1) * 6 + (f - 1);
      if (map[key].empty()) {
        tang(f, dims[3 * (b - 1)], dims[3 * (b - 1) + 1], dims[3 * (b - 1) + 2], nt);
        map[key].assign((size_t)nt[0] * nt[1], 0);
        mdim[2 * key] = nt[0]; mdim[2 * key + 1] = nt[1];
      }
      tang(f, R(n, Fi), R(n, Fj), R(n, Fk), t);
      if (t[0] < 1 || t[1] < 1 || t[0] > mdim[2 * key] || t[1] > mdim[2 * key + 1]) return msg("record %d: cell off its face %d", n + 1, f);
      map[key][(size_t)(t[1] - 1) * mdim[2 * key] + (t[0] - 1)] = n + 1;
    }
    for (int n = p - 1; n < nrec; n += ngroups) {
      int ty = R(n, Ftype);
      if (ty != 101 && ty != 201) continue;
      int b = R(n, Fbs), f = R(n, Ffs), q = 0, t[2];
      if (b >= 1 && b <= nb && f >= 1 && f <= 6) {
        size_t key = (size_t)(b - 1) * 6 + (f - 1);
        if (!map[key].empty()) {
          tang(f, R(n, Fis), R(n, Fjs), R(n, Fks), t);
          if (t[0] >= 1 && t[1] >= 1 && t[0] <= mdim[2 * key] && t[1] <= mdim[2 * key + 1])
            q = map[key][(size_t)(t[1] - 1) * mdim[2 * key] + (t[0] - 1)];
        }
      }
      if (q) {
        int qq = q - 1;
        if (R(qq, Fi) != R(n, Fis) || R(qq, Fj) != R(n, Fjs) || R(qq, Fk) != R(n, Fks)) q = 0;
      }
      if (!q) return msg("record %d points at no connection record of its family (face %d)", n + 1, f);
      if (q == n + 1) return msg("record %d points at its own cell and face %d", n + 1, f);
      int qq = q - 1;
      if (R(qq, Ftype) != ty || R(qq, Fbs) != R(n, Fb) || R(qq, Ffs) != R(n, Ff) || R(qq, Fis) != R(n, Fi) ||
          R(qq, Fjs) != R(n, Fj) || R(qq, Fks) != R(n, Fk))
        return msg("records %d and %d do not point at each other", n + 1, q);
      int across = dims[3 * (b - 1) + (f + 1) / 2 - 1];
      if (across < 2) return msg("record %d: the block across has %d cell across its face", n + 1, across);
      R(n, Fpartner) = q;
      int fn = R(n, Ff), fq = R(qq, Ff);
      if (fn % 2 == 0 && fq % 2 == 1) R(n, Fowner) = 1;
      else if (fn % 2 == 1 && fq % 2 == 0) R(n, Fowner) = 0;
      else {
        int k1[5] = {R(n, Fb), R(n, Ff), R(n, Fk), R(n, Fj), R(n, Fi)};
        int k2[5] = {R(qq, Fb), R(qq, Ff), R(qq, Fk), R(qq, Fj), R(qq, Fi)};
        int less = 0;
        for (int m = 0; m < 5; ++m) if (k1[m] != k2[m]) { less = k1[m] < k2[m]; break; }
        R(n, Fowner) = less;
      }
    }
    int nf = 0;
    for (int n = p - 1; n < nrec; n += ngroups) {
      int ty = R(n, Ftype);
      if ((ty != 101 && ty != 201) || !R(n, Fowner)) continue;
      ++nf;
      R(n, Fcf) = nf;
      R(R(n, Fpartner) - 1, Fcf) = nf;
    }
  }
  return 0;
}

}  // extern "C"
