// ice_mlp.cuh -- the evaporation surrogate: a 7 -> 128 x 4 -> 2 SiLU network in place of the
// iterative closure of the mass and heat transfer rates (compute_source_, Mod_Sources.f90:520-551;
// evaporation + lkCorrection, Lib_Evaporation.f90:145-261), and its inference on the tensor cores.
//
// Inputs (raw): log particle radius, particle T, gas T, |relative velocity|, vapour mass fraction
// far from the drop, gas pressure, particle Reynolds number. They are standardised with the mean and
// standard deviation of the training samples. Outputs: the mass and heat transfer rates relative to
// references the cell evaluates without iterating (closure_ref), standardised. A cell uses the network's rates only inside the envelope of the training inputs and
// when the closure's own equations, evaluated once at those rates, agree with them to 1e-3 (one
// Langmuir-Knudsen fixed-point map for the mass rate, the heat formula for the heat rate); any other
// cell runs the plain closure.
//
// Inference: BF16 operands, FP32 accumulation, tcgen05.mma (kind::f16, cta_group::1, M = 128) with
// the activations of 128 cells (one per thread of four warps) and the layer's weights in shared memory
// in the K-major core-matrix layout without swizzle (8 rows x 16 bytes per core matrix), the
// accumulator in tensor memory, read back with tcgen05.ld (32 lanes x 32 columns per warp).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <string>
#include <vector>
#include "ice_layout.cuh"
#include "ice_tma.cuh"

namespace ice {

constexpr int MLP_IN = 7, MLP_H = 128, MLP_OUT = 2, MLP_NL = 5;    // layers 0..4
constexpr int MLP_K0 = 16;      // layer 0's K in the tensor-core image: 7 inputs, a 1 for the bias, 8 zeros
constexpr int MLP_N4 = 16;      // layer 4's N in the image: 2 outputs, 14 zero rows
__host__ __device__ constexpr int mlp_in(int l) { return l == 0 ? MLP_IN : MLP_H; }
__host__ __device__ constexpr int mlp_out(int l) { return l == MLP_NL - 1 ? MLP_OUT : MLP_H; }
__host__ __device__ constexpr int mlp_woff(int l) {
  int o = 0;
  for (int q = 0; q < l; ++q) o += mlp_in(q) * mlp_out(q) + mlp_out(q);
  return o;
}
__host__ __device__ constexpr int mlp_boff(int l) { return mlp_woff(l) + mlp_in(l) * mlp_out(l); }
constexpr int MLP_NPARAM = mlp_woff(MLP_NL);          // FP32 master parameters: W_l [out][in] then b_l

// The BF16 shared-memory image (bytes): W0 (N 128, K 16, the bias in column 7), W1..W3 (128 x 128),
// W4 (N 16, K 128), then the FP32 biases of layers 1..4.
__host__ __device__ constexpr int mlp_img_w(int l) {
  return l == 0 ? 0 : l == 1 ? 128 * MLP_K0 * 2 : 128 * MLP_K0 * 2 + (l - 1) * 128 * 128 * 2;
}
constexpr int MLP_IMG_BIAS = 128 * MLP_K0 * 2 + 3 * 128 * 128 * 2 + MLP_N4 * 128 * 2;   // 106,496
constexpr int MLP_IMG_BYTES = MLP_IMG_BIAS + (3 * 128 + 4) * 4;                       // + b1..b3, b4 (padded)

// byte offset of element (row r, column k) of a K-major operand with K columns in core matrices
__host__ __device__ constexpr int core_off(int r, int k, int K) {
  return ((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}


// Normalisation and envelope of a trained network (host and device).
struct MlpNorm {
  float in_mean[MLP_IN], in_std[MLP_IN], out_mean[MLP_OUT], out_std[MLP_OUT];
  float env_lo[MLP_IN], env_hi[MLP_IN];
};

// Training options and report (ice_gpu_surrogate_train).
struct MlpTrainOpts {
  long long nsamples;     // training pairs drawn from the plain closure
  int epochs, batch;
  double lr;              // Adam's initial learning rate (cosine decay to 1 % of it)
  double jitter;          // spread of the sampled radius, speed (relative) and temperatures (x 20 K)
  uint64_t seed;
  double val_frac;        // held-out fraction
};
struct MlpTrainReport {
  double train_loss, val_loss, mdot_rel_median, mdot_rel_p99, q_rel_median, q_rel_p99, seconds;
  long long nsamples, steps;
};

// host side (ice_mlp_f32.cu)
int mlp_make_samples(int closure, const Geo& G, const FamDev& F, int drag, int heat_sel, int blow, long long n,
                     uint64_t seed, double jit, float* X, float* T, cudaStream_t s);
int mlp_train(const float* X, const float* T, long long n, const MlpTrainOpts& o, std::vector<float>& w, MlpNorm& nm,
              MlpTrainReport& rep, cudaStream_t s, std::string& err);
void mlp_image(const float* w, std::vector<unsigned char>& img);
void launch_source_mlp(int closure, const LaunchArgs& a, const unsigned char* img, const MlpNorm& nm);
int mlp_grad_host(const float* w, const float* x, const float* t, int n, float* grad, float* loss, std::string& err);
int mlp_infer_host(const float* w, const float* x, int n, float* y, std::string& err);

// ------------------------------------------------------------------ features and the checked closure
// The seven raw inputs of a cell (the quantities compute_source_ forms before the evaporation call).
template <typename R> __device__ __forceinline__ void mlp_features(R Rp, R Ts, R Tg, R du, R Yinf, R pg, R Re, R* f) {
  f[0] = lg(Rp); f[1] = Ts; f[2] = Tg; f[3] = du; f[4] = Yinf; f[5] = pg; f[6] = Re;
}

// The network's two outputs are the two rates relative to references the cell evaluates cheaply:
// the mass transfer rate over the equilibrium (vapour-liquid) rate of the same gas-side model, i.e. the
// closure's first gas-side evaluation, before the Langmuir-Knudsen loop (Lib_Evaporation.f90:205-224),
// and the heat transfer rate over the convective one, 2 Nu k_g pi r (T_g - T_p), before the interface
// override and the blowing factor. Both ratios are smooth and of order one (the Langmuir-Knudsen
// correction and the blowing factor), where the rates themselves span decades and change sign; a zero
// reference (no evaporation, equal temperatures) gives the ratio 1 and the rate 0.
template <typename R> __device__ __forceinline__ void closure_ref(R rhog, R Tg, R gam, R gR, R gmu, R gk, R Ts, R Rp,
                                                                  R Re, R Nu, const Mat& m, R& md_ref, R& Q_ref) {
  Mat mv = m;
  mv.intf = 0;                                    // the equilibrium interface: no Langmuir-Knudsen loop
  R Qd; bool ovr;
  evaporation<R>(rhog, Tg, gam, gR, gmu, gk, Ts, (R)2*Rp, Re, mv, md_ref, Qd, ovr);
  Q_ref = (R)2*Nu*gk*(R)kPi*Rp*(Tg - Ts);
}
template <typename R> __device__ __forceinline__ R mlp_ratio(R x, R ref) { return ref != (R)0 ? x / ref : (R)1; }
template <typename R> __device__ __forceinline__ void mlp_targets(R md, R Q, R md_ref, R Q_ref, R* t) {
  t[0] = mlp_ratio(md, md_ref);
  t[1] = mlp_ratio(Q, Q_ref);
}
template <typename R> __device__ __forceinline__ void mlp_rates(R t0, R t1, R md_ref, R Q_ref, R& md, R& Q) {
  md = t0 * md_ref;
  Q = t1 * Q_ref;
}

// The closure's equations evaluated once at a candidate pair (md, Q): the Langmuir-Knudsen map of the
// mass rate (one pass of lkCorrection's fixed-point loop, Lib_Evaporation.f90:238-258) and the heat
// rate that follows from md. True when both agree with the candidate to `tol` relative (against a
// floor of 1e-6 of the particle's scale pi d mu_g, resp. pi d k_g T_g).
template <typename R> __device__ bool closure_check(R rhog, R Tg, R gamma, R Rg, R mug, R kg, R Tp, R Rp, R Re, R Nu,
                                                   const Mat& m, int blow, R md, R Q, R tol) {
  const R pi = (R)kPi;
  const R dp = (R)2*Rp;
  const R smd = (R)1e-6*pi*dp*mug, sq = (R)1e-6*pi*dp*kg*Tg;
  R mdN = (R)0, QdN = (R)0;
  bool ovrN = false;
  if (m.evap != 0) {
    const double* ep = m.ep;
    EvapEnv<R> e;
    e.rhog = rhog; e.Tg = Tg; e.gamma = gamma; e.Rg = Rg; e.mug = mug; e.kg = kg; e.Tp = Tp; e.dp = dp;
    e.evap = m.evap; e.ep = ep;
    e.cpg = gamma*Rg/(gamma - (R)1);
    e.p = rhog*Rg*Tg;
    e.Mg = (R)kRu/Rg;
    R psat = (R)kPatm*ex(-(R)ep[EP_LVMVRU]*((R)1/Tp - (R)ep[EP_INVTB]));
    R Xs = psat >= e.p ? (R)1 - (R)kXsCap : mn(psat/e.p, (R)1 - (R)kXsCap);
    R Ys = molar2mass(Xs, (R)ep[EP_MV], e.Mg);
    if (Ys > (R)ep[EP_YINF] && (Ys - (R)ep[EP_YINF])/((R)1 - Ys) > (R)0) {
      e.Re05 = sqrt(mx(Re, (R)0));
      e.Pr = mug*e.cpg/kg;
      e.Sc = e.Pr*(R)ep[EP_LE];
      evap_invariants(e);
      if (m.intf == 1) {
        R LKd2 = (R)2*mug*sqrt((R)2*pi*Tp*(R)kRu/(R)ep[EP_MV])/((R)ep[EP_ALPHAE]*e.Sc*e.p)/dp;
        R beta = -md*e.Pr/((R)2*pi*mug*dp);
        R XsN = mx(Xs - LKd2*beta, (R)0);
        R YsN = molar2mass(XsN, (R)ep[EP_MV], e.Mg);
        if (YsN > (R)ep[EP_YINF]) {
          R BMN = (YsN - (R)ep[EP_YINF])/((R)1 - YsN);
          if (BMN > (R)0) gas_side(e, YsN, BMN, mdN, QdN, ovrN);
        }
      } else {
        gas_side(e, Ys, (Ys - (R)ep[EP_YINF])/((R)1 - Ys), mdN, QdN, ovrN);
      }
    }
  }
  R Qc = (R)2*Nu*kg*pi*Rp*(Tg - Tp);
  if (ovrN) Qc = QdN;
  else if (blow == 1) Qc = Qc*blowing<R>(gamma, Rg, mug, kg, (R)m.rho, dp, (R)(4.0/3.0)*pi*(Rp*Rp*Rp)*(R)m.rho, md);
  const bool okm = fabs(mdN - md) <= tol*mx(mx(fabs(mdN), fabs(md)), smd);
  const bool okq = fabs(Qc - Q) <= tol*mx(mx(fabs(Qc), fabs(Q)), sq);
  return okm && okq;
}

// ------------------------------------------------------------------ tcgen05 (sm_100a)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  // K-major, no swizzle: start, leading (K) and stride (M/N) byte offsets in 16-byte units, version 1
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
               :: "r"(dtmem), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(slot)), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// 32 consecutive FP32 columns of this warp's 32 lanes (the thread's own row)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
               "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                 "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                 "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
               : "r"(taddr));
  tmem_wait_ld();
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
  tmem_wait_ld();
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ float silu_f(float x) { return __fdividef(x, 1.0f + __expf(-x)); }

// Shared memory of the inference: the weight image, two activation tiles (128 rows x 128 BF16,
// core-matrix layout) for the two 128-cell tiles of a CTA, the MMA barrier and the TMEM address.
constexpr int MLP_TILES = 2;                               // 128-cell tiles per CTA (256 threads)
constexpr int MLP_THREADS = 128 * MLP_TILES;
__host__ __device__ constexpr int mlp_sm_act() { return (MLP_IMG_BYTES + 127) & ~127; }
constexpr int MLP_SM_BAR = mlp_sm_act() + MLP_TILES * 128 * 128 * 2;
constexpr int MLP_SM_BYTES = MLP_SM_BAR + 16 + 128;        // + the alignment of the base

struct MlpSmem {
  unsigned char* img;      // the weight image
  unsigned char* act;      // MLP_TILES activation tiles
  uint64_t* bar;
  uint32_t* tslot;
};

__device__ __forceinline__ MlpSmem mlp_smem(unsigned char* smdyn) {
  unsigned char* b = smdyn + ((128u - (smem_u32(smdyn) & 127u)) & 127u);
  MlpSmem s;
  s.img = b; s.act = b + mlp_sm_act(); s.bar = (uint64_t*)(b + MLP_SM_BAR); s.tslot = (uint32_t*)(b + MLP_SM_BAR + 8);
  return s;
}

// Set-up of a CTA: copies the weight image from global memory, initialises the barrier, allocates
// 128 TMEM columns per tile (warp 0). Every thread of the CTA calls it.
__device__ __forceinline__ uint32_t mlp_setup(const MlpSmem& s, const unsigned char* __restrict__ gimg) {
  const uint4* src = (const uint4*)gimg;
  uint4* dst = (uint4*)s.img;
  for (int q = threadIdx.x; q < MLP_IMG_BYTES / 16; q += blockDim.x) dst[q] = src[q];
  if (threadIdx.x == 0) { mbar_init(s.bar, 1); fence_mbar_init(); }
  if (threadIdx.x < 32) { tmem_alloc(s.tslot, 128 * MLP_TILES); tmem_relinquish(); }
  fence_proxy_async_smem();                 // the image is read by the tensor cores (async proxy)
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  return *s.tslot;
}

__device__ __forceinline__ void mlp_teardown(const MlpSmem& s, uint32_t tbase) {
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) { tc_fence_after(); tmem_dealloc(tbase, 128 * MLP_TILES); }
}

// Writes the thread's input row (7 standardised inputs, 1, zeros) into its tile's activation buffer.
__device__ __forceinline__ void mlp_put_input(const MlpSmem& s, const float* x) {
  const int t = threadIdx.x >> 7, r = threadIdx.x & 127;
  unsigned char* A = s.act + t * 128 * 128 * 2;
  __align__(16) __nv_bfloat16 v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __float2bfloat16_rn(q < MLP_IN ? x[q] : q == MLP_IN ? 1.0f : 0.0f);
  *(uint4*)(A + core_off(r, 0, MLP_K0)) = *(const uint4*)&v[0];
  *(uint4*)(A + core_off(r, 8, MLP_K0)) = *(const uint4*)&v[8];
}

// The forward pass of every tile of the CTA: all 256 threads call it after mlp_put_input; returns
// the thread's two (standardised) outputs. `parity` is the barrier phase, advanced per layer.
// False when a wait for the tensor cores gave up (two seconds), which the caller reports.
__device__ __forceinline__ bool mlp_forward(const MlpSmem& s, uint32_t tbase, uint32_t& parity, float* y) {
  const int t = threadIdx.x >> 7, r = threadIdx.x & 127, w = (threadIdx.x >> 5) & 3;
  unsigned char* A = s.act + t * 128 * 128 * 2;
  const float* bias = (const float*)(s.img + MLP_IMG_BIAS);
  const uint32_t trow = tbase + ((uint32_t)(32 * w) << 16) + (uint32_t)(128 * t);   // lanes of this warp, tile t
  for (int l = 0; l < MLP_NL; ++l) {
    const int K = l == 0 ? MLP_K0 : MLP_H;
    const int N = l == MLP_NL - 1 ? MLP_N4 : MLP_H;
    fence_proxy_async_smem();               // this thread's activation row, for the tensor cores
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      const uint32_t idesc = umma_idesc_bf16(128, N);
      const uint32_t bimg = smem_u32(s.img + mlp_img_w(l));
      for (int tt = 0; tt < MLP_TILES; ++tt) {
        const uint32_t abase = smem_u32(s.act + tt * 128 * 128 * 2);
        for (int kk = 0; kk < K / 16; ++kk) {
          const uint64_t ad = umma_desc(abase + kk * 256, 128, (K / 8) * 128);
          const uint64_t bd = umma_desc(bimg + kk * 256, 128, (K / 8) * 128);
          umma_bf16(tbase + 128 * tt, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
      }
      umma_commit(s.bar);
    }
    // a wait that gives up ends the pass for every thread of the CTA (after one more bounded wait
    // for the tensor cores' work in flight)
    const bool okw = mbar_wait(s.bar, parity);
    if (__syncthreads_or(!okw)) {
      if (!okw) mbar_wait(s.bar, parity);
      return false;
    }
    parity ^= 1u;
    tc_fence_after();
    if (l < MLP_NL - 1) {
      const float* b = l == 0 ? nullptr : bias + (l - 1) * 128;
#pragma unroll 1
      for (int c0 = 0; c0 < MLP_H; c0 += 32) {
        float v[32];
        tmem_ld32(trow + c0, v);
        __align__(16) __nv_bfloat16 h[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) h[q] = __float2bfloat16_rn(silu_f(b ? v[q] + b[c0 + q] : v[q]));
#pragma unroll
        for (int q = 0; q < 4; ++q) *(uint4*)(A + core_off(r, c0 + 8 * q, MLP_H)) = *(const uint4*)&h[8 * q];
      }
    } else {
      float v[16];
      tmem_ld16(trow, v);
      y[0] = v[0] + bias[3 * 128 + 0];
      y[1] = v[1] + bias[3 * 128 + 1];
    }
  }
  return true;
}

}  // namespace ice
