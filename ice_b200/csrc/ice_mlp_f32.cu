// ice_mlp_f32.cu -- the evaporation surrogate's kernels: training samples from the plain closure,
// training (forward, backward, Adam) in FP32, and the surrogate source kernel with tensor-core inference
// (ice_mlp.cuh). Compiled with the FP32-flux form's flags: the surrogate belongs to that form.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <chrono>
#include "ice_kernels.cuh"
#include "ice_mlp.cuh"

namespace ice {
namespace {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {     // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double unif(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

// ------------------------------------------------------------------ samples
// One training pair per thread: a cell of the family's state drawn at random and moved somewhere in the
// envelope its particles visit in the frozen gas: the particle temperature anywhere between 25 K below
// the cooler of its own and the gas temperature (evaporative cooling) and the warmer of the two, the
// relative speed anywhere between zero and the larger of its own and the gas speed (a particle at rest
// in the moving gas), the radius spread by up to +-jit (relative); then the plain closure's rates in FP64
// for those inputs. X: the seven raw inputs; T: the two targets (mlp_targets).
template <int CL>
__global__ void k_mlp_samples(Geo G, FamDev F, int drag, int heat_sel, int blow, long long n, uint64_t seed, double jit,
                              float* __restrict__ X, float* __restrict__ T) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  constexpr int nc = NC<CL>::v;
  uint64_t h = mix64(seed ^ (uint64_t)s * 0xD1B54A32D192ED03ull);
  const long long q = (long long)(unif(h) * (double)G.NI) % G.NI;
  const DBlock& B = G.blk[find_block(G.blk, G.nb, q)];
  int i, j, k; decode(B, q, i, j, k);
  const long long g = gidx(B, i, j, k);
  double p[nc], gas[5];
#pragma unroll
  for (int v = 0; v < nc; ++v) p[v] = F.Up[(long long)v * G.NG + g];
#pragma unroll
  for (int v = 0; v < 5; ++v) gas[v] = G.gas[(long long)v * G.NI + q];
  const double gR = G.gas[5 * G.NI + q], gg = G.gas[6 * G.NI + q], gk = G.gas[7 * G.NI + q], gm = G.gas[8 * G.NI + q];
  CellPhys<double> c = cell_phys<CL, double>(p, gas, gR, gg, gk, gm, F.mat, drag, heat_sel);
  double u[3];
  for (int a = 0; a < 3; ++a) { h = mix64(h); u[a] = unif(h); }
  const double Rp = c.Rp * ice_exp(jit * (2.0 * u[0] - 1.0));
  const double ug = sqrt(gas[1] * gas[1] + gas[2] * gas[2] + gas[3] * gas[3]);
  const double du = fmax(c.du, ug) * u[1];
  const double Tg = gas[4];
  const double Tlo = fmin(c.T, Tg) - 25.0, Thi = fmax(c.T, Tg);
  const double Ts = Tlo + u[2] * (Thi - Tlo);
  const double rhog = gas[0];
  const double Re = 2.0 * rhog * Rp * du / gm;
  const double Ma = du / sqrt(gg * gR * Tg);
  const double Nu = heat(Re, c.Pr, Ma, heat_sel);
  double md, Q;
  closure_rates<double>(rhog, Tg, gg, gR, gm, gk, Ts, Rp, Re, Nu, F.mat, blow, md, Q);
  double f[MLP_IN];
  mlp_features<double>(Rp, Ts, Tg, du, F.mat.ep[EP_YINF], rhog * gR * Tg, Re, f);
#pragma unroll
  for (int a = 0; a < MLP_IN; ++a) X[s * MLP_IN + a] = (float)f[a];
  double mr, Qr, t[2];
  closure_ref<double>(rhog, Tg, gg, gR, gm, gk, Ts, Rp, Re, Nu, F.mat, mr, Qr);
  mlp_targets<double>(md, Q, mr, Qr, t);
  T[s * 2 + 0] = (float)t[0];
  T[s * 2 + 1] = (float)t[1];
}

// ------------------------------------------------------------------ training (FP32)
// C[M x N] (row-major, ldc) = sum_k A(m, k) B(k, n); A(m, k) = TA ? A[k lda + m] : A[m lda + k],
// B(k, n) = TB ? B[n ldb + k] : B[k ldb + n]. 16 x 16 threads, 16 x 16 tiles.
template <bool TA, bool TB>
__global__ void k_sgemm(int M, int N, int K, const float* __restrict__ A, int lda, const float* __restrict__ Bm, int ldb,
                        float* __restrict__ C, int ldc) {
  __shared__ float As[16][17], Bs[16][17];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int m = blockIdx.y * 16 + ty, n = blockIdx.x * 16 + tx;
  float acc = 0.f;
  for (int k0 = 0; k0 < K; k0 += 16) {
    const int am = blockIdx.y * 16 + ty, ak = k0 + tx;
    As[ty][tx] = (am < M && ak < K) ? (TA ? A[(long long)ak * lda + am] : A[(long long)am * lda + ak]) : 0.f;
    const int bk = k0 + ty, bn = blockIdx.x * 16 + tx;
    Bs[ty][tx] = (bk < K && bn < N) ? (TB ? Bm[(long long)bn * ldb + bk] : Bm[(long long)bk * ldb + bn]) : 0.f;
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) acc += As[ty][kk] * Bs[kk][tx];
    __syncthreads();
  }
  if (m < M && n < N) C[(long long)m * ldc + n] = acc;
}

template <bool TA, bool TB>
void sgemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc, cudaStream_t s) {
  dim3 blk(16, 16), grd((N + 15) / 16, (M + 15) / 16);
  k_sgemm<TA, TB><<<grd, blk, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc);
}

// z += b (per column); a = silu(z), or z on the output layer
__global__ void k_bias_act(float* __restrict__ z, float* __restrict__ a, const float* __restrict__ b, int rows, int cols,
                           int act) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)rows * cols) return;
  const float v = z[e] + b[e % cols];
  z[e] = v;
  a[e] = act ? v / (1.f + expf(-v)) : v;
}

// dz = da * silu'(z) (or da on the output layer), in place on da
__global__ void k_act_bwd(float* __restrict__ da, const float* __restrict__ z, long long n, int act) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !act) return;
  const float sg = 1.f / (1.f + expf(-z[e]));
  da[e] = da[e] * sg * (1.f + z[e] * (1.f - sg));
}

// db[c] = sum over rows of dz
__global__ void k_colsum(const float* __restrict__ dz, float* __restrict__ db, int rows, int cols) {
  const int c = blockIdx.x;
  float acc = 0.f;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) acc += dz[(long long)r * cols + c];
  __shared__ float red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] = red[0];
}

// mean-square loss over rows x 2: dy = 2 (y - t) / (2 rows); loss accumulated in FP64
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy, int rows,
                      double* __restrict__ loss) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  float d = 0.f;
  if (e < rows * 2) {
    d = y[e] - t[e];
    dy[e] = 2.f * d / (float)(rows * 2);
  }
  float sq = d * d;
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, (double)sq / (double)(rows * 2));
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float c1, float c2) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float gg = g[e];
  const float mm = b1 * m[e] + (1.f - b1) * gg, vv = b2 * v[e] + (1.f - b2) * gg * gg;
  m[e] = mm; v[e] = vv;
  w[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + 1e-8f);
}

// a random batch of the training part of the samples, standardised
__global__ void k_gather(const float* __restrict__ X, const float* __restrict__ T, long long ntrain, MlpNorm nm,
                         uint64_t seed, float* __restrict__ xb, float* __restrict__ tb, int rows) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const long long s = (long long)(mix64(seed ^ (uint64_t)r * 0x9E3779B97F4A7C15ull) % (uint64_t)ntrain);
#pragma unroll
  for (int a = 0; a < MLP_IN; ++a) xb[r * MLP_IN + a] = (X[s * MLP_IN + a] - nm.in_mean[a]) / nm.in_std[a];
  tb[r * 2 + 0] = (T[s * 2 + 0] - nm.out_mean[0]) / nm.out_std[0];
  tb[r * 2 + 1] = (T[s * 2 + 1] - nm.out_mean[1]) / nm.out_std[1];
}

// The training network's buffers for a batch of `rows`.
struct Net {
  int rows = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // parameters, gradient, Adam moments
  float *x = nullptr, *t = nullptr, *dy = nullptr;                 // inputs, targets, output gradient
  float *z[MLP_NL] = {}, *a[MLP_NL] = {}, *da = nullptr, *da2 = nullptr;
  double* loss = nullptr;
  cudaError_t alloc(int r) {
    rows = r;
    cudaError_t e = cudaSuccess;
    auto A = [&](float** p, size_t n) { if (e == cudaSuccess) e = cudaMalloc((void**)p, n * sizeof(float)); };
    A(&w, MLP_NPARAM); A(&g, MLP_NPARAM); A(&m, MLP_NPARAM); A(&v, MLP_NPARAM);
    A(&x, (size_t)r * MLP_IN); A(&t, (size_t)r * 2); A(&dy, (size_t)r * 2);
    for (int l = 0; l < MLP_NL; ++l) { A(&z[l], (size_t)r * mlp_out(l)); A(&a[l], (size_t)r * mlp_out(l)); }
    A(&da, (size_t)r * MLP_H); A(&da2, (size_t)r * MLP_H);
    if (e == cudaSuccess) e = cudaMalloc((void**)&loss, sizeof(double));
    return e;
  }
  ~Net() {
    for (float* p : {w, g, m, v, x, t, dy, da, da2}) if (p) cudaFree(p);
    for (int l = 0; l < MLP_NL; ++l) { if (z[l]) cudaFree(z[l]); if (a[l]) cudaFree(a[l]); }
    if (loss) cudaFree(loss);
  }
};

void forward(Net& N, int rows, cudaStream_t s) {
  const float* in = N.x;
  for (int l = 0; l < MLP_NL; ++l) {
    const int I = mlp_in(l), O = mlp_out(l);
    sgemm<false, true>(rows, O, I, in, I, N.w + mlp_woff(l), I, N.z[l], O, s);
    const long long ne = (long long)rows * O;
    k_bias_act<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(N.z[l], N.a[l], N.w + mlp_boff(l), rows, O, l < MLP_NL - 1);
    in = N.a[l];
  }
}

// gradient of the mean-square loss on N.t into N.g; the loss into *N.loss (accumulated)
void backward(Net& N, int rows, cudaStream_t s) {
  k_mse<<<(rows * 2 + 255) / 256, 256, 0, s>>>(N.a[MLP_NL - 1], N.t, N.dy, rows, N.loss);
  float* dcur = N.dy;              // gradient with respect to the layer's output
  for (int l = MLP_NL - 1; l >= 0; --l) {
    const int I = mlp_in(l), O = mlp_out(l);
    const long long ne = (long long)rows * O;
    k_act_bwd<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(dcur, N.z[l], ne, l < MLP_NL - 1);
    const float* inp = l == 0 ? N.x : N.a[l - 1];
    sgemm<true, false>(O, I, rows, dcur, O, inp, I, N.g + mlp_woff(l), I, s);    // dW = dz^T x
    k_colsum<<<O, 256, 0, s>>>(dcur, N.g + mlp_boff(l), rows, O);                  // db
    if (l > 0) {
      float* dnext = dcur == N.da ? N.da2 : N.da;
      sgemm<false, false>(rows, I, O, dcur, O, N.w + mlp_woff(l), I, dnext, I, s);   // dx = dz W
      dcur = dnext;
    }
  }
}

// ------------------------------------------------------------------ inference
// The surrogate source of every cell of one family: its standardised inputs through the network on
// the tensor cores, the closure check, the plain closure where the check fails or the cell lies
// outside the envelope, then the rest of compute_source_. S and tau as k_source writes them.
template <int CL>
__global__ void __launch_bounds__(MLP_THREADS, 1)
k_source_mlp(Geo G, FamDev F, const unsigned char* __restrict__ img, MlpNorm nm, Status* st) {
  extern __shared__ __align__(128) unsigned char smdyn[];
  const MlpSmem S = mlp_smem(smdyn);
  const uint32_t tbase = mlp_setup(S, img);
  uint32_t parity = 0;
  constexpr int nc = NC<CL>::v;
  const float yinf = (float)F.mat.ep[EP_YINF];
  bool ok = true;
  for (long long base = (long long)blockIdx.x * MLP_THREADS; base < G.NI && ok; base += (long long)gridDim.x * MLP_THREADS) {
    const long long q = base + threadIdx.x;
    const bool valid = q < G.NI;
    float x[MLP_IN];
    bool inenv = false;
    float p[nc], gas[5], gR = 0.f, gg = 0.f, gk = 0.f, gm = 0.f;
    CellPhys<float> c{};
    long long g = 0;
    if (valid) {
      const DBlock& B = G.blk[find_block(G.blk, G.nb, q)];
      int i, j, k; decode(B, q, i, j, k);
      g = gidx(B, i, j, k);
#pragma unroll
      for (int v = 0; v < nc; ++v) p[v] = (float)F.Up[(long long)v * G.NG + g];
#pragma unroll
      for (int v = 0; v < 5; ++v) gas[v] = G.gasf[(long long)v * G.NI + q];
      gR = G.gasf[5 * G.NI + q]; gg = G.gasf[6 * G.NI + q];
      gk = G.gasf[7 * G.NI + q]; gm = G.gasf[8 * G.NI + q];
      c = cell_phys<CL, float>(p, gas, gR, gg, gk, gm, F.mat, F.drag, F.heat);
      float f[MLP_IN];
      mlp_features<float>(c.Rp, c.T, gas[4], c.du, yinf, gas[0] * gR * gas[4], c.Re, f);
      inenv = true;
#pragma unroll
      for (int a = 0; a < MLP_IN; ++a) {
        inenv = inenv && f[a] >= nm.env_lo[a] && f[a] <= nm.env_hi[a];
        x[a] = (f[a] - nm.in_mean[a]) / nm.in_std[a];
      }
    } else {
#pragma unroll
      for (int a = 0; a < MLP_IN; ++a) x[a] = 0.f;
    }
    mlp_put_input(S, x);
    float y[2];
    ok = mlp_forward(S, tbase, parity, y);
    bool used = false;
    if (valid && ok) {
      float md, Q, mr, Qr;
      closure_ref<float>(gas[0], gas[4], gg, gR, gm, gk, c.T, c.Rp, c.Re, c.Nu, F.mat, mr, Qr);
      mlp_rates<float>(y[0] * nm.out_std[0] + nm.out_mean[0], y[1] * nm.out_std[1] + nm.out_mean[1], mr, Qr, md, Q);
      used = inenv && closure_check<float>(gas[0], gas[4], gg, gR, gm, gk, c.T, c.Rp, c.Re, c.Nu, F.mat, F.blow, md, Q,
                                           1e-3f);
      if (!used) closure_rates<float>(gas[0], gas[4], gg, gR, gm, gk, c.T, c.Rp, c.Re, c.Nu, F.mat, F.blow, md, Q);
      float s[nc];
      const float tau = cell_source_finish<CL, float>(c, p, gas, F.mat, md, Q, s);
#pragma unroll
      for (int v = 0; v < nc; ++v) F.Sf[(long long)v * G.NI + q] = (F.frozen_mask & (1u << v)) ? 0.f : s[v];
      if (F.write_tau) F.tau[q] = (double)tau;
    }
    // per warp: cells, envelope fallbacks, check fallbacks
    const unsigned mv = __ballot_sync(0xffffffffu, valid), me = __ballot_sync(0xffffffffu, valid && !inenv),
                   mr = __ballot_sync(0xffffffffu, valid && inenv && !used);
    if ((threadIdx.x & 31) == 0 && mv) {
      atomicAdd(&st->sur_cells, (unsigned long long)__popc(mv));
      if (me) atomicAdd(&st->sur_env, (unsigned long long)__popc(me));
      if (mr) atomicAdd(&st->sur_res, (unsigned long long)__popc(mr));
    }
  }
  mlp_teardown(S, tbase);
  if (!ok && threadIdx.x == 0) atomicOr(&st->flags, (unsigned)ICE_GPU_ST_TIMEOUT);
}

// The network alone on standardised inputs (the inference check of the tests): n rows of X in, Y out.
__global__ void __launch_bounds__(MLP_THREADS, 1)
k_mlp_infer(const unsigned char* __restrict__ img, const float* __restrict__ X, float* __restrict__ Y, int n, int* fail) {
  extern __shared__ __align__(128) unsigned char smdyn[];
  const MlpSmem S = mlp_smem(smdyn);
  const uint32_t tbase = mlp_setup(S, img);
  uint32_t parity = 0;
  bool ok = true;
  for (int base = blockIdx.x * MLP_THREADS; base < n && ok; base += gridDim.x * MLP_THREADS) {
    const int r = base + threadIdx.x;
    float x[MLP_IN];
#pragma unroll
    for (int a = 0; a < MLP_IN; ++a) x[a] = r < n ? X[(long long)r * MLP_IN + a] : 0.f;
    mlp_put_input(S, x);
    float y[2];
    ok = mlp_forward(S, tbase, parity, y);
    if (ok && r < n) { Y[2 * r] = y[0]; Y[2 * r + 1] = y[1]; }
  }
  mlp_teardown(S, tbase);
  if (!ok && threadIdx.x == 0) atomicExch(fail, 1);
}

int grid_mlp() {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nsm;
}

// the shared memory the inference kernels take (set on every launch: the kernels of the three closures
// share one signature, so no per-type flag could tell them apart)
template <typename K> void allow_smem(K kern) {
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_SM_BYTES);
}

}  // namespace

// ------------------------------------------------------------------ host side
void mlp_image(const float* w, std::vector<unsigned char>& img) {
  img.assign(MLP_IMG_BYTES, 0);
  auto put = [&](int base, int r, int k, int K, float v) {
    __nv_bfloat16 b = __float2bfloat16_rn(v);
    std::memcpy(&img[base + core_off(r, k, K)], &b, 2);
  };
  for (int n = 0; n < 128; ++n) {                       // layer 0: K 16, the bias as column 7
    for (int k = 0; k < MLP_IN; ++k) put(mlp_img_w(0), n, k, MLP_K0, w[mlp_woff(0) + n * MLP_IN + k]);
    put(mlp_img_w(0), n, MLP_IN, MLP_K0, w[mlp_boff(0) + n]);
  }
  for (int l = 1; l < MLP_NL; ++l) {
    const int O = mlp_out(l);
    for (int n = 0; n < O; ++n)
      for (int k = 0; k < MLP_H; ++k) put(mlp_img_w(l), n, k, MLP_H, w[mlp_woff(l) + n * MLP_H + k]);
  }
  float* bias = (float*)&img[MLP_IMG_BIAS];
  for (int l = 1; l < MLP_NL; ++l)
    for (int n = 0; n < mlp_out(l); ++n) bias[(l - 1) * 128 + n] = w[mlp_boff(l) + n];
}

void mlp_init(std::vector<float>& w, uint64_t seed) {          // Glorot-uniform weights, zero biases
  w.assign(MLP_NPARAM, 0.f);
  uint64_t h = seed;
  for (int l = 0; l < MLP_NL; ++l) {
    const int I = mlp_in(l), O = mlp_out(l);
    const double a = std::sqrt(6.0 / (I + O));
    for (int e = 0; e < I * O; ++e) { h = mix64(h); w[mlp_woff(l) + e] = (float)(a * (2.0 * ((h >> 11) * (1.0 / 9007199254740992.0)) - 1.0)); }
  }
}

int mlp_make_samples(int closure, const Geo& G, const FamDev& F, int drag, int heat_sel, int blow, long long n,
                     uint64_t seed, double jit, float* X, float* T, cudaStream_t s) {
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (closure == MK) k_mlp_samples<MK><<<grid, 256, 0, s>>>(G, F, drag, heat_sel, blow, n, seed, jit, X, T);
  else if (closure == IG) k_mlp_samples<IG><<<grid, 256, 0, s>>>(G, F, drag, heat_sel, blow, n, seed, jit, X, T);
  else k_mlp_samples<AG><<<grid, 256, 0, s>>>(G, F, drag, heat_sel, blow, n, seed, jit, X, T);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Trains the network on device samples (raw X, scaled T; the last val_frac of them held out):
// standardisation and envelope from the samples, Adam with a cosine learning-rate decay, and the
// held-out errors of the two scaled rates.
int mlp_train(const float* X, const float* T, long long n, const MlpTrainOpts& o, std::vector<float>& w, MlpNorm& nm,
              MlpTrainReport& rep, cudaStream_t s, std::string& err) {
  auto t0 = std::chrono::steady_clock::now();
  std::vector<float> hx((size_t)n * MLP_IN), ht((size_t)n * 2);
  if (cudaMemcpyAsync(hx.data(), X, hx.size() * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(ht.data(), T, ht.size() * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) { err = "surrogate: copying the samples"; return 1; }
  const long long nval = std::max(1LL, (long long)(o.val_frac * (double)n)), ntr = n - nval;
  if (ntr < 64) { err = "surrogate: too few samples"; return 1; }
  for (int a = 0; a < MLP_IN; ++a) {
    double sm = 0, sq = 0; float lo = 1e30f, hi = -1e30f;
    for (long long e = 0; e < ntr; ++e) { double v = hx[e * MLP_IN + a]; sm += v; sq += v * v; lo = std::min(lo, (float)v); hi = std::max(hi, (float)v); }
    const double mean = sm / ntr, var = std::max(sq / ntr - mean * mean, 0.0);
    nm.in_mean[a] = (float)mean;
    nm.in_std[a] = var > 1e-30 * (1.0 + mean * mean) ? (float)std::sqrt(var) : 1.f;
    // the envelope, widened by 1e-3 of its size (a constant input, such as a uniform pressure, is then
    // not missed by the last bit of its single-precision evaluation in a cell)
    const float margin = 1e-3f * std::max(hi - lo, std::max(std::fabs(lo), std::fabs(hi)));
    nm.env_lo[a] = lo - margin; nm.env_hi[a] = hi + margin;
  }
  for (int a = 0; a < 2; ++a) {
    double sm = 0, sq = 0;
    for (long long e = 0; e < ntr; ++e) { double v = ht[e * 2 + a]; sm += v; sq += v * v; }
    const double mean = sm / ntr, var = std::max(sq / ntr - mean * mean, 0.0);
    nm.out_mean[a] = (float)mean;
    nm.out_std[a] = var > 0 ? (float)std::sqrt(var) : 1.f;
  }
  Net N;
  if (N.alloc(o.batch) != cudaSuccess) { err = "surrogate: allocating the training buffers"; return 1; }
  mlp_init(w, o.seed);
  cudaMemcpyAsync(N.w, w.data(), MLP_NPARAM * 4, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(N.m, 0, MLP_NPARAM * 4, s);
  cudaMemsetAsync(N.v, 0, MLP_NPARAM * 4, s);
  const long long steps = std::max(1LL, (long long)o.epochs * ntr / o.batch);
  const long long tail = std::min<long long>(20, steps);          // the reported loss: the last 20 batches
  const float b1 = 0.9f, b2 = 0.999f;
  double last_loss = 0.0;
  cudaMemsetAsync(N.loss, 0, sizeof(double), s);
  for (long long it = 0; it < steps; ++it) {
    k_gather<<<(o.batch + 255) / 256, 256, 0, s>>>(X, T, ntr, nm, mix64(o.seed + 7 + it), N.x, N.t, o.batch);
    forward(N, o.batch, s);
    if (it == steps - tail) cudaMemsetAsync(N.loss, 0, sizeof(double), s);
    backward(N, o.batch, s);
    const double frac = (double)it / (double)steps;
    const float lr = (float)(o.lr * (0.01 + 0.99 * 0.5 * (1.0 + std::cos(3.141592653589793 * frac))));
    const float c1 = 1.f - std::pow(b1, (float)(it + 1)), c2 = 1.f - std::pow(b2, (float)(it + 1));
    k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(N.w, N.g, N.m, N.v, MLP_NPARAM, lr, b1, b2, c1, c2);
  }
  double l20 = 0;
  cudaMemcpyAsync(&l20, N.loss, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(w.data(), N.w, MLP_NPARAM * 4, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { err = "surrogate: training"; return 1; }
  last_loss = l20 / (double)tail;
  // held-out samples through the trained FP32 network
  std::vector<float> pred((size_t)nval * 2);
  std::vector<float> xs((size_t)o.batch * MLP_IN);
  for (long long b0 = 0; b0 < nval; b0 += o.batch) {
    const int rows = (int)std::min<long long>(o.batch, nval - b0);
    for (int r = 0; r < rows; ++r)
      for (int a = 0; a < MLP_IN; ++a) xs[r * MLP_IN + a] = (hx[(ntr + b0 + r) * MLP_IN + a] - nm.in_mean[a]) / nm.in_std[a];
    cudaMemcpyAsync(N.x, xs.data(), (size_t)rows * MLP_IN * 4, cudaMemcpyHostToDevice, s);
    forward(N, rows, s);
    cudaMemcpyAsync(&pred[b0 * 2], N.a[MLP_NL - 1], (size_t)rows * 2 * 4, cudaMemcpyDeviceToHost, s);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) { err = "surrogate: validation"; return 1; }
  std::vector<double> em, eq;
  double vl = 0;
  for (long long e = 0; e < nval; ++e) {
    for (int a = 0; a < 2; ++a) {
      const double p = pred[e * 2 + a] * nm.out_std[a] + nm.out_mean[a], t = ht[(ntr + e) * 2 + a];
      const double z = (p - t) / nm.out_std[a];
      vl += z * z;
      // relative error of the rate (the target is the rate over its reference)
      const double rel = std::fabs(p - t) / std::max(std::fabs(t), 1e-3);
      (a == 0 ? em : eq).push_back(rel);
    }
  }
  auto q = [](std::vector<double>& v, double f) { std::sort(v.begin(), v.end()); return v[(size_t)(f * (v.size() - 1))]; };
  rep.train_loss = last_loss;
  rep.val_loss = vl / (2.0 * nval);
  rep.mdot_rel_median = q(em, 0.5); rep.mdot_rel_p99 = q(em, 0.99);
  rep.q_rel_median = q(eq, 0.5); rep.q_rel_p99 = q(eq, 0.99);
  rep.nsamples = n;
  rep.steps = steps;
  rep.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

void launch_source_mlp(int closure, const LaunchArgs& a, const unsigned char* img, const MlpNorm& nm) {
  const int grid = grid_mlp();
  if (closure == MK) { allow_smem(k_source_mlp<MK>); k_source_mlp<MK><<<grid, MLP_THREADS, MLP_SM_BYTES, a.s>>>(a.G, a.F, img, nm, a.st); }
  else if (closure == IG) { allow_smem(k_source_mlp<IG>); k_source_mlp<IG><<<grid, MLP_THREADS, MLP_SM_BYTES, a.s>>>(a.G, a.F, img, nm, a.st); }
  else { allow_smem(k_source_mlp<AG>); k_source_mlp<AG><<<grid, MLP_THREADS, MLP_SM_BYTES, a.s>>>(a.G, a.F, img, nm, a.st); }
}

// The standalone checks behind ice_gpu_mlp_grad / ice_gpu_mlp_infer (host arrays in and out).
int mlp_grad_host(const float* w, const float* x, const float* t, int n, float* grad, float* loss, std::string& err) {
  Net N;
  if (N.alloc(n) != cudaSuccess) { err = "mlp_grad: allocation"; return 1; }
  cudaStream_t s = 0;
  cudaMemcpy(N.w, w, MLP_NPARAM * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(N.x, x, (size_t)n * MLP_IN * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(N.t, t, (size_t)n * 2 * 4, cudaMemcpyHostToDevice);
  cudaMemset(N.loss, 0, sizeof(double));
  forward(N, n, s);
  backward(N, n, s);
  double l = 0;
  cudaMemcpy(grad, N.g, MLP_NPARAM * 4, cudaMemcpyDeviceToHost);
  cudaError_t e = cudaMemcpy(&l, N.loss, sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) { err = std::string("mlp_grad: ") + cudaGetErrorString(e); return 1; }
  *loss = (float)l;
  return 0;
}

int mlp_infer_host(const float* w, const float* x, int n, float* y, std::string& err) {
  std::vector<unsigned char> img;
  mlp_image(w, img);
  unsigned char* dimg = nullptr; float *dx = nullptr, *dy = nullptr; int* dfail = nullptr;
  cudaError_t e = cudaMalloc((void**)&dimg, img.size());
  if (e == cudaSuccess) e = cudaMalloc((void**)&dx, (size_t)n * MLP_IN * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dy, (size_t)n * 2 * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&dfail, 4);
  if (e == cudaSuccess) e = cudaMemcpy(dimg, img.data(), img.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, (size_t)n * MLP_IN * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dfail, 0, 4);
  int fail = 0;
  if (e == cudaSuccess) {
    allow_smem(k_mlp_infer);
    const int grid = std::min(grid_mlp(), (n + MLP_THREADS - 1) / MLP_THREADS);
    k_mlp_infer<<<grid, MLP_THREADS, MLP_SM_BYTES>>>(dimg, dx, dy, n, dfail);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(y, dy, (size_t)n * 2 * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&fail, dfail, 4, cudaMemcpyDeviceToHost);
  }
  for (void* p : {(void*)dimg, (void*)dx, (void*)dy, (void*)dfail}) if (p) cudaFree(p);
  if (e != cudaSuccess) { err = std::string("mlp_infer: ") + cudaGetErrorString(e); return 1; }
  if (fail) { err = "mlp_infer: a wait for the tensor cores gave up"; return 1; }
  return 0;
}

}  // namespace ice
