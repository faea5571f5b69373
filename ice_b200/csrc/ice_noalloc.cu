// ice_noalloc.cu -- ice_gpu_residual_sq_noalloc: the residual-norm sums of one block of one family,
// computed without allocating anything.
//
// Some drivers cannot let a library allocate device memory: the host application owns every device
// allocation through its own pool (a coupler running inside a gas solver with a fixed memory
// budget, or a Fortran/OpenACC runtime that holds the state arrays). Such a caller already has the
// block's new and old state on the device and wants the residual of the step without creating a
// solve context, whose set-up allocates. This entry point reads those two arrays and writes five
// host doubles; its scratch (one partial sum per chunk of cells) is a file-scope __device__ array
// that every GPU loading the library holds until the process exits.
//
// The arithmetic is the residual norm's (residual_sq, diagnostic/Mod_Diagnostic.f90:106-130), in
// the order of the context's own norm kernel: chunks of kChunk cells, one CTA each, a strided
// per-thread sum and a tree over the CTA, then the chunks summed in order. For the same states the
// two entry points give the same bits.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <mutex>
#include "../../include/ice_gpu.h"

namespace {

constexpr int kChunk = 2048;                 // cells per CTA (the context's norm chunk)
constexpr int kThreads = 256;
constexpr int kMaxChunks = 4096;             // => at most 8,388,608 cells per call
constexpr int kMaxDevices = 64;

// the partial sums of every chunk, then the five totals
__device__ __align__(256) double g_noalloc_scratch[(kMaxChunks + 1) * 5];

// per CUDA context: the address of g_noalloc_scratch in that context's copy of the module (the
// host-side symbol is only a stand-in and must not be given to a kernel). The key is the current
// context, not the device ordinal: a caller whose runtime made its own context (cuCtxCreate) holds the
// module, and so the array, at another address than the device's primary context.
struct ScratchOf {
  void* ctx;
  double* addr;
};
ScratchOf g_scratch_of[kMaxDevices] = {};
int g_nscratch = 0;
std::mutex g_scratch_mu;

// cuCtxGetCurrent through the runtime's driver entry point (the library links no libcuda)
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static bool looked = false;
  if (!looked) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (CtxGetCurrentFn)f;
    looked = true;
  }
  return fn;
}

__global__ void k_residual_sq_chunks(const double* __restrict__ pn, const double* __restrict__ po, int nc, int it,
                                     int ni, int nj, long long ncell, double* __restrict__ part) {
  const long long q0 = (long long)blockIdx.x * kChunk;
  const long long q1 = q0 + kChunk < ncell ? q0 + kChunk : ncell;
  double acc[5] = {0, 0, 0, 0, 0};
  for (long long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    const int i = (int)(q % ni);
    const long long r = q / ni;
    const int j = (int)(r % nj);
    const long long k = r / nj;
    const long long g = (long long)nc * (((k + 2) * (nj + 4) + (j + 2)) * (long long)(ni + 4) + (i + 2));
    const int vs[5] = {0, 1, 2, 3, it};
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const double d = fabs(pn[g + vs[m]] - po[g + vs[m]]);
      acc[m] = acc[m] + d*d;
    }
  }
  __shared__ double red[5][kThreads];
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

// the chunks in order, as the host sums the context's partials
__global__ void k_residual_sq_total(const double* __restrict__ part, int nchunk, double* __restrict__ total) {
  if (threadIdx.x >= 5) return;
  const int m = threadIdx.x;
  double a = 0.0;
  for (int q = 0; q < nchunk; ++q) a = a + part[(long long)q * 5 + m];
  total[m] = a;
}

int fail(char* err, int errlen, int code, const char* msg, const char* detail = "") {
  if (err && errlen > 0) snprintf(err, errlen, "%s%s", msg, detail);
  return code;
}

}  // namespace

extern "C" int ice_gpu_residual_sq_noalloc(const double* prim_new, const double* prim_old, int32_t nc, int32_t t_slot,
                                           const int32_t* dims, double* sums, void* stream, char* err,
                                           int32_t errlen) {
  if (!prim_new || !prim_old || !dims || !sums) return fail(err, errlen, ICE_GPU_EINVAL, "residual_sq_noalloc: null argument");
  const int ni = dims[0], nj = dims[1], nk = dims[2];
  if (ni < 1 || nj < 1 || nk < 1) return fail(err, errlen, ICE_GPU_EINVAL, "residual_sq_noalloc: dims must be >= 1");
  if (nc < 5 || nc > 12 || t_slot < 5 || t_slot > nc)
    return fail(err, errlen, ICE_GPU_EINVAL, "residual_sq_noalloc: nc must be 5..12 and the temperature slot 5..nc");
  const long long ncell = (long long)ni * nj * nk;
  const long long nchunk = (ncell + kChunk - 1) / kChunk;
  if (nchunk > kMaxChunks) {
    char d[96];
    snprintf(d, sizeof d, " (%lld cells given; the limit is %d)", ncell, kMaxChunks * kChunk);
    return fail(err, errlen, ICE_GPU_EINVAL, "residual_sq_noalloc: the block has more cells than the static scratch holds", d);
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(err, errlen, ICE_GPU_ECUDA, "residual_sq_noalloc: cudaGetDevice: ", cudaGetErrorString(e));
  CtxGetCurrentFn cur = ctx_get_current();
  void* ctx = nullptr;
  if (!cur || cur(&ctx) != 0)
    return fail(err, errlen, ICE_GPU_ECUDA, "residual_sq_noalloc: cuCtxGetCurrent is not available from the driver");
  if (!ctx) {
    // no context is current yet on this thread: the runtime's first call on the device makes the
    // device's primary context current
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(err, errlen, ICE_GPU_ECUDA, "residual_sq_noalloc: cudaGetSymbolAddress: ", cudaGetErrorString(e));
    if (cur(&ctx) != 0 || !ctx) return fail(err, errlen, ICE_GPU_ECUDA, "residual_sq_noalloc: no current CUDA context");
  }
  double* scratch = nullptr;
  {
    // set-up, once per context, with its device current (the first call in a context does it)
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    for (int q = 0; q < g_nscratch; ++q)
      if (g_scratch_of[q].ctx == ctx) scratch = g_scratch_of[q].addr;
    if (!scratch) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return fail(err, errlen, ICE_GPU_ECUDA, "residual_sq_noalloc: cudaGetSymbolAddress: ", cudaGetErrorString(e));
      scratch = (double*)p;
      if (g_nscratch < kMaxDevices) g_scratch_of[g_nscratch++] = {ctx, scratch};
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  double* total = scratch + (size_t)kMaxChunks * 5;
  k_residual_sq_chunks<<<(unsigned)nchunk, kThreads, 0, s>>>(prim_new, prim_old, nc, t_slot - 1, ni, nj, ncell, scratch);
  k_residual_sq_total<<<1, 32, 0, s>>>(scratch, (int)nchunk, total);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(err, errlen, ICE_GPU_ECUDA, "residual_sq_noalloc: launch: ", cudaGetErrorString(e));
  e = cudaMemcpyAsync(sums, total, 5 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(err, errlen, ICE_GPU_ECUDA, "residual_sq_noalloc: ", cudaGetErrorString(e));
  return 0;
}
