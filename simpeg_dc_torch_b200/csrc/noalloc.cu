// Allocation-free solve of one small SPD system (dct_solve_small_noalloc).
//
// Some callers of this library cannot allocate device memory: hosts whose
// framework owns every byte of device memory through its own pool (a second
// allocator would fight it for memory), and latency-bound loops that must not
// take the device-wide synchronisation a cudaMalloc/cudaFree may cause.  For
// them this entry point factors and solves a small system without any
// allocation: the caller passes the CSR pattern and values, the right-hand
// sides and the output, and the only scratch (the dense factor) lives in the
// file-scope array below.  It holds kNoAllocMaxN^2 doubles (2 MiB) on every
// GPU that loads the library, until the process exits.
//
// In host code `g_noalloc_factor` is a host-side stand-in, not a device
// address; its device address is obtained once per device with
// cudaGetSymbolAddress (with that device current) on the first call made on
// that device, and cached.  All calls share the one array and it keeps the
// contents of the last call: each call clears the part it uses before writing
// it, and two calls whose work overlaps on the GPU (different streams, no
// ordering) race on it and must not be issued.
//
// The call returns without waiting for the GPU, so it cannot return a status
// for a matrix that is not positive definite: a non-positive or NaN pivot
// instead makes every entry of x NaN.  The CSR pattern must be canonical
// (column indices in [0, n), no duplicates: a duplicate entry overwrites the
// other instead of adding to it); entries with an out-of-range column, and
// rows whose row pointers decrease, are skipped.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "dct_internal.h"

namespace {

constexpr int kNoAllocMaxN = 512;    // largest system order
constexpr int kNoAllocMaxRhs = 64;   // most right-hand sides per call
constexpr int kNaPanel = 16;         // panel width of the factorization
constexpr int kNaThreads = 1024;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_factor[kNoAllocMaxN * kNoAllocMaxN];

std::mutex g_na_mu;
double* g_na_addr[kMaxDevices] = {nullptr};

__global__ void k_na_clear(double* __restrict__ S, int64_t count) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x)
    S[i] = 0.0;
}

// lower triangle of the CSR matrix into the dense column-major factor;
// entries whose column lies outside [0, i] are not stored
__global__ void k_na_scatter(int n, const int32_t* __restrict__ crow,
                             const int32_t* __restrict__ col,
                             const double* __restrict__ vals,
                             double* __restrict__ S) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    for (int e = crow[i]; e < crow[i + 1]; ++e) {
      const int j = col[e];
      if (j >= 0 && j <= i) S[i + int64_t(j) * n] = vals[e];
    }
}

// Blocked right-looking Cholesky of the dense n x n lower triangle, one CTA.
// Each 16-column panel is factored in shared memory, written back, and then
// applied to the trailing lower triangle.  A non-positive or NaN pivot
// becomes NaN: it spreads through the rest of the factor and through both
// substitutions (each of which reads every entry below the diagonal), so
// every entry of x comes back NaN.
__global__ void __launch_bounds__(kNaThreads) k_na_potrf(int n, double* __restrict__ S) {
  extern __shared__ double Ps[];   // (n - p0) x w panel, ld = n
  const int tid = threadIdx.x;
  for (int p0 = 0; p0 < n; p0 += kNaPanel) {
    const int w = min(kNaPanel, n - p0);
    const int m = n - p0;
    for (int idx = tid; idx < m * w; idx += blockDim.x) {
      const int r = idx % m, c = idx / m;
      Ps[r + c * m] = S[(p0 + r) + int64_t(p0 + c) * n];
    }
    __syncthreads();
    for (int c = 0; c < w; ++c) {
      double piv = Ps[c + c * m];
      if (!(piv > 0.0)) piv = __longlong_as_double(0x7ff8000000000000ll);   // NaN
      const double d = sqrt(piv);
      __syncthreads();
      if (tid == 0) Ps[c + c * m] = d;
      for (int r = c + 1 + tid; r < m; r += blockDim.x) Ps[r + c * m] /= d;
      __syncthreads();
      for (int idx = tid; idx < (m - c - 1) * (w - c - 1); idx += blockDim.x) {
        const int r = c + 1 + idx % (m - c - 1);
        const int cc = c + 1 + idx / (m - c - 1);
        if (r >= cc) Ps[r + cc * m] -= Ps[r + c * m] * Ps[cc + c * m];
      }
      __syncthreads();
    }
    for (int idx = tid; idx < m * w; idx += blockDim.x) {
      const int r = idx % m, c = idx / m;
      if (r >= c) S[(p0 + r) + int64_t(p0 + c) * n] = Ps[r + c * m];
    }
    const int t = m - w;   // trailing order
    for (int idx = tid; idx < t * t; idx += blockDim.x) {
      const int i = idx % t, j = idx / t;
      if (i < j) continue;
      double acc = 0.0;
      for (int c = 0; c < w; ++c) acc += Ps[(w + i) + c * m] * Ps[(w + j) + c * m];
      S[(p0 + w + i) + int64_t(p0 + w + j) * n] -= acc;
    }
    __syncthreads();
  }
}

// Forward and backward substitution of one right-hand side per CTA.
__global__ void __launch_bounds__(kNaThreads)
k_na_trsv(int n, int k, const double* __restrict__ S, const double* __restrict__ b,
          double* __restrict__ x) {
  __shared__ double y[kNoAllocMaxN];
  const int j = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = b[int64_t(i) * k + j];
  __syncthreads();
  for (int c = 0; c < n; ++c) {
    const double v = y[c] / S[c + int64_t(c) * n];
    __syncthreads();
    if (threadIdx.x == 0) y[c] = v;
    for (int i = c + 1 + threadIdx.x; i < n; i += blockDim.x)
      y[i] -= S[i + int64_t(c) * n] * v;
    __syncthreads();
  }
  for (int c = n - 1; c >= 0; --c) {
    // y[c] -= sum_{i > c} L[i, c] x[i]: one warp-reduced dot product
    double part = 0.0;
    for (int i = c + 1 + threadIdx.x; i < n; i += blockDim.x)
      part += S[i + int64_t(c) * n] * y[i];
    __shared__ double red[kNaThreads / 32];
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int q = 0; q < blockDim.x / 32; ++q) s += red[q];
      y[c] = (y[c] - s) / S[c + int64_t(c) * n];
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[int64_t(i) * k + j] = y[i];
}

int na_fail(int code, const std::string& msg) {
  dct::set_last_error(msg.c_str());
  return code;
}

}  // namespace

extern "C" int dct_solve_small_noalloc(int32_t n, const int32_t* d_crow,
                                       const int32_t* d_col, const double* d_vals,
                                       const double* d_b, int32_t k, double* d_x,
                                       void* stream) {
  if (n < 1 || n > kNoAllocMaxN)
    return na_fail(DCT_ERR_ARG, "dct_solve_small_noalloc: n must be 1.." +
                                    std::to_string(kNoAllocMaxN));
  if (k < 1 || k > kNoAllocMaxRhs)
    return na_fail(DCT_ERR_ARG, "dct_solve_small_noalloc: k must be 1.." +
                                    std::to_string(kNoAllocMaxRhs));
  if (!d_crow || !d_col || !d_vals || !d_b || !d_x)
    return na_fail(DCT_ERR_ARG, "dct_solve_small_noalloc: null pointer");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return na_fail(DCT_ERR_CUDA, "dct_solve_small_noalloc: no current device");
  double* S = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (g_na_addr[dev] == nullptr) {
      // set-up, once per device, with that device current
      e = cudaGetSymbolAddress(reinterpret_cast<void**>(&S), g_noalloc_factor);
      if (e != cudaSuccess)
        return na_fail(DCT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
                                         cudaGetErrorString(e));
      g_na_addr[dev] = S;
    }
    S = g_na_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t count = int64_t(n) * n;
  k_na_clear<<<(count + 255) / 256, 256, 0, st>>>(S, count);
  k_na_scatter<<<(n + 255) / 256, 256, 0, st>>>(n, d_crow, d_col, d_vals, S);
  const size_t smem = sizeof(double) * size_t(n) * kNaPanel;
  e = cudaFuncSetAttribute(k_na_potrf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem));
  if (e != cudaSuccess)
    return na_fail(DCT_ERR_CUDA, std::string("cudaFuncSetAttribute: ") +
                                     cudaGetErrorString(e));
  k_na_potrf<<<1, kNaThreads, smem, st>>>(n, S);
  k_na_trsv<<<k, kNaThreads, 0, st>>>(n, k, S, d_b, d_x);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return na_fail(DCT_ERR_CUDA, std::string("dct_solve_small_noalloc: ") +
                                     cudaGetErrorString(e));
  return DCT_OK;
}
