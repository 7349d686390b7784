// Fused DC engine kernels around the solver: conductivity -> matrix values,
// right-hand-side scatter, quadrature sum + receiver projection, value-gradient
// contraction and its transpose through the assembly map.  All float64.
#include <cuda_runtime.h>

#include "dct_internal.h"

namespace dct {
namespace {

constexpr int kT = 256;

inline unsigned blocks_for(int64_t work, int64_t per_block) {
  int64_t b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return static_cast<unsigned>(b);
}

__global__ void k_sigma(int64_t nC, const double* __restrict__ m,
                        double* __restrict__ sigma) {
  for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < nC;
       c += int64_t(gridDim.x) * blockDim.x)
    sigma[c] = exp(-m[c]);
}

// one thread per row: rows of the assembly map hold 1..12 entries
__global__ void k_csr_rows(int64_t nrows, const int64_t* __restrict__ ptr,
                           const int32_t* __restrict__ col,
                           const double* __restrict__ val,
                           const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < nrows;
       r += int64_t(gridDim.x) * blockDim.x) {
    double acc = 0.0;
    for (int64_t q = ptr[r]; q < ptr[r + 1]; ++q) acc += val[q] * __ldg(&x[col[q]]);
    y[r] = acc;
  }
}

// one warp per cell: rows of L^T hold tens to hundreds of entries
__global__ void k_values_vjp(int64_t nC, const int64_t* __restrict__ ptr,
                             const int32_t* __restrict__ col,
                             const double* __restrict__ val,
                             const double* __restrict__ sigma,
                             const double* __restrict__ gv, double* __restrict__ gm) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; c < nC;
       c += warps) {
    double acc = 0.0;
    for (int64_t q = ptr[c] + lane; q < ptr[c + 1]; q += 32)
      acc += val[q] * __ldg(&gv[col[q]]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) gm[c] = -sigma[c] * acc;
  }
}

__global__ void k_scatter_pairs(int64_t npairs, int k, const int64_t* __restrict__ ptr,
                                const int32_t* __restrict__ row,
                                const int32_t* __restrict__ src,
                                const int32_t* __restrict__ datum,
                                const double* __restrict__ coef,
                                const double* __restrict__ g, double* __restrict__ dst) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npairs;
       p += int64_t(gridDim.x) * blockDim.x) {
    double acc = 0.0;
    for (int64_t q = ptr[p]; q < ptr[p + 1]; ++q)
      acc += coef[q] * (g != nullptr ? g[datum[q]] : 1.0);
    dst[int64_t(row[p]) * k + src[p]] = acc;
  }
}

__global__ void k_project(int nbatch, int64_t n, int k, int64_t nD,
                          const int32_t* __restrict__ pptr,
                          const int32_t* __restrict__ pcol,
                          const double* __restrict__ pval,
                          const int32_t* __restrict__ sidx,
                          const int32_t* __restrict__ iperm,
                          const double* __restrict__ w,
                          const double* __restrict__ X, double* __restrict__ d) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nD;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int s = sidx[i];
    double acc = 0.0;
    for (int b = 0; b < nbatch; ++b) {
      const double* Xb = X + int64_t(b) * n * k;
      double part = 0.0;
      for (int q = pptr[i]; q < pptr[i + 1]; ++q)
        part += pval[q] * Xb[int64_t(iperm[pcol[q]]) * k + s];
      acc += (w != nullptr ? w[b] : 1.0) * part;
    }
    d[i] = acc;
  }
}

// one warp per (entry, system); lanes stride over the right-hand sides
template <typename T, bool kPermuted>
__global__ void k_gather_contract(int nbatch, int64_t n, int64_t nnz, int k,
                                  const int32_t* __restrict__ row,
                                  const int32_t* __restrict__ col,
                                  const int32_t* __restrict__ iperm,
                                  const double* __restrict__ scale,
                                  const T* __restrict__ Y, const T* __restrict__ X,
                                  T* __restrict__ gv) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int64_t total = nnz * nbatch;
  for (int64_t t = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; t < total;
       t += warps) {
    const int b = static_cast<int>(t / nnz);
    const int64_t e = t - int64_t(b) * nnz;
    int64_t r = row[e], c = col[e];
    if (kPermuted) {
      r = iperm[r];
      c = iperm[c];
    }
    const T* y = Y + (int64_t(b) * n + r) * k;
    const T* x = X + (int64_t(b) * n + c) * k;
    double acc = 0.0;
    for (int j = lane; j < k; j += 32) acc += double(y[j]) * double(x[j]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) gv[t] = T(-(scale != nullptr ? scale[b] : 1.0) * acc);
  }
}

// The same contraction (permuted Y and X, k <= 32 R) with one warp per run
// of kGcRun consecutive entries: the row of Y stays in registers while
// consecutive entries share it, as they do in CSR order (about 27 entries
// per row on a 3-D grid), so Y is read about once per row instead of once per
// entry.  Any entry order gives the same result.
#ifndef DCT_GC_ROWS
#define DCT_GC_ROWS 1
#endif
constexpr int kGcRun = 32;
template <int R>
__global__ void k_gather_contract_rows(int nbatch, int64_t n, int64_t nnz, int k,
                                       const int32_t* __restrict__ row,
                                       const int32_t* __restrict__ col,
                                       const int32_t* __restrict__ iperm,
                                       const double* __restrict__ scale,
                                       const double* __restrict__ Y,
                                       const double* __restrict__ X, double* __restrict__ gv) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int64_t runs = (nnz + kGcRun - 1) / kGcRun;
  const int64_t total = runs * nbatch;
  for (int64_t t = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; t < total;
       t += warps) {
    const int b = static_cast<int>(t / runs);
    const int64_t e0 = (t - int64_t(b) * runs) * kGcRun;
    const int64_t e1 = e0 + kGcRun < nnz ? e0 + kGcRun : nnz;
    const double sc = -(scale != nullptr ? scale[b] : 1.0);
    int64_t cur = -1;
    double y[R];
    for (int64_t e = e0; e < e1; ++e) {
      const int64_t r = iperm[row[e]];
      if (r != cur) {
        cur = r;
        const double* yr = Y + (int64_t(b) * n + r) * k;
#pragma unroll
        for (int q = 0; q < R; ++q) y[q] = lane + 32 * q < k ? yr[lane + 32 * q] : 0.0;
      }
      const double* x = X + (int64_t(b) * n + iperm[col[e]]) * k;
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < R; ++q)
        if (lane + 32 * q < k) acc += y[q] * x[lane + 32 * q];
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) gv[int64_t(b) * nnz + e] = sc * acc;
    }
  }
}

// complex128: gv[b, e] = -sum_r Y[b, row_e, r] X[b, col_e, r] (no
// conjugation: the caller conjugates where its convention asks)
__global__ void k_gather_contract_c(int nbatch, int64_t n, int64_t nnz, int k,
                                    const int32_t* __restrict__ row,
                                    const int32_t* __restrict__ col,
                                    const cplx* __restrict__ Y, const cplx* __restrict__ X,
                                    cplx* __restrict__ gv) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int64_t total = nnz * nbatch;
  for (int64_t t = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; t < total;
       t += warps) {
    const int b = static_cast<int>(t / nnz);
    const int64_t e = t - int64_t(b) * nnz;
    const cplx* y = Y + (int64_t(b) * n + row[e]) * k;
    const cplx* x = X + (int64_t(b) * n + col[e]) * k;
    cplx acc;
    for (int j = lane; j < k; j += 32) acc += y[j] * x[j];
    for (int o = 16; o > 0; o >>= 1) {
      acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
      acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
    }
    if (lane == 0) gv[t] = -acc;
  }
}

int report(cudaError_t e) {
  if (e == cudaSuccess) return DCT_OK;
  set_last_error(cudaGetErrorString(e));
  return DCT_ERR_CUDA;
}

}  // namespace
}  // namespace dct

using namespace dct;

extern "C" {

int dct_sigma_values(int64_t nrows, const int64_t* d_L_ptr, const int32_t* d_L_col,
                     const double* d_L_val, int64_t nC, const double* d_m,
                     double* d_sigma, double* d_vals, void* stream) {
  if (nrows < 0 || nC < 1 || !d_L_ptr || !d_m || !d_sigma || !d_vals)
    return DCT_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_sigma<<<blocks_for(nC, kT), kT, 0, st>>>(nC, d_m, d_sigma);
  if (nrows > 0)
    k_csr_rows<<<blocks_for(nrows, kT), kT, 0, st>>>(nrows, d_L_ptr, d_L_col,
                                                     d_L_val, d_sigma, d_vals);
  return report(cudaGetLastError());
}

int dct_values_vjp(int64_t nC, const int64_t* d_Lt_ptr, const int32_t* d_Lt_col,
                   const double* d_Lt_val, const double* d_sigma, const double* d_gv,
                   double* d_gm, void* stream) {
  if (nC < 1 || !d_Lt_ptr || !d_sigma || !d_gv || !d_gm) return DCT_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_values_vjp<<<blocks_for(nC * 32, kT), kT, 0, st>>>(nC, d_Lt_ptr, d_Lt_col,
                                                       d_Lt_val, d_sigma, d_gv, d_gm);
  return report(cudaGetLastError());
}

int dct_scatter_rhs(int64_t n, int32_t k, int64_t npairs, const int64_t* d_ptr,
                    const int32_t* d_row, const int32_t* d_src,
                    const int32_t* d_datum, const double* d_coef, const double* d_g,
                    double* d_dst, void* stream) {
  if (n < 1 || k < 1 || npairs < 0 || !d_dst) return DCT_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(d_dst, 0, sizeof(double) * n * k, st);
  if (e != cudaSuccess) return report(e);
  if (npairs > 0)
    k_scatter_pairs<<<blocks_for(npairs, kT), kT, 0, st>>>(
        npairs, k, d_ptr, d_row, d_src, d_datum, d_coef, d_g, d_dst);
  return report(cudaGetLastError());
}

int dct_project_data(int32_t nbatch, int64_t n, int32_t k, int64_t nD,
                     const int32_t* d_Pd_ptr, const int32_t* d_Pd_col,
                     const double* d_Pd_val, const int32_t* d_sidx,
                     const int32_t* d_iperm, const double* d_w, const double* d_X,
                     double* d_out, void* stream) {
  if (nbatch < 1 || n < 1 || k < 1 || nD < 0 || !d_X || !d_out) return DCT_ERR_ARG;
  if (nD == 0) return DCT_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_project<<<blocks_for(nD, kT), kT, 0, st>>>(nbatch, n, k, nD, d_Pd_ptr, d_Pd_col,
                                               d_Pd_val, d_sidx, d_iperm, d_w, d_X,
                                               d_out);
  return report(cudaGetLastError());
}

int dct_gather_contract(int32_t nbatch, int64_t n, int64_t nnz, int32_t k,
                        const int32_t* d_row, const int32_t* d_col,
                        const int32_t* d_iperm, const double* d_scale,
                        const double* d_Y, const double* d_X, double* d_gv,
                        void* stream) {
  if (nbatch < 1 || n < 1 || nnz < 0 || k < 1 || !d_iperm || !d_Y || !d_X || !d_gv)
    return DCT_ERR_ARG;
  if (nnz == 0) return DCT_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t run_threads = (nnz + kGcRun - 1) / kGcRun * nbatch * 32;
  if (!DCT_GC_ROWS)
    k_gather_contract<double, true><<<blocks_for(nnz * nbatch * 32, kT), kT, 0, st>>>(
        nbatch, n, nnz, k, d_row, d_col, d_iperm, d_scale, d_Y, d_X, d_gv);
  else if (k <= 64)
    k_gather_contract_rows<2><<<blocks_for(run_threads, kT), kT, 0, st>>>(
        nbatch, n, nnz, k, d_row, d_col, d_iperm, d_scale, d_Y, d_X, d_gv);
  else if (k <= 128)
    k_gather_contract_rows<4><<<blocks_for(run_threads, kT), kT, 0, st>>>(
        nbatch, n, nnz, k, d_row, d_col, d_iperm, d_scale, d_Y, d_X, d_gv);
  else if (k <= 256)
    k_gather_contract_rows<8><<<blocks_for(run_threads, kT), kT, 0, st>>>(
        nbatch, n, nnz, k, d_row, d_col, d_iperm, d_scale, d_Y, d_X, d_gv);
  else
    k_gather_contract<double, true><<<blocks_for(nnz * nbatch * 32, kT), kT, 0, st>>>(
        nbatch, n, nnz, k, d_row, d_col, d_iperm, d_scale, d_Y, d_X, d_gv);
  return report(cudaGetLastError());
}

int dct_gather_contract_plain(int32_t nbatch, int64_t n, int64_t nnz, int32_t k,
                              const int32_t* d_row, const int32_t* d_col,
                              int32_t dtype, const void* d_Y, const void* d_X,
                              void* d_gv, void* stream) {
  if (nbatch < 1 || n < 1 || nnz < 0 || k < 1 || !d_Y || !d_X || !d_gv)
    return DCT_ERR_ARG;
  if (nnz == 0) return DCT_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned g = blocks_for(nnz * nbatch * 32, kT);
  if (dtype == DCT_C128)
    k_gather_contract_c<<<g, kT, 0, st>>>(
        nbatch, n, nnz, k, d_row, d_col, static_cast<const cplx*>(d_Y),
        static_cast<const cplx*>(d_X), static_cast<cplx*>(d_gv));
  else if (dtype == DCT_F64)
    k_gather_contract<double, false><<<g, kT, 0, st>>>(
        nbatch, n, nnz, k, d_row, d_col, nullptr, nullptr,
        static_cast<const double*>(d_Y), static_cast<const double*>(d_X),
        static_cast<double*>(d_gv));
  else
    k_gather_contract<float, false><<<g, kT, 0, st>>>(
        nbatch, n, nnz, k, d_row, d_col, nullptr, nullptr,
        static_cast<const float*>(d_Y), static_cast<const float*>(d_X),
        static_cast<float*>(d_gv));
  return report(cudaGetLastError());
}

}  // extern "C"
