// Kernels of the linearised products of the 2.5-D engine (Jacobian-vector
// products, the explicit Jacobian, diag(J^T D J)): they reuse the factors,
// the permuted fields and the assembly map of the evaluation path.
// All float64.
#include <cuda_runtime.h>

#include "dct_internal.h"

namespace dct {
namespace {

constexpr int kT = 256;

inline unsigned grid_for(int64_t work, int64_t per_block) {
  int64_t b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return static_cast<unsigned>(b);
}

// y = M x for a CSR matrix (int64 row pointers), one thread per row
__global__ void k_spmv(int64_t nrows, const int64_t* __restrict__ ptr,
                       const int32_t* __restrict__ col, const double* __restrict__ val,
                       const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < nrows;
       r += int64_t(gridDim.x) * blockDim.x) {
    double acc = 0.0;
    for (int64_t q = ptr[r]; q < ptr[r + 1]; ++q) acc += val[q] * __ldg(&x[col[q]]);
    y[r] = acc;
  }
}

// Y_b[iperm i, :] = alpha * sum_e vals_b[e] X_b[iperm col_e, :] over the
// entries e of row i of the pattern (user order); X, Y permuted (n, k).
// One warp per (system, row), lanes over the right-hand sides.
__global__ void k_pattern_spmm(int nbatch, int n, int k, const int32_t* __restrict__ crow,
                               const int32_t* __restrict__ col,
                               const int32_t* __restrict__ iperm,
                               const double* __restrict__ vals, int64_t nnz, double alpha,
                               const double* __restrict__ X, double* __restrict__ Y) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int64_t total = int64_t(nbatch) * n;
  for (int64_t t = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; t < total;
       t += warps) {
    const int b = static_cast<int>(t / n);
    const int i = static_cast<int>(t - int64_t(b) * n);
    const double* Xb = X + int64_t(b) * n * k;
    const double* vb = vals + int64_t(b) * nnz;
    double* y = Y + (int64_t(b) * n + iperm[i]) * k;
    const int e0 = crow[i], e1 = crow[i + 1];
    for (int j = lane; j < k; j += 32) {
      double acc = 0.0;
      for (int e = e0; e < e1; ++e) acc += vb[e] * Xb[int64_t(iperm[col[e]]) * k + j];
      y[j] = alpha * acc;
    }
  }
}

// gv[(b nnz + e) nb + r] = -scale_b Y_b[iperm row_e, r] U_b[iperm col_e, sidx_r]
// (one adjoint column r per datum, contracted with that datum's own source)
__global__ void k_gather_pairwise(int nbatch, int64_t n, int64_t nnz, int nb, int ns,
                                  const int32_t* __restrict__ row,
                                  const int32_t* __restrict__ col,
                                  const int32_t* __restrict__ iperm,
                                  const double* __restrict__ scale,
                                  const int32_t* __restrict__ sidx,
                                  const double* __restrict__ Y,
                                  const double* __restrict__ U, double* __restrict__ gv) {
  const int64_t total = int64_t(nbatch) * nnz * nb;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
       t += int64_t(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(t % nb);
    const int64_t be = t / nb;
    const int b = static_cast<int>(be / nnz);
    const int64_t e = be - int64_t(b) * nnz;
    const double y = Y[(int64_t(b) * n + iperm[row[e]]) * nb + r];
    const double u = U[(int64_t(b) * n + iperm[col[e]]) * ns + sidx[r]];
    gv[t] = -(scale != nullptr ? scale[b] : 1.0) * y * u;
  }
}

// out[c, r] = -sigma_c sum_q Lt_val[q] gv[Lt_col[q], r]: one warp per cell,
// lanes over the columns r
__global__ void k_values_vjp_multi(int64_t nC, int nb, const int64_t* __restrict__ ptr,
                                   const int32_t* __restrict__ col,
                                   const double* __restrict__ val,
                                   const double* __restrict__ sigma,
                                   const double* __restrict__ gv, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; c < nC;
       c += warps) {
    for (int r = lane; r < nb; r += 32) {
      double acc = 0.0;
      for (int64_t q = ptr[c]; q < ptr[c + 1]; ++q)
        acc += val[q] * gv[int64_t(col[q]) * nb + r];
      out[c * nb + r] = -sigma[c] * acc;
    }
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

int dct_csr_spmv(int64_t nrows, const int64_t* d_ptr, const int32_t* d_col,
                 const double* d_val, const double* d_x, double* d_y, void* stream) {
  if (nrows < 0 || !d_ptr || !d_x || !d_y) return DCT_ERR_ARG;
  if (nrows == 0) return DCT_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_spmv<<<grid_for(nrows, kT), kT, 0, st>>>(nrows, d_ptr, d_col, d_val, d_x, d_y);
  return report(cudaGetLastError());
}

int dct_pattern_spmm(int32_t nbatch, int32_t n, int32_t k, const int32_t* d_crow,
                     const int32_t* d_col, const int32_t* d_iperm, const double* d_vals,
                     int64_t nnz, double alpha, const double* d_X, double* d_Y,
                     void* stream) {
  if (nbatch < 1 || n < 1 || k < 1 || nnz < 0 || !d_crow || !d_col || !d_iperm ||
      !d_vals || !d_X || !d_Y || d_X == d_Y)
    return DCT_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_pattern_spmm<<<grid_for(int64_t(nbatch) * n * 32, kT), kT, 0, st>>>(
      nbatch, n, k, d_crow, d_col, d_iperm, d_vals, nnz, alpha, d_X, d_Y);
  return report(cudaGetLastError());
}

int dct_gather_pairwise(int32_t nbatch, int64_t n, int64_t nnz, int32_t nb, int32_t ns,
                        const int32_t* d_row, const int32_t* d_col,
                        const int32_t* d_iperm, const double* d_scale,
                        const int32_t* d_sidx, const double* d_Y, const double* d_U,
                        double* d_gv, void* stream) {
  if (nbatch < 1 || n < 1 || nnz < 0 || nb < 1 || ns < 1 || !d_row || !d_col ||
      !d_iperm || !d_sidx || !d_Y || !d_U || !d_gv)
    return DCT_ERR_ARG;
  if (nnz == 0) return DCT_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_gather_pairwise<<<grid_for(int64_t(nbatch) * nnz * nb, kT), kT, 0, st>>>(
      nbatch, n, nnz, nb, ns, d_row, d_col, d_iperm, d_scale, d_sidx, d_Y, d_U, d_gv);
  return report(cudaGetLastError());
}

int dct_values_vjp_multi(int64_t nC, int32_t nb, const int64_t* d_Lt_ptr,
                         const int32_t* d_Lt_col, const double* d_Lt_val,
                         const double* d_sigma, const double* d_gv, double* d_out,
                         void* stream) {
  if (nC < 1 || nb < 1 || !d_Lt_ptr || !d_sigma || !d_gv || !d_out) return DCT_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_values_vjp_multi<<<grid_for(nC * 32, kT), kT, 0, st>>>(nC, nb, d_Lt_ptr, d_Lt_col,
                                                           d_Lt_val, d_sigma, d_gv, d_out);
  return report(cudaGetLastError());
}

}  // extern "C"
