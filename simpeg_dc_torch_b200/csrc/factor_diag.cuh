// Dense 64 x 64 diagonal-block Cholesky and inverse of the large-front
// panels, shared by the float64 update kernel (factor.cu) and the float32
// tensor-core update (update_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include "dct_internal.h"

namespace dct {
namespace {

__device__ __forceinline__ void flag_pivot(int* status, int s, int b) {
  if (atomicCAS(&status[0], 0, DCT_ERR_ZERO_PIVOT) == 0) {
    status[1] = s;
    status[2] = b;
  }
}

template <typename T>
__device__ __forceinline__ bool good_pivot(T v) {
  return v > T(0) && v < T(INFINITY);
}

// Blocked Cholesky D = L L^T of a 64 x 64 diagonal block and X = L^{-1}, in
// shared memory (ld kDLD, padded so that row and column walks are both free
// of bank conflicts), over four 16-column block steps kb:
//   (a) one warp factors D_kk (16 x 16) in registers with shuffles and forms
//       its inverse X_kk (forward substitution, one column per lane);
//   (b) all threads: L_rk = D_rk X_kk^T for the rows below, and block row kb
//       of X, X_kj = X_kk R_kj (j < kb), R being the right-hand side of the
//       elimination on [L | I] kept in X's storage;
//   (c) all threads: D_rc -= L_rk L_ck^T (trailing lower triangle) and
//       R_rj -= L_rk X_kj (j <= kb).
// Blocks narrower than 64 are padded with the identity.  With FACTOR false
// D already holds L and only X is formed.  A non-positive or non-finite pivot
// is flagged and replaced by 1.
// 1/sqrt(x) for x > 0: the hardware reciprocal square root estimate in
// float, then Newton-Raphson steps y <- y (3 - x y^2) / 2 (each doubles the
// correct bits; one for float, three for double from the float estimate).
__device__ __forceinline__ float inv_sqrt(float x) {
  float y = rsqrtf(x);
  return y * (1.5f - 0.5f * x * y * y);
}
__device__ __forceinline__ double inv_sqrt(double x) {
  double y = double(rsqrtf(float(x)));
#pragma unroll
  for (int it = 0; it < 3; ++it) y = y * (1.5 - 0.5 * x * y * y);
  return y;
}

constexpr int kDLD = kPanel + 1;
constexpr int kDiagSmemElems = 2 * kPanel * kDLD;

// Step (a) of diag_chol_inv for one 16 x 16 diagonal block at offset o:
// run by one warp only (a separate, non-inlined function so that the other
// warps branch around it instead of issuing it predicated off).
template <typename T, bool FACTOR>
__device__ __noinline__ void diag_leaf16(T* D, T* X, int o, int* status, int s, int b) {
  const int lane = threadIdx.x & 31;
  const int i = lane & 15;
  T v[16];
  T myr = T(0);   // 1 / L[i, i], held by lane i
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = D[(o + i) + (o + q) * kDLD];
  if constexpr (FACTOR) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      T piv = __shfl_sync(0xffffffffu, v[k], k);
      const bool bad = !good_pivot(piv);
      if (bad) piv = T(1);
      const T rk = inv_sqrt(piv);
      const T dk = piv * rk;
      if (bad && lane == 0) flag_pivot(status, s, b);
      if (i > k) v[k] *= rk;
      if (i == k) {
        v[k] = dk;
        myr = rk;
      }
#pragma unroll
      for (int j = k + 1; j < 16; ++j) {
        const T ljk = __shfl_sync(0xffffffffu, v[k], j);
        if (i >= j) v[j] -= v[k] * ljk;
      }
    }
    if (lane < 16) {
#pragma unroll
      for (int q = 0; q < 16; ++q) D[(o + i) + (o + q) * kDLD] = q <= i ? v[q] : T(0);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if (i == k) myr = T(1) / v[k];
  }
  // column j = lane of X_kk: x_i = (delta_ij - sum_{q<i} L_iq x_q) / L_ii
  T x[16];
#pragma unroll
  for (int ii = 0; ii < 16; ++ii) {
    T acc = (ii == i) ? T(1) : T(0);
#pragma unroll
    for (int q = 0; q < ii; ++q) acc -= __shfl_sync(0xffffffffu, v[q], ii) * x[q];
    x[ii] = acc * __shfl_sync(0xffffffffu, myr, ii);
  }
  if (lane < 16) {
#pragma unroll
    for (int ii = 0; ii < 16; ++ii) X[(o + ii) + (o + i) * kDLD] = x[ii];
  }
}

template <typename T, int NT, bool FACTOR>
__device__ __forceinline__ void diag_chol_inv(T* D, T* X, int* status, int s, int b) {
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int kb = 0; kb < 4; ++kb) {
    const int o = kb * 16;
    if (warp == 0) diag_leaf16<T, FACTOR>(D, X, o, status, s, b);   // (a)
    __syncthreads();
    // (b) L_rk for rows r >= o + 16, and X_kj = X_kk R_kj for j < kb; the
    //     results overwrite their inputs, so they are staged in registers
    //     and stored after a barrier
    {
      const int nrow = kPanel - o - 16;
      const int nl = FACTOR ? nrow * 16 : 0, nx = 16 * o;   // nl + nx <= 768
      constexpr int kMax = (48 * 16 + NT - 1) / NT;
      T val[kMax];
#pragma unroll
      for (int u = 0; u < kMax; ++u) {
        const int e = tid + u * NT;
        T acc = T(0);
        if (e < nl) {
          const int r = o + 16 + e % nrow, c = e / nrow;
#pragma unroll
          for (int q = 0; q < 16; ++q) acc += D[r + (o + q) * kDLD] * X[(o + c) + (o + q) * kDLD];
        } else if (e < nl + nx) {
          const int f = e - nl, r = f % 16, c = f / 16;   // X[o + r, c], c < o
#pragma unroll
          for (int q = 0; q < 16; ++q) acc += X[(o + r) + (o + q) * kDLD] * X[(o + q) + c * kDLD];
        }
        val[u] = acc;
      }
      __syncthreads();
#pragma unroll
      for (int u = 0; u < kMax; ++u) {
        const int e = tid + u * NT;
        if (e < nl) {
          const int r = o + 16 + e % nrow, c = e / nrow;
          D[r + (o + c) * kDLD] = val[u];
        } else if (e < nl + nx) {
          const int f = e - nl;
          X[(o + f % 16) + (f / 16) * kDLD] = val[u];
        }
      }
    }
    __syncthreads();
    // (c) trailing updates with block column kb of L and block row kb of X
    {
      const int t0 = o + 16, nt = kPanel - t0;
      const int nd = FACTOR ? nt * nt : 0, nr = nt * (o + 16);
      for (int e = tid; e < nd + nr; e += NT) {
        if (e < nd) {
          const int r = t0 + e % nt, c = t0 + e / nt;
          if (c > r) continue;
          T acc = T(0);
#pragma unroll
          for (int q = 0; q < 16; ++q) acc += D[r + (o + q) * kDLD] * D[c + (o + q) * kDLD];
          D[r + c * kDLD] -= acc;
        } else {
          const int f = e - nd, r = t0 + f % nt, c = f / nt;
          T acc = T(0);
#pragma unroll
          for (int q = 0; q < 16; ++q) acc += D[r + (o + q) * kDLD] * X[(o + q) + c * kDLD];
          X[r + c * kDLD] -= acc;
        }
      }
    }
    __syncthreads();
  }
}

// D (and X = I) from the w x w block at rows/columns c0 of the front F
// (order N), lower part, padded to 64 with the identity
template <typename T, int NT>
__device__ __forceinline__ void diag_load(const T* F, int N, int c0, int w, T* D, T* X) {
  for (int idx = threadIdx.x; idx < kPanel * kPanel; idx += NT) {
    const int r = idx & 63, c = idx >> 6;
    T v = (r == c) ? T(1) : T(0);
    if (r < w && c < w && r >= c) v = F[(c0 + r) + int64_t(c0 + c) * N];
    D[r + c * kDLD] = v;
    X[r + c * kDLD] = (r == c) ? T(1) : T(0);
  }
  __syncthreads();
}

// Factor the diagonal block of the panel starting at column c0 (width w) of
// front F (order N) with NT threads: L_pp is written back into F (lower
// part) and D_p^{-1} (w x w, ld w) to `inv`.  Needs kDiagSmemElems elements
// of shared memory at sm.
template <typename T, int NT>
__device__ __noinline__ void factor_diag(T* F, int N, int c0, int w, T* sm, T* inv,
                                            int* status, int s, int b) {
  T* D = sm;
  T* X = sm + kPanel * kDLD;
  diag_load<T, NT>(F, N, c0, w, D, X);
  diag_chol_inv<T, NT, true>(D, X, status, s, b);
  for (int idx = threadIdx.x; idx < kPanel * kPanel; idx += NT) {
    const int r = idx & 63, c = idx >> 6;
    if (r < w && c < w) {
      if (r >= c) F[(c0 + r) + int64_t(c0 + c) * N] = D[r + c * kDLD];
      inv[r + c * w] = X[r + c * kDLD];
    }
  }
}

}  // namespace
}  // namespace dct
