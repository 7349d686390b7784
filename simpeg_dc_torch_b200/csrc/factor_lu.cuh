// Fronts of general (unsymmetric-valued, structurally symmetric) float64
// plans: P A P^T = L U without row exchanges, with static pivoting -- a
// pivot whose magnitude is below floor * max|block| (floor = sqrt(eps) by
// default, the threshold of SuperLU_DIST's static pivoting) is replaced by
// that bound with the pivot's sign and counted in status[4]; a non-finite
// pivot records DCT_ERR_ZERO_PIVOT.
//
// Storage, with the layout of the symmetric plans' fronts:
//   F1 (the plan's fronts):   L's multipliers below the diagonal, 1 on it;
//   F2 (the plan's fronts2):  U^T, F2[r][c] = U[c][r] for r >= c.
// A front's boundary block (its Schur complement, the update matrix for the
// parent) keeps its lower part in F1 and its upper part, transposed, in F2,
// so extend-add, the panel TRSM and the substitution kernels of the
// symmetric plans apply to each buffer unchanged.
#pragma once
#include <cuda_runtime.h>

#include "factor_diag.cuh"

namespace dct {
namespace {

// the pivot used at step k of a general front: p itself when finite and not
// smaller than tau in magnitude, else the static replacement
__device__ __forceinline__ double static_pivot(double p, double tau, int* status, int s,
                                               int b) {
  if (!(fabs(p) < INFINITY)) {
    flag_pivot(status, s, b);
    return tau > 0.0 ? tau : 1.0;
  }
  if (fabs(p) >= tau && p != 0.0) return p;
  atomicAdd(&status[4], 1);
  const double t = tau > 0.0 ? tau : 1.0;
  return p < 0.0 ? -t : t;
}

// max over the CTA of the threads' values (NT threads, NT / 32 doubles of red)
template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = 0.0;
  for (int i = 0; i < NT / 32; ++i) m = fmax(m, red[i]);
  __syncthreads();
  return m;
}

// LU of the w x w diagonal block of panel p (columns c0 ..) of a general
// front (order N): D = [lower from F1 | upper from F2^T], padded to 64 with
// the identity; writes L (unit) to F1, U^T to F2, L^{-1} to dinv_l and
// (U^T)^{-1} to dinv_m (w x w, ld w).  Needs kDiagSmemElems doubles at sm.
template <int NT>
__device__ __noinline__ void lu_diag(double* F1, double* F2, int N, int c0, int w, double* sm,
                                     double* dinv_l, double* dinv_m, int* status, int s, int b,
                                     double floor_rel) {
  __shared__ double red[NT / 32];
  double* D = sm;
  double* X = sm + kPanel * kDLD;
  const int tid = threadIdx.x;
  double mx = 0.0;
  for (int idx = tid; idx < kPanel * kPanel; idx += NT) {
    const int r = idx & 63, c = idx >> 6;
    double v = (r == c) ? 1.0 : 0.0;
    if (r < w && c < w) {
      v = r >= c ? F1[(c0 + r) + int64_t(c0 + c) * N] : F2[(c0 + c) + int64_t(c0 + r) * N];
      mx = fmax(mx, fabs(v));
    }
    D[r + c * kDLD] = v;
  }
  const double tau = floor_rel * block_max<NT>(mx, red);
  for (int k = 0; k < kPanel; ++k) {
    if (tid == 0 && k < w) D[k + k * kDLD] = static_pivot(D[k + k * kDLD], tau, status, s, b);
    __syncthreads();
    const double inv = 1.0 / D[k + k * kDLD];
    for (int r = k + 1 + tid; r < kPanel; r += NT) D[r + k * kDLD] *= inv;
    __syncthreads();
    const int nt = kPanel - 1 - k;
    for (int e = tid; e < nt * nt; e += NT) {
      const int r = k + 1 + e % nt, c = k + 1 + e / nt;
      D[r + c * kDLD] -= D[r + k * kDLD] * D[k + c * kDLD];
    }
    __syncthreads();
  }
  // X = L^{-1} (L unit lower: D below the diagonal), one column per thread
  if (tid < kPanel) {
    const int c = tid;
    for (int i = 0; i < kPanel; ++i) {
      double x = 0.0;
      if (i == c) {
        x = 1.0;
      } else if (i > c) {
        double acc = 0.0;
        for (int q = c; q < i; ++q) acc += D[i + q * kDLD] * X[q + c * kDLD];
        x = -acc;
      }
      X[i + c * kDLD] = x;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < w * w; idx += NT) {
    const int r = idx % w, c = idx / w;
    dinv_l[idx] = X[r + c * kDLD];
  }
  __syncthreads();
  // X = M^{-1} for M = U^T (lower, M[i][q] = U[q][i] = D[q][i]), one column
  // per thread
  if (tid < kPanel) {
    const int c = tid;
    for (int i = 0; i < kPanel; ++i) {
      double x = 0.0;
      if (i == c) {
        x = 1.0 / D[c + c * kDLD];
      } else if (i > c) {
        double acc = 0.0;
        for (int q = c; q < i; ++q) acc += D[q + i * kDLD] * X[q + c * kDLD];
        x = -acc / D[i + i * kDLD];
      }
      X[i + c * kDLD] = x;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < w * w; idx += NT) {
    const int r = idx % w, c = idx / w;
    dinv_m[idx] = X[r + c * kDLD];
    if (r >= c) {
      F1[(c0 + r) + int64_t(c0 + c) * N] = r == c ? 1.0 : D[r + c * kDLD];
      F2[(c0 + r) + int64_t(c0 + c) * N] = D[c + r * kDLD];
    }
  }
}

// One CTA per general front of order N <= the single-CTA limit: assemble
// the whole front in shared memory (A's lower entries and, through the
// transpose map, its upper ones; the children's update matrices from both
// buffers), eliminate the ns pivots right-looking over the whole front (the
// boundary block receives its Schur complement), and write L / U^T.
__global__ void __launch_bounds__(kThreads)
k_small_front_lu(DevSym S, const PanelTask* __restrict__ tasks, const double* vals,
                 int64_t vals_stride, const int32_t* __restrict__ tr, double* fronts,
                 double* fronts2, int64_t front_stride, int* status, double floor_rel) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[kThreads / 32];
  double* F = reinterpret_cast<double*>(smem_raw);
  const int s = tasks[blockIdx.x].s;
  const int b = blockIdx.y;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int tid = threadIdx.x;
  const int64_t off = int64_t(b) * front_stride + S.front_off[s];
  for (int i = tid; i < N * N; i += blockDim.x) F[i] = 0.0;
  __syncthreads();
  const double* V = vals + int64_t(b) * vals_stride;
  for (int64_t q = S.amap_ptr[s] + tid; q < S.amap_ptr[s + 1]; q += blockDim.x) {
    const int pos = S.amap_pos[q];
    const int r = pos % N, c = pos / N;
    const int e = S.amap_e[q];
    F[pos] = V[e];
    if (r != c) F[c + r * N] = V[tr[e]];
  }
  __syncthreads();
  for (int ci = S.child_ptr[s]; ci < S.child_ptr[s + 1]; ++ci) {
    const int c = S.child[ci];
    const int nc = S.front_n[c];
    const int nsc = S.sn_first[c + 1] - S.sn_first[c];
    const int nbc = nc - nsc;
    const int64_t coff = int64_t(b) * front_stride + S.front_off[c];
    const double* U1 = fronts + coff;
    const double* U2 = fronts2 + coff;
    const int32_t* rel = S.rel + S.rel_ptr[c];
    for (int idx = tid; idx < nbc * nbc; idx += blockDim.x) {
      const int i = idx % nbc, j = idx / nbc;
      if (i >= j) F[rel[i] + rel[j] * N] += U1[(nsc + i) + int64_t(nsc + j) * nc];
      if (i > j) F[rel[j] + rel[i] * N] += U2[(nsc + i) + int64_t(nsc + j) * nc];
    }
    __syncthreads();
  }
  double mx = 0.0;
  for (int i = tid; i < N * N; i += blockDim.x) mx = fmax(mx, fabs(F[i]));
  const double tau = floor_rel * block_max<kThreads>(mx, red);
  for (int k = 0; k < ns; ++k) {
    if (tid == 0) F[k + k * N] = static_pivot(F[k + k * N], tau, status, s, b);
    __syncthreads();
    const double inv = 1.0 / F[k + k * N];
    for (int r = k + 1 + tid; r < N; r += blockDim.x) F[r + k * N] *= inv;
    __syncthreads();
    const int nt = N - 1 - k;
    for (int e = tid; e < nt * nt; e += blockDim.x) {
      const int r = k + 1 + e % nt, c = k + 1 + e / nt;
      F[r + c * N] -= F[r + k * N] * F[k + c * N];
    }
    __syncthreads();
  }
  double* o1 = fronts + off;
  double* o2 = fronts2 + off;
  for (int i = tid; i < N * N; i += blockDim.x) {
    const int r = i % N, c = i / N;
    o1[i] = r >= c ? ((r == c && c < ns) ? 1.0 : F[i]) : 0.0;
    o2[i] = r >= c ? F[c + r * N] : 0.0;
  }
}

}  // namespace
}  // namespace dct
