// Numeric multifrontal Cholesky (A = L L^T) of nbatch systems on one pattern.
//
// Fronts are dense N x N column-major blocks (ld = N) in one buffer per
// system.  Levels of the assembly tree run bottom-up; within a level every
// front (and every system of the batch, grid.y) is independent.
//
//  * small fronts (N <= 160 f64 / 224 f32): one CTA assembles the front in
//    shared memory (zero, scatter A entries, extend-add each child's update
//    matrix in turn), runs the partial Cholesky of its ns pivot columns and
//    writes the factor panel and the update matrix back;
//  * large fronts: entries are scattered into the (pre-zeroed) global front,
//    children are extend-added one child slot per launch (so two children of
//    a front never race), then every 64-column panel is factored by a panel
//    kernel (diagonal block Cholesky + TRSM of all rows below it, one CTA per
//    64-row tile) followed by a trailing-update kernel (one CTA per 64x64
//    lower tile, C -= L_i L_j^T).
//
// A non-positive or NaN pivot is replaced by 1 so the factorization runs to
// the end, and the first such front is recorded in the status words; the host
// reports DCT_ERR_ZERO_PIVOT.  No device assert or trap is used.
#include <cuda_runtime.h>

#include "dct_internal.h"
#include "tile_mm.cuh"
#include "tc_common.cuh"

namespace dct {
namespace {

template <typename T>
__device__ __forceinline__ T load_val(const void* p, int dtype, int64_t i) {
  return dtype == DCT_F64 ? T(static_cast<const double*>(p)[i])
                          : T(static_cast<const float*>(p)[i]);
}

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

// ---------------------------------------------------------------- small
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_small_front(DevSym S, const PanelTask* __restrict__ tasks, const void* vals,
              int vals_dtype, int64_t vals_stride, T* fronts,
              int64_t front_stride, int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* F = reinterpret_cast<T*>(smem_raw);
  const int s = tasks[blockIdx.x].s;
  const int b = blockIdx.y;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int tid = threadIdx.x;
  T* out = fronts + int64_t(b) * front_stride + S.front_off[s];

  for (int i = tid; i < N * N; i += blockDim.x) F[i] = T(0);
  __syncthreads();
  const int64_t a0 = S.amap_ptr[s], a1 = S.amap_ptr[s + 1];
  for (int64_t q = a0 + tid; q < a1; q += blockDim.x)
    F[S.amap_pos[q]] = load_val<T>(vals, vals_dtype,
                                   int64_t(b) * vals_stride + S.amap_e[q]);
  __syncthreads();
  for (int ci = S.child_ptr[s]; ci < S.child_ptr[s + 1]; ++ci) {
    const int c = S.child[ci];
    const int nc = S.front_n[c];
    const int nsc = S.sn_first[c + 1] - S.sn_first[c];
    const int nbc = nc - nsc;
    const T* U = fronts + int64_t(b) * front_stride + S.front_off[c];
    const int32_t* rel = S.rel + S.rel_ptr[c];
    for (int idx = tid; idx < nbc * nbc; idx += blockDim.x) {
      const int i = idx % nbc, j = idx / nbc;
      if (i >= j)
        F[rel[i] + rel[j] * N] += U[(nsc + i) + int64_t(nsc + j) * nc];
    }
    __syncthreads();
  }
  // (1) the ns pivot columns: right-looking, updates confined to the panel
  //     (rows below k, columns k+1 .. ns-1); each thread owns whole rows
  for (int k = 0; k < ns; ++k) {
    T piv = F[k + k * N];
    const bool bad = !good_pivot(piv);
    if (bad) piv = T(1);
    const T d = sqrt(piv);
    const T inv = T(1) / d;
    for (int r = k + 1 + tid; r < N; r += blockDim.x) F[r + k * N] *= inv;
    __syncthreads();
    if (tid == 0) {
      F[k + k * N] = d;
      if (bad) flag_pivot(status, s, b);
    }
    for (int r = k + 1 + tid; r < N; r += blockDim.x) {
      const T lrk = F[r + k * N];
      const int cmax = min(r, ns - 1);
      for (int c = k + 1; c <= cmax; ++c) F[r + c * N] -= lrk * F[c + k * N];
    }
    __syncthreads();
  }
  // (2) Schur complement of the boundary rows, F_BB -= L_B L_B^T, in 64 x 64
  //     register tiles (4 x 4 per thread) of the lower triangle
  const int nbr = N - ns;
  const int jg = tid & 15, ag = tid >> 4;
  for (int ti = 0; ti * 64 < nbr; ++ti)
    for (int tj = 0; tj <= ti; ++tj) {
      T acc[4][4];
      zero_acc(acc);
      int ra[4], rb[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        ra[p] = min(ns + ti * 64 + ag + 16 * p, N - 1);
        rb[p] = min(ns + tj * 64 + jg + 16 * p, N - 1);
      }
      for (int k = 0; k < ns; ++k) {
        T x[4], y[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          x[p] = F[ra[p] + k * N];
          y[p] = F[rb[p] + k * N];
        }
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] += x[p] * y[q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int i = ti * 64 + ag + 16 * p, j = tj * 64 + jg + 16 * q;
          if (i < nbr && j <= i) F[(ns + i) + (ns + j) * N] -= acc[p][q];
        }
    }
  __syncthreads();
  // the whole front, upper part as zeros, so the buffer needs no clearing
  for (int i = tid; i < N * N; i += blockDim.x) {
    const int r = i % N, c = i / N;
    out[i] = r >= c ? F[i] : T(0);
  }
}

// ------------------------------------------------------------ large: setup
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_large_scatter(DevSym S, const PanelTask* __restrict__ tasks, const void* vals,
                int vals_dtype, int64_t vals_stride, T* fronts,
                int64_t front_stride) {
  const int s = tasks[blockIdx.x].s;
  const int b = blockIdx.y;
  T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  const int64_t a0 = S.amap_ptr[s], a1 = S.amap_ptr[s + 1];
  for (int64_t q = a0 + threadIdx.x; q < a1; q += blockDim.x)
    F[S.amap_pos[q]] = load_val<T>(vals, vals_dtype,
                                   int64_t(b) * vals_stride + S.amap_e[q]);
}

// Zero the lower triangle (diagonal included) of the large fronts of a
// level before their entries are scattered; the upper triangle of a front is
// never read, and single-CTA fronts write all of theirs.  kZeroSplit CTAs
// per front, one column per warp at a time.
constexpr int kZeroSplit = 32;
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_zero_lower(DevSym S, const PanelTask* __restrict__ tasks, T* fronts,
             int64_t front_stride) {
  const int s = tasks[blockIdx.x].s;
  const int b = blockIdx.y / kZeroSplit, part = blockIdx.y % kZeroSplit;
  const int N = S.front_n[s];
  T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kW = kThreads / 32;
  for (int c = part * kW + warp; c < N; c += kZeroSplit * kW)
    for (int r = c + lane; r < N; r += 32) F[r + int64_t(c) * N] = T(0);
}

// task: s = parent, t0 = child, t1 = first column of the child's update
// matrix handled by this CTA (8 columns, one warp each)
#ifndef DCT_EXTEND_BATCH
#define DCT_EXTEND_BATCH 4
#endif
constexpr int kExtendBatch = DCT_EXTEND_BATCH;

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_large_extend_add(DevSym S, const PanelTask* __restrict__ tasks, T* fronts,
                   int64_t front_stride) {
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s, c = tk.t0;
  const int N = S.front_n[s];
  const int nc = S.front_n[c];
  const int nsc = S.sn_first[c + 1] - S.sn_first[c];
  const int nbc = nc - nsc;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = tk.t1 + warp;
  if (j >= nbc) return;
  T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  const T* U = fronts + int64_t(b) * front_stride + S.front_off[c];
  const int32_t* rel = S.rel + S.rel_ptr[c];
  const int64_t dst_col = int64_t(rel[j]) * N;
  const T* src = U + (nsc + j) * int64_t(nc) + nsc;
  // batches of kExtendBatch per lane, loads before stores (F and U share
  // one buffer); the row map, the child values and then the parent values
  // of a whole batch are in flight together
  for (int i0 = j + lane; i0 < nbc; i0 += kExtendBatch * 32) {
    T sv[kExtendBatch], fv[kExtendBatch];
    int32_t ri[kExtendBatch];
#pragma unroll
    for (int u = 0; u < kExtendBatch; ++u) {
      const int i = i0 + 32 * u;
      ri[u] = i < nbc ? rel[i] : -1;
      sv[u] = i < nbc ? src[i] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kExtendBatch; ++u) fv[u] = ri[u] >= 0 ? F[ri[u] + dst_col] : T(0);
#pragma unroll
    for (int u = 0; u < kExtendBatch; ++u)
      if (ri[u] >= 0) F[ri[u] + dst_col] = fv[u] + sv[u];
  }
}

// ------------------------------------------------------------ large: panels
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
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
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

// task: s, p, t0 >= 1: the 64-row tile t0-1 below panel p becomes
// F_rows D_p^{-T}, using the inverse stored when the diagonal was factored.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_large_panel(DevSym S, const PanelTask* __restrict__ tasks, T* fronts,
              int64_t front_stride, const T* dinv, const int64_t* dinv_off,
              int64_t dinv_stride) {
  pdl_wait();   // launched with launch_pdl: the predecessor's writes first
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);   // [q][c] = Dinv[c, q]
  T* S2 = S1 + kPanel * kPanel;              // [q][r] = F[r, q]
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  const T* Di = dinv + int64_t(b) * dinv_stride + dinv_off[s] +
                int64_t(tk.p) * kPanel * kPanel;
  const int r0 = c0 + w + (tk.t0 - 1) * kPanel;
  const int nr = min(kPanel, N - r0);
#pragma unroll
  for (int idx = threadIdx.x; idx < kPanel * kPanel; idx += kThreads) {
    const int a = idx % kPanel, q = idx / kPanel;
    S1[idx] = (a < w && q < w) ? Di[a + q * w] : T(0);
    S2[idx] = (a < nr && q < w) ? F[(r0 + a) + int64_t(c0 + q) * N] : T(0);
  }
  __syncthreads();
  T acc[4][4];
  zero_acc(acc);
  mm64<T, kPanel, kPanel>(S1, S2, w, w, acc);
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int c = ag + 16 * p;
    if (c >= w) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = jg + 16 * q;
      if (r < nr) F[(r0 + r) + int64_t(c0 + c) * N] = acc[p][q];
    }
  }
}

// task: s, p, t0 = i, t1 = j (i >= j): 64 x 64 tile of the trailing block
// that starts after panel p, F_ij -= L_i L_j^T with K = w (4 x 4 outputs per
// thread, rows on the fast thread index so the tile is written coalesced).
// The CTA of tile (0, 0) -- the next panel's diagonal block -- factors that
// block after its own update (no other task of the launch touches it).
// t0 = -1: factor the diagonal block of panel p itself (a front's first panel).
constexpr int kUT = kUpdateTile;

template <typename T>
__global__ void __launch_bounds__(kThreads, 2)
k_large_update(DevSym S, const PanelTask* __restrict__ tasks, T* fronts,
               int64_t front_stride, T* dinv, const int64_t* dinv_off,
               int64_t dinv_stride, int* status) {
  pdl_wait();   // launched with launch_pdl: the predecessor's writes first
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);   // [k][row of tile i], ld 64
  T* Bs = As + kPanel * kUT;                // [k][row of tile j], ld 64
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  const int base = c0 + w;
  T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  T* Dv = dinv + int64_t(b) * dinv_stride + dinv_off[s];
  const int tid = threadIdx.x;
  if (tk.t0 < 0) {
    factor_diag<T, kThreads>(F, N, c0, w, As, Dv + int64_t(tk.p) * kPanel * kPanel, status, s, b);
    return;
  }
  const int ri = base + tk.t0 * kUT, rj = base + tk.t1 * kUT;
  const int ni = min(kUT, N - ri), nj = min(kUT, N - rj);
#pragma unroll
  for (int idx = tid; idx < kPanel * kUT; idx += kThreads) {
    const int r = idx % kUT, k = idx / kUT;
    const bool kin = k < w;
    As[idx] = (kin && r < ni) ? F[(ri + r) + int64_t(c0 + k) * N] : T(0);
    Bs[idx] = (kin && r < nj) ? F[(rj + r) + int64_t(c0 + k) * N] : T(0);
  }
  __syncthreads();
  T acc[4][4];
  zero_acc(acc);
  mm64<T, kUT, kUT>(Bs, As, w, nj, acc);    // acc[p][q]: col ag+16p, row jg+16q
  const int jg = tid & 15, ag = tid >> 4;
  // all loads first, then the stores: the loads cannot be hoisted over
  // stores to the same buffer, so a fused read-modify-write loop would
  // serialise one global round trip per element
  T cur[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int cc = ag + 16 * p, rr = jg + 16 * q;
      cur[p][q] = (cc < nj && rr < ni) ? F[(ri + rr) + int64_t(rj + cc) * N] : T(0);
    }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int cc = ag + 16 * p, rr = jg + 16 * q;
      if (cc < nj && rr < ni) F[(ri + rr) + int64_t(rj + cc) * N] = cur[p][q] - acc[p][q];
    }
  if (tk.t0 == 0 && tk.t1 == 0 && base < ns) {
    __syncthreads();   // this CTA's updates of the block are complete
    factor_diag<T, kThreads>(F, N, base, min(kPanel, ns - base), As,
                Dv + int64_t(tk.p + 1) * kPanel * kPanel, status, s, b);
  }
}

// ------------------------------------------------------------ tensor cores
// float32 fronts: the trailing update F_ij -= L_i L_j^T of one 128 x 128 tile
// on the 5th-generation tensor cores (tcgen05.mma kind::tf32, accumulator in
// TMEM), with K = the columns [ka, base) given by update_range: one panel for
// the narrow updates inside a block of panels, up to kUpdateBlockPanels
// panels for the deferred update of the columns beyond the block, so that
// the trailing block is read and written once per block instead of once per
// panel.  Each float32 operand x is split as x_hi = tf32(x),
// x_lo = tf32(x - x_hi), and the product is x_hi y_hi + x_hi y_lo + x_lo y_hi
// (the 3xTF32 scheme of Markidis et al., 2018, and Ootomo & Yokota, 2022),
// which restores float32 accuracy from TF32 products accumulated in float32.
//
// K is staged 32 columns at a time through a two-stage shared-memory ring;
// the next stage's operands are loaded into registers while the MMAs of the
// current stage run.  Shared-memory operands are K-major without swizzle:
// core matrices of 8 rows x 16 bytes (4 values), element (m, k) at byte
//   (m / 8) * kUpSbo + (k / 4) * kUpLbo + (m % 8) * 16 + (k % 4) * 4.
// Lane l of a warp handles row m % 8 = l / 4 and column k % 4 = l % 4 of one
// core matrix, so each warp stores one contiguous 128-byte block per operand
// (no bank conflicts) and reads four 32-byte pieces of the front.
constexpr int kUpStK = 32;                                   // K per stage
constexpr uint32_t kUpLbo = 128, kUpSbo = (kUpStK / 4) * kUpLbo;   // 1024
constexpr int kUpOpBytes = (kTcM / 8) * kUpSbo;              // 128 x 32 floats
constexpr int kUpStageBytes = 4 * kUpOpBytes;                // A hi/lo, B hi/lo
constexpr int kUpPer = (kTcM / 8) * (kUpStK / 4) / (kTcThreads / 32);   // 8
// TMEM accumulators: one per panel of a block (a chain of at most kPanel
// K values each; longer float32 accumulation chains inside the tensor core
// measurably lose accuracy), all 512 columns of the SM's TMEM -- one CTA
// per SM
constexpr int kUpAcc = 4;
constexpr int kUpTmemCols = kUpAcc * kTcN;
static_assert(kUpTmemCols <= 512, "TMEM columns of one SM");

// task: s, p, t0 = i, t1 = j (i >= j) over 128-row / 128-column tiles of the
// trailing block after panel p (columns up to update_range's cend), or
// t0 = -1: factor the diagonal block of panel p.  The CTA of tile (0, 0)
// factors the next panel's diagonal block afterwards.
__global__ void __launch_bounds__(kTcThreads, 1)
k_large_update_tc(DevSym S, const PanelTask* __restrict__ tasks, float* fronts,
                  int64_t front_stride, float* dinv, const int64_t* dinv_off,
                  int64_t dinv_stride, int bpan, int* status) {
  pdl_wait();   // launched with launch_pdl: the predecessor's writes first
  pdl_trigger();
  // dynamic shared memory is 16-byte aligned, all the descriptors need;
  // addressing it directly keeps the accesses in the shared state space
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + 2 * kUpStageBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);

  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  const int base = c0 + w;
  float* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  float* Dv = dinv + int64_t(b) * dinv_stride + dinv_off[s];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float* sm = reinterpret_cast<float*>(smem_raw);
  if (tk.t0 < 0) {
    factor_diag<float, kTcThreads>(F, N, c0, w, sm, Dv + int64_t(tk.p) * kPanel * kPanel, status, s,
                                    b);
    return;
  }
  const UpdateRange R = update_range(tk.p, ns, N, bpan);
  const int ri = base + tk.t0 * kTcM, rj = base + tk.t1 * kTcN;
  const int ni = min(kTcM, N - ri), nj = min(kTcN, R.cend - rj);
  const int np = (nj + 15) & ~15;   // MMA N: a multiple of 16
  const int nst = (base - R.ka + kUpStK - 1) / kUpStK;

  if (warp == 0) tmem_alloc(tmem_slot, kUpTmemCols);
  if (tid == 0) {
    mbar_init(&mbar[0]);
    mbar_init(&mbar[1]);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc_tf32(kTcM, np);
  // slot u of this thread: core matrix cm = warp + 16 u, rows
  // m = 8 (cm % 16) + lane / 4, columns kl = 4 (cm / 16) + lane % 4
  const int m_lo = lane >> 2, k_lo = lane & 3;
  float va[kUpPer], vb[kUpPer];
  // the panel columns [ka, base) are read-only in this launch (all writes
  // go to columns >= base), so the read-only path is safe
  auto load_stage = [&](int st) {
    const int kb = R.ka + st * kUpStK;
    const int kw = min(kUpStK, base - kb);
#pragma unroll
    for (int u = 0; u < kUpPer; ++u) {
      const int cm = warp + u * (kTcThreads / 32);
      const int m = (cm % (kTcM / 8)) * 8 + m_lo, kl = (cm / (kTcM / 8)) * 4 + k_lo;
      const int64_t col = int64_t(kb + kl) * N;
      va[u] = (m < ni && kl < kw) ? __ldg(F + (ri + m) + col) : 0.0f;
      vb[u] = (m < nj && kl < kw) ? __ldg(F + (rj + m) + col) : 0.0f;
    }
  };
  bool ok = true;
  load_stage(0);
  for (int st = 0; st < nst; ++st) {
    const int buf = st & 1;
    // the ring slot is free once the MMAs of stage st - 2 have completed
    if (st >= 2) {
      ok = tc_wait(&mbar[buf], uint32_t((st - 2) >> 1) & 1u, status,
                   DCT_ERR_DEVICE_TIMEOUT, s, b);
      if (!ok) break;
    }
    unsigned char* Ahi = smem_raw + buf * kUpStageBytes;
    unsigned char* Alo = Ahi + kUpOpBytes;
    unsigned char* Bhi = Alo + kUpOpBytes;
    unsigned char* Blo = Bhi + kUpOpBytes;
    const int kw = min(kUpStK, base - (R.ka + st * kUpStK));
#pragma unroll
    for (int u = 0; u < kUpPer; ++u) {
      const int cm = warp + u * (kTcThreads / 32);
      const uint32_t off =
          uint32_t(cm % (kTcM / 8)) * kUpSbo + uint32_t(cm / (kTcM / 8)) * kUpLbo + lane * 4;
      tc_store_split(Ahi, Alo, off, va[u]);
      tc_store_split(Bhi, Blo, off, vb[u]);
    }
    if (st + 1 < nst) load_stage(st + 1);
    tc_publish_smem();
    if (tid == 0) {
      const uint32_t ah = smem_u32(Ahi), al = smem_u32(Alo);
      const uint32_t bh = smem_u32(Bhi), bl = smem_u32(Blo);
      for (int kk = 0; kk < (kw + 7) / 8; ++kk) {
        const uint32_t ko = uint32_t(kk) * 2 * kUpLbo;
        const uint64_t dah = umma_desc(ah + ko, kUpLbo, kUpSbo);
        const uint64_t dal = umma_desc(al + ko, kUpLbo, kUpSbo);
        const uint64_t dbh = umma_desc(bh + ko, kUpLbo, kUpSbo);
        const uint64_t dbl = umma_desc(bl + ko, kUpLbo, kUpSbo);
        // one accumulator (128 TMEM columns) per panel of the K range
        const int a = min(st * kUpStK / kPanel, kUpAcc - 1);
        const uint32_t acc = tmem + uint32_t(a * kTcN);
        const bool fresh = st * kUpStK == a * kPanel && kk == 0;
        umma_tf32(acc, dah, dbh, idesc, fresh ? 0u : 1u);
        umma_tf32(acc, dah, dbl, idesc, 1u);
        umma_tf32(acc, dal, dbh, idesc, 1u);
      }
      umma_commit(&mbar[buf]);
    }
  }
  // the last commit tracks every MMA issued before it
  if (ok)
    ok = tc_wait(&mbar[(nst - 1) & 1], uint32_t((nst - 1) >> 1) & 1u, status,
                 DCT_ERR_DEVICE_TIMEOUT, s, b);
  if (ok) {
    // warp w reads TMEM lanes (tile rows) 32(w%4) .. +31, columns 32(w/4) .. +31
    const int row = (warp & 3) * 32 + lane;
    const int cb = (warp >> 2) * 32;
    if (cb < np) {
      float* dst = F + (ri + min(row, ni - 1)) + int64_t(rj + cb) * N;
      float cur[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) cur[c] = (row < ni && cb + c < nj) ? dst[int64_t(c) * N] : 0.0f;
      // the panels' products are subtracted one at a time, each rounded
      // to float32 as in a panel-by-panel update
      const int nacc = min((base - R.ka + kPanel - 1) / kPanel, kUpAcc);
      for (int a = 0; a < nacc; ++a) {
        uint32_t v[32];
        tmem_ld32(tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(a * kTcN + cb), v);
#pragma unroll
        for (int c = 0; c < 32; ++c) cur[c] -= __uint_as_float(v[c]);
      }
      if (row < ni) {
#pragma unroll
        for (int c = 0; c < 32; ++c)
          if (cb + c < nj) dst[int64_t(c) * N] = cur[c];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kUpTmemCols);
  if (ok && tk.t0 == 0 && tk.t1 == 0 && base < ns) {
    __syncthreads();   // this CTA's updates of the block are complete
    factor_diag<float, kTcThreads>(F, N, base, min(kPanel, ns - base), sm,
                Dv + int64_t(tk.p + 1) * kPanel * kPanel, status, s, b);
  }
}

constexpr size_t kTcSmem = 2 * size_t(kUpStageBytes) + 64;
static_assert(2 * size_t(kUpStageBytes) >= sizeof(float) * kDiagSmemElems,
              "tensor-core update smem must also hold factor_diag's workspace");
static_assert(kUpSbo % 16 == 0 && kUpOpBytes % 16 == 0, "descriptor alignment");

// task: s, p.  D_p^{-1} of the factored diagonal block of panel p of a small
// front, written column-major (ld w) at dinv + dinv_off[s] + p*64*64.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_panel_inverse(DevSym S, const PanelTask* __restrict__ tasks, const T* fronts,
                int64_t front_stride, T* dinv, const int64_t* dinv_off,
                int64_t dinv_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* L = reinterpret_cast<T*>(smem_raw);       // ld kDLD
  T* X = L + kPanel * kDLD;                     // ld kDLD
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  const T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  diag_load<T, kThreads>(F, N, c0, w, L, X);
  diag_chol_inv<T, kThreads, false>(L, X, nullptr, s, b);
  T* out = dinv + int64_t(b) * dinv_stride + dinv_off[s] + int64_t(tk.p) * kPanel * kPanel;
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int r = idx % w, c = idx / w;
    out[r + c * w] = X[r + c * kDLD];
  }
}

// ------------------------------------------------------------ supernode inverses
// L_ss^{-1} (ns x ns, column-major, ld ns) of every supernode wider than one
// panel, by recursive doubling from the panel inverses (see the schedule in
// capi.cu).  Blocks of 64 x 64 tiles; K loops skip the zero upper blocks.
struct LinvArgs {
  DevSym S;
  const PanelTask* tasks;
  int64_t front_stride;
  const int64_t* dinv_off;
  int64_t dinv_stride;
  const int64_t* linv_off;
  int64_t linv_stride;
  int h;
};

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_linv_init(LinvArgs g, const T* dinv, T* linv) {
  const PanelTask tk = g.tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s;
  const int ns = g.S.sn_first[s + 1] - g.S.sn_first[s];
  const int c0 = tk.p * kPanel, w = min(kPanel, ns - c0);
  const T* Di = dinv + int64_t(b) * g.dinv_stride + g.dinv_off[s] + int64_t(tk.p) * kPanel * kPanel;
  T* X = linv + int64_t(b) * g.linv_stride + g.linv_off[s];
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int r = idx % w, c = idx / w;
    X[(c0 + r) + int64_t(c0 + c) * ns] = Di[r + c * w];
  }
}

// T[d-block, a-block] = C A^{-1}: C = L[d0.., a0..] (front rows), A^{-1} the
// top block's inverse.  out tile (rt, ct): rows d0 + 64 rt, cols a0 + 64 ct.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_linv_t(LinvArgs g, const T* fronts, const T* linv, T* ltmp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);       // [k][c], ld 65: A^{-1}[k, c]
  T* S2 = S1 + (kPanel + 1) * kPanel;           // [k][r], ld 64: C[r, k]
  const PanelTask tk = g.tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s, h = g.h;
  const DevSym& S = g.S;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int a0 = 2 * tk.p * h, d0 = a0 + h;
  const int hd = min(h, ns - d0);
  const int r0 = tk.t0 * kPanel, cc0 = tk.t1 * kPanel;
  const int nr = min(kPanel, hd - r0);
  const T* F = fronts + int64_t(b) * g.front_stride + S.front_off[s];
  const T* X = linv + int64_t(b) * g.linv_stride + g.linv_off[s];
  T* Tt = ltmp + int64_t(b) * g.linv_stride + g.linv_off[s];
  T acc[4][4];
  zero_acc(acc);
  for (int k0 = cc0; k0 < h; k0 += kPanel) {
    __syncthreads();
#pragma unroll
    for (int idx = threadIdx.x; idx < kPanel * kPanel; idx += kThreads) {
      const int q = idx % kPanel, c = idx / kPanel;   // q: k index (contiguous)
      S1[q * (kPanel + 1) + c] = X[(a0 + k0 + q) + int64_t(a0 + cc0 + c) * ns];
      const int r = idx % kPanel, kk = idx / kPanel;
      S2[kk * kPanel + r] = (r < nr) ? F[(d0 + r0 + r) + int64_t(a0 + k0 + kk) * N] : T(0);
    }
    __syncthreads();
    mm64<T, kPanel + 1, kPanel>(S1, S2, kPanel, kPanel, acc);   // acc[c][r]
  }
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = ag + 16 * p, r = jg + 16 * q;
      if (r < nr) Tt[(d0 + r0 + r) + int64_t(a0 + cc0 + c) * ns] = acc[p][q];
    }
}

// X[d-block, a-block] = -D^{-1} T with D^{-1} the bottom block's inverse.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_linv_x(LinvArgs g, const T* ltmp, T* linv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);       // [k][c], ld 65: T[k, c]
  T* S2 = S1 + (kPanel + 1) * kPanel;           // [k][r], ld 64: D^{-1}[r, k]
  const PanelTask tk = g.tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s, h = g.h;
  const int ns = g.S.sn_first[s + 1] - g.S.sn_first[s];
  const int a0 = 2 * tk.p * h, d0 = a0 + h;
  const int hd = min(h, ns - d0);
  const int r0 = tk.t0 * kPanel, cc0 = tk.t1 * kPanel;
  const int nr = min(kPanel, hd - r0);
  T* X = linv + int64_t(b) * g.linv_stride + g.linv_off[s];
  const T* Tt = ltmp + int64_t(b) * g.linv_stride + g.linv_off[s];
  T acc[4][4];
  zero_acc(acc);
  for (int k0 = 0; k0 <= r0; k0 += kPanel) {
    const int kw = min(kPanel, hd - k0);
    __syncthreads();
#pragma unroll
    for (int idx = threadIdx.x; idx < kPanel * kPanel; idx += kThreads) {
      const int q = idx % kPanel, c = idx / kPanel;
      S1[q * (kPanel + 1) + c] =
          (q < kw) ? Tt[(d0 + k0 + q) + int64_t(a0 + cc0 + c) * ns] : T(0);
      const int r = idx % kPanel, kk = idx / kPanel;
      S2[kk * kPanel + r] =
          (r < nr && kk < kw) ? X[(d0 + r0 + r) + int64_t(d0 + k0 + kk) * ns] : T(0);
    }
    __syncthreads();
    mm64<T, kPanel + 1, kPanel>(S1, S2, kw, kPanel, acc);
  }
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = ag + 16 * p, r = jg + 16 * q;
      if (r < nr) X[(d0 + r0 + r) + int64_t(a0 + cc0 + c) * ns] = -acc[p][q];
    }
}

template <typename T>
cudaError_t run_linv(dct_plan* P, cudaStream_t st) {
  const int nb = P->nbatch;
  const size_t smem = sizeof(T) * ((kPanel + 1) * kPanel + kPanel * kPanel);
  cudaError_t e = cudaFuncSetAttribute(k_linv_t<T>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_linv_x<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  LinvArgs g{P->ds, nullptr, P->front_stride, P->d_dinv_off, P->dinv_stride,
             P->d_linv_off, P->linv_stride, 0};
  for (size_t li = 0; li < P->linv_sched.launches.size(); ++li) {
    const Launch& L = P->linv_sched.launches[li];
    if (L.count <= 0) continue;
    if ((e = P->prof.begin(L.kind, 0.0, 0.0, st)) != cudaSuccess) return e;
    g.tasks = P->linv_sched.d_tasks + L.first;
    g.h = L.arg;
    dim3 grid(static_cast<unsigned>(L.count), nb);
    if (L.kind == kLinvInit)
      k_linv_init<T><<<grid, kThreads, 0, st>>>(g, static_cast<const T*>(P->dinv),
                                               static_cast<T*>(P->linv));
    else if (L.kind == kLinvT)
      k_linv_t<T><<<grid, kThreads, smem, st>>>(g, static_cast<const T*>(P->fronts),
                                               static_cast<const T*>(P->linv),
                                               static_cast<T*>(P->ltmp));
    else
      k_linv_x<T><<<grid, kThreads, smem, st>>>(g, static_cast<const T*>(P->ltmp),
                                               static_cast<T*>(P->linv));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = P->prof.end(st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename T>
cudaError_t factor_impl(dct_plan* P, const void* vals, int vals_dtype,
                        int64_t vals_stride, cudaStream_t st) {
  T* fronts = static_cast<T*>(P->fronts);
  const int nb = P->nbatch;
  cudaError_t e = cudaSuccess;
  const int small_max = sizeof(T) == 8 ? kSmallFrontF64 : kSmallFrontF32;
  const size_t small_smem = sizeof(T) * (size_t(small_max) * small_max + small_max);
  const size_t panel_smem = sizeof(T) * (2 * kPanel * kPanel);
  // the update kernel's tiles, or factor_diag's D and X, whichever is larger
  constexpr int kUpdateElems =
      2 * kPanel * kUT > kDiagSmemElems ? 2 * kPanel * kUT : kDiagSmemElems;
  const size_t update_smem = sizeof(T) * kUpdateElems;
  // attributes are per device: set them on every call (cheap host calls)
  e = cudaFuncSetAttribute(k_small_front<T>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(small_smem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_large_panel<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(panel_smem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_large_update<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(update_smem));
  if (e == cudaSuccess && sizeof(T) == 4)
    e = cudaFuncSetAttribute(k_large_update_tc,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kTcSmem));
  if (e != cudaSuccess) return e;
  const PanelTask* tasks = P->fact.d_tasks;
  for (size_t li = 0; li < P->fact.launches.size(); ++li) {
    const Launch& L = P->fact.launches[li];
    if (L.count <= 0) continue;
    e = P->prof.begin(L.kind, P->fact.flops[li] * nb, P->fact.bytes[li] * nb, st);
    if (e != cudaSuccess) return e;
    // grid.x is limited to 2^31-1, far above any task count here
    dim3 grid(static_cast<unsigned>(L.count), nb);
    const PanelTask* t = tasks + L.first;
    switch (L.kind) {
      case kSmallFront: {
        const size_t smem = sizeof(T) * (size_t(L.arg) * L.arg + L.arg);
        k_small_front<T><<<grid, kThreads, smem, st>>>(
            P->ds, t, vals, vals_dtype, vals_stride, fronts, P->front_stride,
            P->status);
        break;
      }
      case kLargeScatter:
        k_zero_lower<T><<<dim3(static_cast<unsigned>(L.count), nb * kZeroSplit), kThreads,
                          0, st>>>(P->ds, t, fronts, P->front_stride);
        k_large_scatter<T><<<grid, kThreads, 0, st>>>(
            P->ds, t, vals, vals_dtype, vals_stride, fronts, P->front_stride);
        break;
      case kLargeExtendAdd:
        k_large_extend_add<T><<<grid, kThreads, 0, st>>>(P->ds, t, fronts,
                                                         P->front_stride);
        break;
      case kLargePanel:
        e = launch_pdl(k_large_panel<T>, grid, dim3(kThreads), panel_smem, st, P->ds, t, fronts,
                       P->front_stride, static_cast<const T*>(P->dinv), P->d_dinv_off,
                       P->dinv_stride);
        if (e != cudaSuccess) return e;
        break;
      case kLargeUpdate:
        if constexpr (sizeof(T) == 4) {
          e = launch_pdl(k_large_update_tc, grid, dim3(kTcThreads), kTcSmem, st, P->ds, t,
                         reinterpret_cast<float*>(fronts), P->front_stride,
                         static_cast<float*>(P->dinv), P->d_dinv_off, P->dinv_stride,
                         P->update_bpan, P->status);
        } else {
          e = launch_pdl(k_large_update<T>, grid, dim3(kThreads), update_smem, st, P->ds, t,
                         fronts, P->front_stride, static_cast<T*>(P->dinv), P->d_dinv_off,
                         P->dinv_stride, P->status);
        }
        if (e != cudaSuccess) return e;
        break;
      default:
        return cudaErrorInvalidValue;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = P->prof.end(st);
    if (e != cudaSuccess) return e;
  }
  // inverses of the diagonal blocks of small fronts, for the substitution
  // (large fronts store theirs while factoring)
  const size_t inv_smem = sizeof(T) * kDiagSmemElems;
  e = cudaFuncSetAttribute(k_panel_inverse<T>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(inv_smem));
  if (e != cudaSuccess) return e;
  const int64_t ninv = int64_t(P->inv.tasks.size());
  if (ninv > 0) {
    e = P->prof.begin(kPanelInverse, 0.0, 0.0, st);
    if (e != cudaSuccess) return e;
    k_panel_inverse<T><<<dim3(static_cast<unsigned>(ninv), nb), kThreads, inv_smem,
                         st>>>(P->ds, P->inv.d_tasks, fronts, P->front_stride,
                               static_cast<T*>(P->dinv), P->d_dinv_off,
                               P->dinv_stride);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = P->prof.end(st);
    if (e != cudaSuccess) return e;
  }
  return run_linv<T>(P, st);
}

}  // namespace

cudaError_t run_factor(dct_plan* P, const void* vals, int vals_dtype,
                       int64_t vals_stride, cudaStream_t st) {
  if (P->dtype == DCT_F64)
    return factor_impl<double>(P, vals, vals_dtype, vals_stride, st);
  return factor_impl<float>(P, vals, vals_dtype, vals_stride, st);
}

}  // namespace dct
