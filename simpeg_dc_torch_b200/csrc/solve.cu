// Multi-RHS supernodal substitution L L^T x = b for nbatch systems, in the
// permuted order, on row-major (n, k) right-hand sides.
//
// Per tree level (forward bottom-up, backward top-down):
//   supernodes of one panel (ns <= 64): one CTA per (supernode, system, 64
//     right-hand sides) does the whole step with the stored panel inverse
//     D^{-1} (k_fwd_small / k_bwd_small);
//   larger supernodes: products with the explicit supernode inverse
//     L_ss^{-1} (formed after the factorization) and with the boundary block
//     L_Bs, in 64-row tiles on CUDA cores (float64 plans: k_fwd_linv,
//     k_fwd_bnd, k_bwd_gemm, k_bwd_linv) or in 128-row tiles on the tensor
//     cores (float32 plans, solve_tc.cu).
//
// Two work buffers A and B of nbatch*n*k elements are used so that no launch
// ever reads a location that another CTA of the same launch writes:
//   forward:  b lives in A and receives the updates -L_Bs y_s of the rows
//             below (atomics: several supernodes of a level may share
//             ancestor rows); y_s goes to B.
//   backward: y_s -= L_Bs^T x_B with x_B (rows of ancestors, final) in A;
//             x_s = L_ss^{-T} y_s goes to A.
// The tensor-core kinds split long K ranges over CTAs and accumulate with
// atomics, so in float32 plans B is cleared before the forward pass and A
// (whose right-hand side is consumed by then) before the backward pass.
#include <cuda_runtime.h>

#include "dct_internal.h"
#include "tile_mm.cuh"

namespace dct {
namespace {

constexpr int kRC = kRhsChunk;          // right-hand sides per CTA (64)
constexpr int kLD = kPanel;             // leading dimension of smem tiles

template <typename T>
__device__ __forceinline__ void atomic_sub(T* p, T v) {
  atomicAdd(p, -v);
}

// a finished refinement: the remaining correction launches do nothing
__device__ __forceinline__ bool ir_skip(const int* skip) {
  return skip != nullptr && *reinterpret_cast<const volatile int*>(skip) != 0;
}

// resident CTAs per SM the CUDA-core substitution kernels are compiled for:
// their shared memory admits 4 (float) / 2 (double); 3 caps float at 85
// registers
template <typename T>
constexpr int kSolveMinBlocks = sizeof(T) == 4 ? 3 : (sizeof(T) == 8 ? 2 : 1);

// S1 (the "a" operand) uses a padded leading dimension: several loaders
// store it transposed, which would otherwise hit one bank 32 times.
constexpr int kLD1 = kLD + 1;

template <typename T>
__device__ __forceinline__ void mm_tile(const T* __restrict__ S1,
                                        const T* __restrict__ S2, int K,
                                        int arows, T (&acc)[4][4]) {
  mm64<T, kLD1, kLD>(S1, S2, K, arows, acc);
}

// rows [r0, r0+nr) x right-hand sides [j0, j0+rc) of a (n, k) buffer into
// S[r][j] (ld kLD), zero elsewhere; rows may be gathered through `map`.
template <typename T>
__device__ __forceinline__ void load_rhs(T* S, const T* __restrict__ src, int k,
                                         int j0, int rc, int nr,
                                         const int32_t* map, int64_t r0) {
#pragma unroll
  for (int idx = threadIdx.x; idx < kLD * kRC; idx += kThreads) {
    const int r = idx / kRC, j = idx % kRC;
    T v = T(0);
    if (r < nr && j < rc) {
      const int64_t row = map ? int64_t(map[r]) : r0 + r;
      v = src[row * k + j0 + j];
    }
    S[r * kLD + j] = v;
  }
}

// D^{-1} of panel p (w x w, column-major, ld w) as S[c][r] = Dinv[r, c]
// (transposed = false: forward product) or S[r][c] = Dinv[r, c] (true).
template <typename T>
__device__ __forceinline__ void load_dinv(T* S, const T* __restrict__ Di, int w,
                                          bool transposed) {
#pragma unroll
  for (int idx = threadIdx.x; idx < kLD * kLD; idx += kThreads) {
    const int r = idx % kLD, c = idx / kLD;
    const T v = (r < w && c < w) ? Di[r + c * w] : T(0);
    if (transposed) S[r * kLD1 + c] = v;
    else S[c * kLD1 + r] = v;
  }
}

// ------------------------------------------------------------ forward, small
// one CTA: y = D^{-1} b (to B), then b[boundary rows] -= L_B y (atomics, A)
template <typename T>
__global__ void __launch_bounds__(kThreads, kSolveMinBlocks<T>) k_fwd_small(SolveArgs<T> g) {
  if (ir_skip(g.skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);
  T* S2 = S1 + kLD1 * kLD;
  T* Y = S2 + kLD * kLD;
  // the right-hand-side chunks of a task are adjacent CTAs (its L block
  // is then read from HBM once and from L2 by the other chunks)
  const int s = g.tasks[blockIdx.x / g.nchunk].s;
  const int b = blockIdx.y;
  const int j0 = (blockIdx.x % g.nchunk) * kRC;
  const int rc = min(kRC, g.k - j0);
  const DevSym& S = g.S;
  const int N = S.front_n[s], first = S.sn_first[s];
  const int w = S.sn_first[s + 1] - first;
  const T* F = g.fronts + int64_t(b) * g.front_stride + S.front_off[s];
  T* A = g.A + int64_t(b) * g.n * g.k;
  T* Bo = g.B + int64_t(b) * g.n * g.k;
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
  load_dinv(S1, g.dinv + b * g.dinv_stride + g.dinv_off[s], w, false);
  load_rhs(S2, A, g.k, j0, rc, w, nullptr, first);
  __syncthreads();
  T acc[4][4];
  zero_acc(acc);
  mm_tile(S1, S2, w, w, acc);
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ag + 16 * p, j = jg + 16 * q;
      Y[r * kLD + j] = acc[p][q];
      if (r < w && j < rc) Bo[int64_t(first + r) * g.k + j0 + j] = acc[p][q];
    }
  const int32_t* rows = S.rows + S.rows_ptr[s];
  for (int r0 = w; r0 < N; r0 += kLD) {
    const int nr = min(kLD, N - r0);
    __syncthreads();
#pragma unroll
    for (int idx = threadIdx.x; idx < kLD * kLD; idx += kThreads) {
      const int r = idx % kLD, c = idx / kLD;
      S1[c * kLD1 + r] = (r < nr && c < w) ? F[(r0 + r) + int64_t(c) * N] : T(0);
    }
    __syncthreads();
    zero_acc(acc);
    mm_tile(S1, Y, w, nr, acc);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int r = ag + 16 * p;
      if (r >= nr) continue;
      T* dst = A + int64_t(rows[r0 + r]) * g.k + j0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = jg + 16 * q;
        if (j < rc) atomic_sub(dst + j, acc[p][q]);
      }
    }
  }
}

// ------------------------------------------------------------ forward, boundary
// large supernodes, after all of their panel steps: the 64-row tile t of the
// boundary rows [ns, N) receives -L[tile, 0:ns] y_s (y_s = all panels, in B),
// accumulated over the panels before one atomic update per element.
template <typename T>
__global__ void __launch_bounds__(kThreads, kSolveMinBlocks<T>) k_fwd_bnd(SolveArgs<T> g) {
  if (ir_skip(g.skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);
  T* S2 = S1 + kLD1 * kLD;
  const PanelTask tk = g.tasks[blockIdx.x / g.nchunk];
  const int b = blockIdx.y;
  const int j0 = (blockIdx.x % g.nchunk) * kRC;
  const int rc = min(kRC, g.k - j0);
  const DevSym& S = g.S;
  const int s = tk.s;
  const int N = S.front_n[s], first = S.sn_first[s];
  const int ns = S.sn_first[s + 1] - first;
  const int r0 = ns + tk.t0 * kLD;
  const int nr = min(kLD, N - r0);
  const T* F = g.fronts + int64_t(b) * g.front_stride + S.front_off[s];
  T* A = g.A + int64_t(b) * g.n * g.k;
  const T* Bo = g.B + int64_t(b) * g.n * g.k;
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
  T acc[4][4];
  zero_acc(acc);
  for (int c0 = 0; c0 < ns; c0 += kPanel) {
    const int w = min(kPanel, ns - c0);
    __syncthreads();
#pragma unroll
    for (int idx = threadIdx.x; idx < kLD * kLD; idx += kThreads) {
      const int r = idx % kLD, c = idx / kLD;
      S1[c * kLD1 + r] = (r < nr && c < w) ? F[(r0 + r) + int64_t(c0 + c) * N] : T(0);
    }
    load_rhs(S2, Bo, g.k, j0, rc, w, nullptr, first + c0);
    __syncthreads();
    mm_tile(S1, S2, w, nr, acc);
  }
  const int32_t* rows = S.rows + S.rows_ptr[s];
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int r = ag + 16 * p;
    if (r >= nr) continue;
    T* dst = A + int64_t(rows[r0 + r]) * g.k + j0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = jg + 16 * q;
      if (j < rc) atomic_sub(dst + j, acc[p][q]);
    }
  }
}

// ------------------------------------------------------------ inverse products
// large supernodes: y_s = L_ss^{-1} b_s, 64-row tile t0 per CTA (B <- A rows)
template <typename T>
__global__ void __launch_bounds__(kThreads, kSolveMinBlocks<T>) k_fwd_linv(SolveArgs<T> g) {
  if (ir_skip(g.skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);   // [k][a], ld kLD1: Linv[a, k]
  T* S2 = S1 + kLD1 * kLD;                  // [k][j]: b[k, j]
  const PanelTask tk = g.tasks[blockIdx.x / g.nchunk];
  const int b = blockIdx.y;
  const int j0 = (blockIdx.x % g.nchunk) * kRC;
  const int rc = min(kRC, g.k - j0);
  const DevSym& S = g.S;
  const int s = tk.s;
  const int first = S.sn_first[s];
  const int ns = S.sn_first[s + 1] - first;
  const int r0 = tk.t0 * kLD, nr = min(kLD, ns - r0);
  const T* X = g.linv + int64_t(b) * g.linv_stride + g.linv_off[s];
  const T* A = g.A + int64_t(b) * g.n * g.k;
  T* Bo = g.B + int64_t(b) * g.n * g.k;
  T acc[4][4];
  zero_acc(acc);
  for (int k0 = 0; k0 <= r0; k0 += kLD) {
    const int kw = min(kLD, ns - k0);
    __syncthreads();
#pragma unroll
    for (int idx = threadIdx.x; idx < kLD * kLD; idx += kThreads) {
      const int a = idx % kLD, kk = idx / kLD;
      S1[kk * kLD1 + a] = (a < nr && kk < kw) ? X[(r0 + a) + int64_t(k0 + kk) * ns] : T(0);
    }
    load_rhs(S2, A, g.k, j0, rc, kw, nullptr, first + k0);
    __syncthreads();
    mm_tile(S1, S2, kw, nr, acc);
  }
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ag + 16 * p, j = jg + 16 * q;
      if (r < nr && j < rc) Bo[int64_t(first + r0 + r) * g.k + j0 + j] = acc[p][q];
    }
}

// large supernodes: x_s = L_ss^{-T} y_s, 64-row tile t0 per CTA (A <- B rows)
template <typename T>
__global__ void __launch_bounds__(kThreads, kSolveMinBlocks<T>) k_bwd_linv(SolveArgs<T> g) {
  if (ir_skip(g.skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);   // [k][a], ld kLD1: Linv[k, a]
  T* S2 = S1 + kLD1 * kLD;                  // [k][j]: y[k, j]
  const PanelTask tk = g.tasks[blockIdx.x / g.nchunk];
  const int b = blockIdx.y;
  const int j0 = (blockIdx.x % g.nchunk) * kRC;
  const int rc = min(kRC, g.k - j0);
  const DevSym& S = g.S;
  const int s = tk.s;
  const int first = S.sn_first[s];
  const int ns = S.sn_first[s + 1] - first;
  const int r0 = tk.t0 * kLD, nr = min(kLD, ns - r0);
  const T* X = g.linv + int64_t(b) * g.linv_stride + g.linv_off[s];
  T* A = g.A + int64_t(b) * g.n * g.k;
  const T* Bo = g.B + int64_t(b) * g.n * g.k;
  T acc[4][4];
  zero_acc(acc);
  for (int k0 = r0; k0 < ns; k0 += kLD) {
    const int kw = min(kLD, ns - k0);
    __syncthreads();
#pragma unroll
    for (int idx = threadIdx.x; idx < kLD * kLD; idx += kThreads) {
      const int kk = idx % kLD, a = idx / kLD;
      S1[kk * kLD1 + a] = (a < nr && kk < kw) ? X[(k0 + kk) + int64_t(r0 + a) * ns] : T(0);
    }
    load_rhs(S2, Bo, g.k, j0, rc, kw, nullptr, first + k0);
    __syncthreads();
    mm_tile(S1, S2, kw, nr, acc);
  }
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ag + 16 * p, j = jg + 16 * q;
      if (r < nr && j < rc) A[int64_t(first + r0 + r) * g.k + j0 + j] = acc[p][q];
    }
}

// acc[c][j] += sum_r L[rows_r, c0 + c] x[rows_r, j] over the boundary rows
// [ns, N) of front s (x gathered from A through the front's row list).
template <typename T>
__device__ void boundary_product(const T* F, int N, int ns, int c0, int w,
                                 const int32_t* rows, const T* A, int k, int j0,
                                 int rc, T* S1, T* S2, T (&acc)[4][4]) {
  for (int i0 = ns; i0 < N; i0 += kLD) {
    const int ni = min(kLD, N - i0);
    __syncthreads();
#pragma unroll
    for (int idx = threadIdx.x; idx < kLD * kLD; idx += kThreads) {
      const int r = idx % kLD, c = idx / kLD;
      S1[r * kLD1 + c] = (r < ni && c < w) ? F[(i0 + r) + int64_t(c0 + c) * N] : T(0);
    }
    load_rhs(S2, A, k, j0, rc, ni, rows + i0, 0);
    __syncthreads();
    mm_tile(S1, S2, ni, w, acc);
  }
}

// ------------------------------------------------------------ backward, small
// one CTA: y -= L_B^T x_B ; x = D^{-T} y (to A)
template <typename T>
__global__ void __launch_bounds__(kThreads, kSolveMinBlocks<T>) k_bwd_small(SolveArgs<T> g) {
  if (ir_skip(g.skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);
  T* S2 = S1 + kLD1 * kLD;
  T* Y = S2 + kLD * kLD;
  // the right-hand-side chunks of a task are adjacent CTAs (its L block
  // is then read from HBM once and from L2 by the other chunks)
  const int s = g.tasks[blockIdx.x / g.nchunk].s;
  const int b = blockIdx.y;
  const int j0 = (blockIdx.x % g.nchunk) * kRC;
  const int rc = min(kRC, g.k - j0);
  const DevSym& S = g.S;
  const int N = S.front_n[s], first = S.sn_first[s];
  const int w = S.sn_first[s + 1] - first;
  const T* F = g.fronts + int64_t(b) * g.front_stride + S.front_off[s];
  T* A = g.A + int64_t(b) * g.n * g.k;
  const T* Bo = g.B + int64_t(b) * g.n * g.k;
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
  T acc[4][4];
  zero_acc(acc);
  boundary_product(F, N, w, 0, w, S.rows + S.rows_ptr[s], A, g.k, j0, rc, S1,
                   S2, acc);
  __syncthreads();
  // Y = y - acc
  load_rhs(Y, Bo, g.k, j0, rc, w, nullptr, first);
  __syncthreads();
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) Y[(ag + 16 * p) * kLD + jg + 16 * q] -= acc[p][q];
  load_dinv(S1, g.dinv + b * g.dinv_stride + g.dinv_off[s], w, true);
  __syncthreads();
  zero_acc(acc);
  mm_tile(S1, Y, w, w, acc);
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ag + 16 * p, j = jg + 16 * q;
      if (r < w && j < rc) A[int64_t(first + r) * g.k + j0 + j] = acc[p][q];
    }
}

// ------------------------------------------------------------ backward gemm
// large supernodes: y_p (B) -= L[boundary rows, panel p]^T x[boundary rows]
template <typename T>
__global__ void __launch_bounds__(kThreads, kSolveMinBlocks<T>) k_bwd_gemm(SolveArgs<T> g) {
  if (ir_skip(g.skip)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S1 = reinterpret_cast<T*>(smem_raw);
  T* S2 = S1 + kLD1 * kLD;
  const PanelTask tk = g.tasks[blockIdx.x / g.nchunk];
  const int b = blockIdx.y;
  const int j0 = (blockIdx.x % g.nchunk) * kRC;
  const int rc = min(kRC, g.k - j0);
  const DevSym& S = g.S;
  const int s = tk.s;
  const int N = S.front_n[s], first = S.sn_first[s];
  const int ns = S.sn_first[s + 1] - first;
  const int c0 = tk.p * kPanel, w = min(kPanel, ns - c0);
  const T* F = g.fronts + int64_t(b) * g.front_stride + S.front_off[s];
  const T* A = g.A + int64_t(b) * g.n * g.k;
  T* Bo = g.B + int64_t(b) * g.n * g.k;
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
  T acc[4][4];
  zero_acc(acc);
  boundary_product(F, N, ns, c0, w, S.rows + S.rows_ptr[s], A, g.k, j0, rc, S1,
                   S2, acc);
  T cur[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = ag + 16 * p, j = jg + 16 * q;
      cur[p][q] = (c < w && j < rc) ? Bo[int64_t(first + c0 + c) * g.k + j0 + j] : T(0);
    }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = ag + 16 * p, j = jg + 16 * q;
      if (c < w && j < rc) Bo[int64_t(first + c0 + c) * g.k + j0 + j] = cur[p][q] - acc[p][q];
    }
}

// ------------------------------------------------------------ permutations
template <typename TI, typename TO>
__global__ void k_perm_in(const TI* __restrict__ b, int64_t bstride,
                          const int32_t* __restrict__ perm, int n, int k,
                          TO* __restrict__ dst) {
  const int64_t total = int64_t(n) * k;
  const int bb = blockIdx.y;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = idx / k;
    const int j = static_cast<int>(idx - i * k);
    dst[int64_t(bb) * total + idx] =
        TO(b[int64_t(bb) * bstride + int64_t(perm[i]) * k + j]);
  }
}

template <typename TI, typename TO>
__global__ void k_perm_out(const TI* __restrict__ src, const int32_t* __restrict__ perm,
                           int n, int k, TO* __restrict__ x) {
  const int64_t total = int64_t(n) * k;
  const int bb = blockIdx.y;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = idx / k;
    const int j = static_cast<int>(idx - i * k);
    x[int64_t(bb) * total + int64_t(perm[i]) * k + j] =
        TO(src[int64_t(bb) * total + idx]);
  }
}

template <typename TI, typename TO>
__global__ void k_convert(const TI* __restrict__ src, int64_t sstride, int64_t count,
                          TO* __restrict__ dst) {
  const int bb = blockIdx.y;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x)
    dst[int64_t(bb) * count + i] = TO(src[int64_t(bb) * sstride + i]);
}

// ------------------------------------------------------------ refinement
// right-hand sides per thread of the refinement residual (1, 2, 4 or 8)
#ifndef DCT_RESIDUAL_RHS
#define DCT_RESIDUAL_RHS 4
#endif
constexpr int kResidualRhs = DCT_RESIDUAL_RHS;

// r = b - A x in float64 (permuted order), stored as float into the f32 work
// buffer, with max|r| and max|b| folded into maxbits[0..1] (the refinement
// state's rmax, bmax).  Threads walk the rows in the permuted order: the
// nested dissection keeps each subdomain's rows together, and b and r move
// as contiguous rows (walking the matrix's own order measured 11 % slower
// on the 269,001-node benchmark).

__global__ void k_residual(DevSym S, const double* __restrict__ vals,
                           int64_t vals_stride, const double* __restrict__ b,
                           int64_t bstride, const double* __restrict__ x, int n,
                           int k, float* __restrict__ r32,
                           unsigned long long* __restrict__ maxbits, const int* skip) {
  if (ir_skip(skip)) return;
  const int bb = blockIdx.y;
  const double* V = vals + int64_t(bb) * vals_stride;
  const double* X = x + int64_t(bb) * n * k;
  const double* Bv = b + int64_t(bb) * bstride;
  float* R = r32 + int64_t(bb) * n * k;
  double rmax = 0.0, bmax = 0.0;
  // n * k < 2^31 (checked at launch): 32-bit index arithmetic
  const int total = n * k;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += gridDim.x * blockDim.x) {
    const int i = idx / k;
    const int j = idx - i * k;
    const int orow = S.perm[i];
    double acc = Bv[idx];
    bmax = fmax(bmax, fabs(acc));
    for (int e = S.crow[orow]; e < S.crow[orow + 1]; ++e)
      acc -= V[e] * X[int64_t(S.iperm[S.col[e]]) * k + j];
    R[idx] = static_cast<float>(acc);
    rmax = fmax(rmax, fabs(acc));
  }
  // non-negative doubles order like their bit patterns
  for (int o = 16; o > 0; o >>= 1) {
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&maxbits[0], __double_as_longlong(rmax));
    atomicMax(&maxbits[1], __double_as_longlong(bmax));
  }
}

// The same with RJ = 2, 4 or 8 consecutive right-hand sides per thread (k a
// multiple of RJ, rows 16-byte aligned): the row's pattern, permutation and
// values are read once for RJ outputs, and x, b and r move as 16-byte vectors.
template <int RJ>
__global__ void k_residual_vec(DevSym S, const double* __restrict__ vals,
                               int64_t vals_stride, const double* __restrict__ b,
                               int64_t bstride, const double* __restrict__ x, int n,
                               int k, float* __restrict__ r32,
                               unsigned long long* __restrict__ maxbits, const int* skip) {
  static_assert(RJ == 2 || RJ == 4 || RJ == 8, "2, 4 or 8 right-hand sides per thread");
  if (ir_skip(skip)) return;
  const int bb = blockIdx.y;
  const double* V = vals + int64_t(bb) * vals_stride;
  const double* X = x + int64_t(bb) * n * k;
  const double* Bv = b + int64_t(bb) * bstride;
  float* R = r32 + int64_t(bb) * n * k;
  double rmax = 0.0, bmax = 0.0;
  const int kq = k / RJ;
  // n * k < 2^31 (checked at launch): 32-bit index arithmetic
  const int total = n * kq;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += gridDim.x * blockDim.x) {
    const int i = idx / kq;
    const int o = i * k + (idx - i * kq) * RJ;   // element (i, j)
    const int orow = S.perm[i];
    double acc[RJ];
#pragma unroll
    for (int h = 0; h < RJ; h += 2) {
      const double2 v = *reinterpret_cast<const double2*>(Bv + o + h);
      acc[h] = v.x;
      acc[h + 1] = v.y;
    }
#pragma unroll
    for (int h = 0; h < RJ; ++h) bmax = fmax(bmax, fabs(acc[h]));
    const int j = o - i * k;
    for (int e = S.crow[orow]; e < S.crow[orow + 1]; ++e) {
      const double a = V[e];
      const double* xr = X + S.iperm[S.col[e]] * k + j;
#pragma unroll
      for (int h = 0; h < RJ; h += 2) {
        const double2 v = *reinterpret_cast<const double2*>(xr + h);
        acc[h] -= a * v.x;
        acc[h + 1] -= a * v.y;
      }
    }
    if constexpr (RJ == 2) {
      *reinterpret_cast<float2*>(R + o) = make_float2(float(acc[0]), float(acc[1]));
    } else {
#pragma unroll
      for (int h = 0; h < RJ; h += 4)
        *reinterpret_cast<float4*>(R + o + h) = make_float4(
            float(acc[h]), float(acc[h + 1]), float(acc[h + 2]), float(acc[h + 3]));
    }
#pragma unroll
    for (int h = 0; h < RJ; ++h) rmax = fmax(rmax, fabs(acc[h]));
  }
  for (int off = 16; off > 0; off >>= 1) {
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, off));
    bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&maxbits[0], __double_as_longlong(rmax));
    atomicMax(&maxbits[1], __double_as_longlong(bmax));
  }
}

// x = c (first) or x += c, folding max|c| and max|x| into the refinement
// state (corrections only)
__global__ void k_ir_update(const float* __restrict__ c, int64_t count,
                            double* __restrict__ x, int first, IrState* ir) {
  if (!first && ir_skip(&ir->done)) return;
  double cmax = 0.0, xmax = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double ci = double(c[i]);
    const double xi = first ? ci : x[i] + ci;
    x[i] = xi;
    cmax = fmax(cmax, fabs(ci));
    xmax = fmax(xmax, fabs(xi));
  }
  if (first) return;
  for (int o = 16; o > 0; o >>= 1) {
    cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
  }
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&ir->cmax, __double_as_longlong(cmax));
    atomicMax(&ir->xmax, __double_as_longlong(xmax));
  }
}

// One thread, after correction `iter` (1-based): the estimate of the error
// of x (see IrState), the stopping decision, and DCT_ERR_IR_NOT_CONVERGED in
// the plan's status words (supernode -1, system = iterations) when the
// iterations stagnate or run out above the tolerance.  A NaN correction
// always counts as a failure; a correction at the float64 rounding level of
// x (rho <= 4 eps) ends the refinement as converged.  tol = 0 asks for a
// fixed number of corrections: a stall or running out of them then just
// ends the refinement.
__global__ void k_ir_decide(IrState* ir, int* status, unsigned long long* resid_bits,
                            int iter, int max_iters, double tol) {
  if (ir->done) return;
  // the residual of this iteration becomes the plan's reported residual
  resid_bits[0] = ir->rmax;
  resid_bits[1] = ir->bmax;
  ir->rmax = 0ull;
  ir->bmax = 0ull;
  const double c = __longlong_as_double(static_cast<long long>(ir->cmax));
  const double x = __longlong_as_double(static_cast<long long>(ir->xmax));
  const double rho = x > 0.0 ? c / x : (c > 0.0 ? INFINITY : 0.0);
  const double prev = iter > 1 ? ir->rho[min(iter - 2, kIrHistory - 1)] : 1.0;
  const double q = iter > 1 ? fmin(1.0, rho / prev) : rho;
  const double est = rho * q;
  ir->rho[min(iter - 1, kIrHistory - 1)] = rho;
  ir->iters = iter;
  ir->est = est;
  ir->cmax = 0ull;
  ir->xmax = 0ull;
  const bool nan = !(rho == rho);
  const bool floor = rho <= 4.0 * 2.220446049250313e-16;
  const bool ok = !nan && (floor || (tol > 0.0 && est <= tol));
  const bool stalled = nan || (iter > 1 && rho > 0.5 * prev);
  if (ok) {
    ir->converged = 1;
    ir->done = 1;
  } else if (stalled || iter >= max_iters) {
    // a stall at the accuracy float64 residuals allow is no error under a
    // fixed count (tol = 0); a NaN always is
    ir->done = 1;
    if ((nan || tol > 0.0) && atomicCAS(&status[0], 0, DCT_ERR_IR_NOT_CONVERGED) == 0) {
      status[1] = -1;
      status[2] = iter;
    }
  }
}

inline dim3 grid1d(int64_t total, int ny) {
  int64_t blocks = (total + kThreads - 1) / kThreads;
  blocks = blocks < 1 ? 1 : (blocks > 148 * 16 ? 148 * 16 : blocks);
  return dim3(static_cast<unsigned>(blocks), ny);
}

// transposed: solve A^T x = b (general plans: A^T = (L U)^T = M L^T with
// M = U^T, so the forward pass runs on M and the backward pass on L)
template <typename T>
cudaError_t solve_impl(dct_plan* P, T* bufA, T* bufB, int k, cudaStream_t st,
                       bool transposed = false) {
  const int nchunk = (k + kRC - 1) / kRC;
  const size_t smem3 = sizeof(T) * (kLD1 * kLD + 2 * kLD * kLD);
  cudaError_t e = cudaSuccess;
  const void* kernels[] = {reinterpret_cast<const void*>(k_fwd_small<T>),
                           reinterpret_cast<const void*>(k_fwd_bnd<T>),
                           reinterpret_cast<const void*>(k_fwd_linv<T>),
                           reinterpret_cast<const void*>(k_bwd_linv<T>),
                           reinterpret_cast<const void*>(k_bwd_small<T>),
                           reinterpret_cast<const void*>(k_bwd_gemm<T>)};
  for (const void* kf : kernels) {
    e = cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem3));
    if (e != cudaSuccess) return e;
  }
  SolveArgs<T> g{P->ds, nullptr, static_cast<const T*>(P->fronts), P->front_stride,
                 static_cast<const T*>(P->dinv), P->d_dinv_off, P->dinv_stride,
                 bufA, bufB, P->sym.n, k, nchunk, P->status,
                 static_cast<const T*>(P->linv), P->d_linv_off, P->linv_stride,
                 P->dtype == DCT_F32 && P->ir != nullptr ? &P->ir->done : nullptr};
  constexpr bool kTc = sizeof(T) == 4;
  const size_t work = sizeof(T) * size_t(P->nbatch) * P->sym.n * k;
  const double nb = P->nbatch;
  // general plans: the forward pass runs on L (or M when transposed), the
  // backward pass on the other factor, each with its own inverses
  const T* fac[2] = {static_cast<const T*>(P->fronts), static_cast<const T*>(P->fronts)};
  const T* dv[2] = {static_cast<const T*>(P->dinv), static_cast<const T*>(P->dinv)};
  const T* lv[2] = {static_cast<const T*>(P->linv), static_cast<const T*>(P->linv)};
  if (P->lu) {
    const int m = transposed ? 0 : 1;   // the pass that runs on M = U^T
    fac[m] = static_cast<const T*>(P->fronts2);
    dv[m] = static_cast<const T*>(P->dinv2);
    lv[m] = static_cast<const T*>(P->linv2);
  }
  for (const Schedule* sc : {&P->fwd, &P->bwd}) {
    const int pass = sc == &P->fwd ? 0 : 1;
    g.fronts = fac[pass];
    g.dinv = dv[pass];
    g.linv = lv[pass];
    if (kTc) {
      e = cudaMemsetAsync(sc == &P->fwd ? static_cast<void*>(bufB) : static_cast<void*>(bufA),
                          0, work, st);
      if (e != cudaSuccess) return e;
    }
    for (size_t li = 0; li < sc->launches.size(); ++li) {
      const Launch& L = sc->launches[li];
      if (L.count <= 0) continue;
      if ((e = P->prof.begin(L.kind, sc->flops[li] * k * nb,
                             (sc->bytes[li] + sc->bytes_rhs[li] * k) * nb, st)) !=
          cudaSuccess)
        return e;
      g.tasks = sc->d_tasks + L.first;
      dim3 grid(static_cast<unsigned>(L.count * nchunk), P->nbatch);
      switch (L.kind) {
        case kFwdSmall: k_fwd_small<T><<<grid, kThreads, smem3, st>>>(g); break;
        case kFwdBnd: k_fwd_bnd<T><<<grid, kThreads, smem3, st>>>(g); break;
        case kFwdLinv: k_fwd_linv<T><<<grid, kThreads, smem3, st>>>(g); break;
        case kBwdLinv: k_bwd_linv<T><<<grid, kThreads, smem3, st>>>(g); break;
        case kBwdSmall: k_bwd_small<T><<<grid, kThreads, smem3, st>>>(g); break;
        case kBwdGemm: k_bwd_gemm<T><<<grid, kThreads, smem3, st>>>(g); break;
        case kFwdLinvTc:
        case kFwdBndTc:
        case kBwdGemmTc:
        case kBwdLinvTc:
          if constexpr (kTc) {
            e = launch_solve_tc(L.kind, g, L.count, P->nbatch, st);
            if (e != cudaSuccess) return e;
            break;
          }
          return cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
      }
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if ((e = P->prof.end(st)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

}  // namespace

// f64 plans: the permuted right-hand side is in `xa` (buffer A) and the
// solution is left there; P->bufB serves as buffer B.
cudaError_t run_solve_f64(dct_plan* P, double* xa, int k, cudaStream_t st,
                          bool transposed) {
  return solve_impl<double>(P, xa, static_cast<double*>(P->bufB), k, st, transposed);
}

// complex128 plans: as float64, on complex buffers
cudaError_t run_solve_c128(dct_plan* P, cplx* xa, int k, cudaStream_t st) {
  return solve_impl<cplx>(P, xa, static_cast<cplx*>(P->bufB), k, st);
}

// f32 plans: right-hand side in P->bufA (float, A), P->bufB (B).
cudaError_t run_solve_f32(dct_plan* P, int k, cudaStream_t st) {
  return solve_impl<float>(P, static_cast<float*>(P->bufA),
                           static_cast<float*>(P->bufB), k, st);
}

cudaError_t launch_perm_in_any(const void* b, int b_dtype, int64_t bstride,
                               const int32_t* perm, int n, int k, int nbatch,
                               void* dst, int dst_dtype, cudaStream_t st) {
  dim3 g = grid1d(int64_t(n) * k, nbatch);
  if (b_dtype == DCT_C128 || dst_dtype == DCT_C128) {
    if (b_dtype != dst_dtype) return cudaErrorInvalidValue;
    k_perm_in<cplx, cplx><<<g, kThreads, 0, st>>>(static_cast<const cplx*>(b), bstride, perm,
                                                  n, k, static_cast<cplx*>(dst));
    return cudaGetLastError();
  }
  if (b_dtype == DCT_F64 && dst_dtype == DCT_F64)
    k_perm_in<double, double><<<g, kThreads, 0, st>>>(
        static_cast<const double*>(b), bstride, perm, n, k, static_cast<double*>(dst));
  else if (b_dtype == DCT_F64 && dst_dtype == DCT_F32)
    k_perm_in<double, float><<<g, kThreads, 0, st>>>(
        static_cast<const double*>(b), bstride, perm, n, k, static_cast<float*>(dst));
  else if (b_dtype == DCT_F32 && dst_dtype == DCT_F64)
    k_perm_in<float, double><<<g, kThreads, 0, st>>>(
        static_cast<const float*>(b), bstride, perm, n, k, static_cast<double*>(dst));
  else
    k_perm_in<float, float><<<g, kThreads, 0, st>>>(
        static_cast<const float*>(b), bstride, perm, n, k, static_cast<float*>(dst));
  return cudaGetLastError();
}

cudaError_t launch_perm_out_any(const void* src, int src_dtype, const int32_t* perm,
                                int n, int k, int nbatch, void* x, int x_dtype,
                                cudaStream_t st) {
  dim3 g = grid1d(int64_t(n) * k, nbatch);
  if (src_dtype == DCT_C128 || x_dtype == DCT_C128) {
    if (src_dtype != x_dtype) return cudaErrorInvalidValue;
    k_perm_out<cplx, cplx><<<g, kThreads, 0, st>>>(static_cast<const cplx*>(src), perm, n, k,
                                                   static_cast<cplx*>(x));
    return cudaGetLastError();
  }
  if (src_dtype == DCT_F64 && x_dtype == DCT_F64)
    k_perm_out<double, double><<<g, kThreads, 0, st>>>(
        static_cast<const double*>(src), perm, n, k, static_cast<double*>(x));
  else if (src_dtype == DCT_F64 && x_dtype == DCT_F32)
    k_perm_out<double, float><<<g, kThreads, 0, st>>>(
        static_cast<const double*>(src), perm, n, k, static_cast<float*>(x));
  else if (src_dtype == DCT_F32 && x_dtype == DCT_F64)
    k_perm_out<float, double><<<g, kThreads, 0, st>>>(
        static_cast<const float*>(src), perm, n, k, static_cast<double*>(x));
  else
    k_perm_out<float, float><<<g, kThreads, 0, st>>>(
        static_cast<const float*>(src), perm, n, k, static_cast<float*>(x));
  return cudaGetLastError();
}

cudaError_t launch_convert_any(const void* src, int src_dtype, int64_t sstride,
                               int64_t count, int nbatch, void* dst, int dst_dtype,
                               cudaStream_t st) {
  dim3 g = grid1d(count, nbatch);
  if (src_dtype == DCT_F64 && dst_dtype == DCT_F32)
    k_convert<double, float><<<g, kThreads, 0, st>>>(
        static_cast<const double*>(src), sstride, count, static_cast<float*>(dst));
  else if (src_dtype == DCT_F64 && dst_dtype == DCT_F64)
    k_convert<double, double><<<g, kThreads, 0, st>>>(
        static_cast<const double*>(src), sstride, count, static_cast<double*>(dst));
  else if (src_dtype == DCT_F32 && dst_dtype == DCT_F64)
    k_convert<float, double><<<g, kThreads, 0, st>>>(
        static_cast<const float*>(src), sstride, count, static_cast<double*>(dst));
  else
    k_convert<float, float><<<g, kThreads, 0, st>>>(
        static_cast<const float*>(src), sstride, count, static_cast<float*>(dst));
  return cudaGetLastError();
}

cudaError_t launch_residual(dct_plan* P, const double* b, int64_t bstride,
                            const double* x, int k, cudaStream_t st) {
  const int n = P->sym.n;
  if (int64_t(n) * k >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  const int64_t nnz = static_cast<int64_t>(P->sym.nnz_in);
  float* r = static_cast<float*>(P->bufA);
  // vector rows: k and the batch stride a multiple of kResidualRhs, 16-byte
  // aligned b and x (buffer A comes from cudaMalloc)
  const bool vec = kResidualRhs > 1 && k % kResidualRhs == 0 && bstride % kResidualRhs == 0 &&
                   (reinterpret_cast<uintptr_t>(b) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(x) & 15) == 0;
  if (vec) {
    dim3 g = grid1d(int64_t(n) * (k / kResidualRhs), P->nbatch);
    if (kResidualRhs == 2)
      k_residual_vec<2><<<g, kThreads, 0, st>>>(P->ds, P->vals64, nnz, b, bstride, x, n, k, r,
                                                &P->ir->rmax, &P->ir->done);
    else if (kResidualRhs == 4)
      k_residual_vec<4><<<g, kThreads, 0, st>>>(P->ds, P->vals64, nnz, b, bstride, x, n, k, r,
                                                &P->ir->rmax, &P->ir->done);
    else
      k_residual_vec<8><<<g, kThreads, 0, st>>>(P->ds, P->vals64, nnz, b, bstride, x, n, k, r,
                                                &P->ir->rmax, &P->ir->done);
  } else {
    dim3 g = grid1d(int64_t(n) * k, P->nbatch);
    k_residual<<<g, kThreads, 0, st>>>(P->ds, P->vals64, nnz, b, bstride, x, n, k, r,
                                       &P->ir->rmax, &P->ir->done);
  }
  return cudaGetLastError();
}

cudaError_t launch_ir_update(dct_plan* P, double* x, int k, int first,
                             cudaStream_t st) {
  const int64_t count = int64_t(P->nbatch) * P->sym.n * k;
  dim3 g = grid1d(count, 1);
  k_ir_update<<<g, kThreads, 0, st>>>(static_cast<const float*>(P->bufA), count,
                                      x, first, P->ir);
  return cudaGetLastError();
}

cudaError_t launch_ir_decide(dct_plan* P, int iter, cudaStream_t st) {
  k_ir_decide<<<1, 1, 0, st>>>(P->ir, P->status, P->resid_bits, iter, P->ir_iters,
                                P->ir_tol);
  return cudaGetLastError();
}

}  // namespace dct
