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
  T* dsh = F + N * N;
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
  // right-looking partial Cholesky of the first ns columns
  for (int k = 0; k < ns; ++k) {
    T piv = F[k + k * N];
    if (!good_pivot(piv)) {
      if (tid == 0) flag_pivot(status, s, b);
      piv = T(1);
    }
    const T d = sqrt(piv);
    const T inv = T(1) / d;
    if (tid == 0) dsh[k] = d;
    const int m = N - k - 1;
    for (int i = tid; i < m; i += blockDim.x) F[(k + 1 + i) + k * N] *= inv;
    __syncthreads();
    for (int idx = tid; idx < m * m; idx += blockDim.x) {
      const int ii = idx % m, jj = idx / m;
      if (ii >= jj)
        F[(k + 1 + ii) + (k + 1 + jj) * N] -=
            F[(k + 1 + ii) + k * N] * F[(k + 1 + jj) + k * N];
    }
    __syncthreads();
  }
  for (int k = tid; k < ns; k += blockDim.x) F[k + k * N] = dsh[k];
  __syncthreads();
  for (int i = tid; i < N * N; i += blockDim.x) out[i] = F[i];
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

// task: s = parent, t0 = child, t1 = first column of the child's update
// matrix handled by this CTA (8 columns, one warp each)
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
  for (int i = j + lane; i < nbc; i += 32) F[rel[i] + dst_col] += src[i];
}

// ------------------------------------------------------------ large: panels
// Factor the w x w diagonal block D (column-major, ld 64) in shared memory.
template <typename T>
__device__ void potrf_smem(T* D, int w, T* dsh, int* status, int s, int b,
                           bool report) {
  const int tid = threadIdx.x;
  for (int k = 0; k < w; ++k) {
    T piv = D[k + k * kPanel];
    if (!good_pivot(piv)) {
      if (report && tid == 0) flag_pivot(status, s, b);
      piv = T(1);
    }
    const T d = sqrt(piv);
    const T inv = T(1) / d;
    if (tid == 0) dsh[k] = d;
    const int m = w - k - 1;
    for (int i = tid; i < m; i += blockDim.x) D[(k + 1 + i) + k * kPanel] *= inv;
    __syncthreads();
    for (int idx = tid; idx < m * m; idx += blockDim.x) {
      const int ii = idx % m, jj = idx / m;
      if (ii >= jj)
        D[(k + 1 + ii) + (k + 1 + jj) * kPanel] -=
            D[(k + 1 + ii) + k * kPanel] * D[(k + 1 + jj) + k * kPanel];
    }
    __syncthreads();
  }
  for (int k = tid; k < w; k += blockDim.x) D[k + k * kPanel] = dsh[k];
  __syncthreads();
}

// task: s, p = panel, t0 >= 1 -> TRSM of row tile t0-1 of the rows below the
// panel.  Every CTA factors the (still unfactored) diagonal block itself; the
// factored block is written by the next launch (k_large_update, t0 = -1), so
// no CTA of this launch can observe it half written.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_large_panel(DevSym S, const PanelTask* __restrict__ tasks, T* fronts,
              int64_t front_stride, int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* D = reinterpret_cast<T*>(smem_raw);
  T* X = D + kPanel * kPanel;
  T* dsh = X + kPanel * kPanel;
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kPanel * kPanel; idx += blockDim.x) {
    const int r = idx % kPanel, c = idx / kPanel;
    D[idx] = (r < w && c < w && r >= c) ? F[(c0 + r) + int64_t(c0 + c) * N] : T(0);
  }
  __syncthreads();
  potrf_smem(D, w, dsh, status, s, b, false);
  const int r0 = c0 + w + (tk.t0 - 1) * kPanel;
  const int nr = min(kPanel, N - r0);
  for (int idx = tid; idx < kPanel * kPanel; idx += blockDim.x) {
    const int r = idx % kPanel, c = idx / kPanel;
    X[idx] = (r < nr && c < w) ? F[(r0 + r) + int64_t(c0 + c) * N] : T(0);
  }
  __syncthreads();
  // X <- X D^{-T}: row r solves D x = a, one thread per row
  if (tid < nr) {
    const int r = tid;
    for (int c = 0; c < w; ++c) {
      T acc = X[r + c * kPanel];
      for (int q = 0; q < c; ++q) acc -= D[c + q * kPanel] * X[r + q * kPanel];
      X[r + c * kPanel] = acc / D[c + c * kPanel];
    }
  }
  __syncthreads();
  for (int idx = tid; idx < nr * w; idx += blockDim.x) {
    const int r = idx % nr, c = idx / nr;
    F[(r0 + r) + int64_t(c0 + c) * N] = X[r + c * kPanel];
  }
}

// task: s, p = panel, t0 = tile row i, t1 = tile col j (i >= j) of the
// trailing block that starts after the panel: F_ij -= L_i L_j^T.
// t0 = -1: factor the panel's diagonal block and write it (no other task of
// this launch reads or writes that block).
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_large_update(DevSym S, const PanelTask* __restrict__ tasks, T* fronts,
               int64_t front_stride, int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);   // [k][row], ld kPanel
  T* Bs = As + kPanel * kPanel;
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y;
  const int s = tk.s;
  const int N = S.front_n[s];
  const int ns = S.sn_first[s + 1] - S.sn_first[s];
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  const int base = c0 + w;
  T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  const int tid = threadIdx.x;
  if (tk.t0 < 0) {
    T* D = As;
    T* dsh = Bs;
    for (int idx = tid; idx < kPanel * kPanel; idx += blockDim.x) {
      const int r = idx % kPanel, c = idx / kPanel;
      D[idx] = (r < w && c < w && r >= c) ? F[(c0 + r) + int64_t(c0 + c) * N] : T(0);
    }
    __syncthreads();
    potrf_smem(D, w, dsh, status, s, b, true);
    for (int idx = tid; idx < w * w; idx += blockDim.x) {
      const int r = idx % w, c = idx / w;
      if (r >= c) F[(c0 + r) + int64_t(c0 + c) * N] = D[r + c * kPanel];
    }
    return;
  }
  const int ri = base + tk.t0 * kPanel, rj = base + tk.t1 * kPanel;
  const int ni = min(kPanel, N - ri), nj = min(kPanel, N - rj);
  for (int idx = tid; idx < kPanel * kPanel; idx += blockDim.x) {
    const int r = idx % kPanel, k = idx / kPanel;
    const bool kin = k < w;
    As[idx] = (kin && r < ni) ? F[(ri + r) + int64_t(c0 + k) * N] : T(0);
    Bs[idx] = (kin && r < nj) ? F[(rj + r) + int64_t(c0 + k) * N] : T(0);
  }
  __syncthreads();
  const int tx = tid & 15;   // rows tx + 16 a
  const int ty = tid >> 4;   // cols ty + 16 c
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = T(0);
  for (int k = 0; k < w; ++k) {
    T av[4], bv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) av[a] = As[k * kPanel + tx + 16 * a];
#pragma unroll
    for (int c = 0; c < 4; ++c) bv[c] = Bs[k * kPanel + ty + 16 * c];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][c] += av[a] * bv[c];
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int cc = ty + 16 * c;
    if (cc >= nj) continue;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int rr = tx + 16 * a;
      if (rr < ni) F[(ri + rr) + int64_t(rj + cc) * N] -= acc[a][c];
    }
  }
}

template <typename T>
cudaError_t factor_impl(dct_plan* P, const void* vals, int vals_dtype,
                        int64_t vals_stride, cudaStream_t st) {
  T* fronts = static_cast<T*>(P->fronts);
  const int nb = P->nbatch;
  cudaError_t e = cudaMemsetAsync(fronts, 0,
                                  sizeof(T) * P->front_stride * size_t(nb), st);
  if (e != cudaSuccess) return e;
  const int small_max = sizeof(T) == 8 ? kSmallFrontF64 : kSmallFrontF32;
  const size_t small_smem = sizeof(T) * (size_t(small_max) * small_max + small_max);
  const size_t panel_smem = sizeof(T) * (2 * kPanel * kPanel + kPanel);
  const size_t update_smem = sizeof(T) * (2 * kPanel * kPanel);
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
        k_large_scatter<T><<<grid, kThreads, 0, st>>>(
            P->ds, t, vals, vals_dtype, vals_stride, fronts, P->front_stride);
        break;
      case kLargeExtendAdd:
        k_large_extend_add<T><<<grid, kThreads, 0, st>>>(P->ds, t, fronts,
                                                         P->front_stride);
        break;
      case kLargePanel:
        k_large_panel<T><<<grid, kThreads, panel_smem, st>>>(P->ds, t, fronts,
                                                    P->front_stride, P->status);
        break;
      case kLargeUpdate:
        k_large_update<T><<<grid, kThreads, update_smem, st>>>(
            P->ds, t, fronts, P->front_stride, P->status);
        break;
      default:
        return cudaErrorInvalidValue;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = P->prof.end(st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

cudaError_t run_factor(dct_plan* P, const void* vals, int vals_dtype,
                       int64_t vals_stride, cudaStream_t st) {
  if (P->dtype == DCT_F64)
    return factor_impl<double>(P, vals, vals_dtype, vals_stride, st);
  return factor_impl<float>(P, vals, vals_dtype, vals_stride, st);
}

}  // namespace dct
