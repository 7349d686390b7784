// Multi-RHS supernodal substitution L L^T x = b for nbatch systems, in the
// permuted order, on row-major (n, k) right-hand sides.
//
// Two work buffers A and B of nbatch*n*k elements are used so that no launch
// ever reads a location that another CTA of the same launch writes:
//   forward  (levels bottom-up, panel steps in order): the right-hand side b
//            lives in A and receives the updates -L_below y_p (plain stores for
//            rows of the same supernode, atomics for its boundary rows, which
//            other supernodes of the level may also update); the solved panel
//            y_p = D_p^{-1} b_p is written to B.
//   backward (levels top-down): first y_p -= L_{B,p}^T x_B for every panel
//            (x_B are final rows of ancestors, in A); then panel steps from the
//            last panel down: x_p = D_p^{-T} y_p is written to A and
//            y_i -= L_{p,i}^T x_p updates the earlier panels in B.
// Each CTA of a step recomputes the small triangular solve of its panel
// instead of waiting for another CTA: no inter-CTA synchronisation exists.
#include <cuda_runtime.h>

#include "dct_internal.h"

namespace dct {
namespace {

template <typename T>
__device__ __forceinline__ void atomic_sub(T* p, T v) {
  atomicAdd(p, -v);
}

// Load the lower triangle of the w x w diagonal block of panel p (column-major,
// ld 64) and the panel's right-hand-side rows (w x rc, ld kRhsChunk+1).
template <typename T>
__device__ void load_panel(const T* F, int N, int c0, int w, T* D,
                           const T* src, int64_t rowbase, int k, int j0, int rc,
                           T* Y) {
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int r = idx % w, c = idx / w;
    D[r + c * kPanel] = r >= c ? F[(c0 + r) + int64_t(c0 + c) * N] : T(0);
  }
  for (int idx = threadIdx.x; idx < w * rc; idx += blockDim.x) {
    const int r = idx / rc, j = idx % rc;
    Y[r * (kRhsChunk + 1) + j] = src[(rowbase + r) * k + j0 + j];
  }
}

// ------------------------------------------------------------ forward step
// task: s, p; t0 = 0 -> write y_p to B; t0 >= 1 -> row tile t0-1 below the
// panel receives -L_tile y_p in A.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_fwd_step(DevSym S, const PanelTask* __restrict__ tasks, const T* fronts,
           int64_t front_stride, T* bufA, T* bufB, int n, int k, int nchunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* D = reinterpret_cast<T*>(smem_raw);
  T* Y = D + kPanel * kPanel;
  T* Lt = Y + kPanel * (kRhsChunk + 1);
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y / nchunk;
  const int j0 = (blockIdx.y % nchunk) * kRhsChunk;
  const int rc = min(kRhsChunk, k - j0);
  const int s = tk.s;
  const int N = S.front_n[s];
  const int first = S.sn_first[s];
  const int ns = S.sn_first[s + 1] - first;
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  const T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  T* A = bufA + int64_t(b) * n * k;
  T* Bo = bufB + int64_t(b) * n * k;
  load_panel(F, N, c0, w, D, A, int64_t(first + c0), k, j0, rc, Y);
  __syncthreads();
  // forward substitution, one thread per right-hand side
  if (threadIdx.x < rc) {
    const int j = threadIdx.x;
    for (int c = 0; c < w; ++c) {
      T acc = Y[c * (kRhsChunk + 1) + j];
      for (int q = 0; q < c; ++q) acc -= D[c + q * kPanel] * Y[q * (kRhsChunk + 1) + j];
      Y[c * (kRhsChunk + 1) + j] = acc / D[c + c * kPanel];
    }
  }
  __syncthreads();
  if (tk.t0 == 0) {
    for (int idx = threadIdx.x; idx < w * rc; idx += blockDim.x) {
      const int r = idx / rc, j = idx % rc;
      Bo[int64_t(first + c0 + r) * k + j0 + j] = Y[r * (kRhsChunk + 1) + j];
    }
    return;
  }
  const int r0 = c0 + w + (tk.t0 - 1) * kPanel;
  const int nr = min(kPanel, N - r0);
  for (int idx = threadIdx.x; idx < nr * w; idx += blockDim.x) {
    const int r = idx % nr, c = idx / nr;
    Lt[r + c * kPanel] = F[(r0 + r) + int64_t(c0 + c) * N];
  }
  __syncthreads();
  const int32_t* rows = S.rows + S.rows_ptr[s];
  for (int idx = threadIdx.x; idx < nr * rc; idx += blockDim.x) {
    const int r = idx / rc, j = idx % rc;
    T acc = T(0);
    for (int c = 0; c < w; ++c) acc += Lt[r + c * kPanel] * Y[c * (kRhsChunk + 1) + j];
    const int lr = r0 + r;
    T* dst = A + int64_t(rows[lr]) * k + j0 + j;
    if (lr < ns) *dst -= acc;
    else atomic_sub(dst, acc);
  }
}

// ------------------------------------------------------------ backward gemm
// task: s, p: y_p (in B) -= L[boundary rows, panel p]^T x[boundary rows] (A)
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_bwd_gemm(DevSym S, const PanelTask* __restrict__ tasks, const T* fronts,
           int64_t front_stride, const T* bufA, T* bufB, int n, int k,
           int nchunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Lt = reinterpret_cast<T*>(smem_raw);          // [row][col], ld kPanel
  T* Xt = Lt + kPanel * kPanel;                     // [row][j], ld kRhsChunk+1
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y / nchunk;
  const int j0 = (blockIdx.y % nchunk) * kRhsChunk;
  const int rc = min(kRhsChunk, k - j0);
  const int s = tk.s;
  const int N = S.front_n[s];
  const int first = S.sn_first[s];
  const int ns = S.sn_first[s + 1] - first;
  const int nbd = N - ns;
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  const T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  const T* A = bufA + int64_t(b) * n * k;
  T* Bo = bufB + int64_t(b) * n * k;
  const int32_t* rows = S.rows + S.rows_ptr[s];
  // each thread owns outputs (c, j) = idx, idx + 256, ...
  constexpr int kOut = (kPanel * kRhsChunk + kThreads - 1) / kThreads;
  T acc[kOut];
#pragma unroll
  for (int u = 0; u < kOut; ++u) acc[u] = T(0);
  for (int i0 = 0; i0 < nbd; i0 += kPanel) {
    const int ni = min(kPanel, nbd - i0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < ni * w; idx += blockDim.x) {
      const int r = idx % ni, c = idx / ni;
      Lt[r * kPanel + c] = F[(ns + i0 + r) + int64_t(c0 + c) * N];
    }
    for (int idx = threadIdx.x; idx < ni * rc; idx += blockDim.x) {
      const int r = idx / rc, j = idx % rc;
      Xt[r * (kRhsChunk + 1) + j] = A[int64_t(rows[ns + i0 + r]) * k + j0 + j];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kOut; ++u) {
      const int idx = threadIdx.x + u * kThreads;
      const int c = idx / kRhsChunk, j = idx % kRhsChunk;
      if (c < w && j < rc) {
        T a = acc[u];
        for (int r = 0; r < ni; ++r)
          a += Lt[r * kPanel + c] * Xt[r * (kRhsChunk + 1) + j];
        acc[u] = a;
      }
    }
  }
#pragma unroll
  for (int u = 0; u < kOut; ++u) {
    const int idx = threadIdx.x + u * kThreads;
    const int c = idx / kRhsChunk, j = idx % kRhsChunk;
    if (c < w && j < rc) Bo[int64_t(first + c0 + c) * k + j0 + j] -= acc[u];
  }
}

// ------------------------------------------------------------ backward step
// task: s, p; t0 = i <= p.  i == p -> write x_p to A; i < p -> y_i (in B)
// -= L[panel p rows, panel i cols]^T x_p.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_bwd_step(DevSym S, const PanelTask* __restrict__ tasks, const T* fronts,
           int64_t front_stride, T* bufA, T* bufB, int n, int k, int nchunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* D = reinterpret_cast<T*>(smem_raw);
  T* Y = D + kPanel * kPanel;
  T* Lt = Y + kPanel * (kRhsChunk + 1);
  const PanelTask tk = tasks[blockIdx.x];
  const int b = blockIdx.y / nchunk;
  const int j0 = (blockIdx.y % nchunk) * kRhsChunk;
  const int rc = min(kRhsChunk, k - j0);
  const int s = tk.s;
  const int N = S.front_n[s];
  const int first = S.sn_first[s];
  const int ns = S.sn_first[s + 1] - first;
  const int c0 = tk.p * kPanel;
  const int w = min(kPanel, ns - c0);
  const T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  T* A = bufA + int64_t(b) * n * k;
  T* Bo = bufB + int64_t(b) * n * k;
  load_panel(F, N, c0, w, D, Bo, int64_t(first + c0), k, j0, rc, Y);
  __syncthreads();
  if (threadIdx.x < rc) {
    const int j = threadIdx.x;
    for (int c = w - 1; c >= 0; --c) {
      T acc = Y[c * (kRhsChunk + 1) + j];
      for (int q = c + 1; q < w; ++q) acc -= D[q + c * kPanel] * Y[q * (kRhsChunk + 1) + j];
      Y[c * (kRhsChunk + 1) + j] = acc / D[c + c * kPanel];
    }
  }
  __syncthreads();
  if (tk.t0 == tk.p) {
    for (int idx = threadIdx.x; idx < w * rc; idx += blockDim.x) {
      const int r = idx / rc, j = idx % rc;
      A[int64_t(first + c0 + r) * k + j0 + j] = Y[r * (kRhsChunk + 1) + j];
    }
    return;
  }
  const int ci0 = tk.t0 * kPanel;     // earlier panels are full width
  for (int idx = threadIdx.x; idx < w * kPanel; idx += blockDim.x) {
    const int r = idx % w, c = idx / w;
    Lt[r + c * kPanel] = F[(c0 + r) + int64_t(ci0 + c) * N];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < kPanel * rc; idx += blockDim.x) {
    const int c = idx / rc, j = idx % rc;
    T acc = T(0);
    for (int r = 0; r < w; ++r) acc += Lt[r + c * kPanel] * Y[r * (kRhsChunk + 1) + j];
    Bo[int64_t(first + ci0 + c) * k + j0 + j] -= acc;
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
// r = b - A x in float64 (permuted order), stored as float into the f32 work
// buffer, with max|r| and max|b| folded into the status residual slots.
__global__ void k_residual(DevSym S, const double* __restrict__ vals,
                           int64_t vals_stride, const double* __restrict__ b,
                           int64_t bstride, const double* __restrict__ x, int n,
                           int k, float* __restrict__ r32,
                           unsigned long long* __restrict__ maxbits) {
  const int bb = blockIdx.y;
  const double* V = vals + int64_t(bb) * vals_stride;
  const double* X = x + int64_t(bb) * n * k;
  const double* Bv = b + int64_t(bb) * bstride;
  float* R = r32 + int64_t(bb) * n * k;
  double rmax = 0.0, bmax = 0.0;
  const int64_t total = int64_t(n) * k;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(idx / k);
    const int j = static_cast<int>(idx - int64_t(i) * k);
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

__global__ void k_ir_update(const float* __restrict__ c, int64_t count,
                            double* __restrict__ x, int first) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x)
    x[i] = first ? double(c[i]) : x[i] + double(c[i]);
}

inline dim3 grid1d(int64_t total, int ny) {
  int64_t blocks = (total + kThreads - 1) / kThreads;
  blocks = blocks < 1 ? 1 : (blocks > 148 * 16 ? 148 * 16 : blocks);
  return dim3(static_cast<unsigned>(blocks), ny);
}

template <typename T>
cudaError_t solve_impl(dct_plan* P, T* bufA, T* bufB, int k, cudaStream_t st) {
  const int n = P->sym.n;
  const int nchunk = (k + kRhsChunk - 1) / kRhsChunk;
  const size_t step_smem =
      sizeof(T) * (2 * kPanel * kPanel + kPanel * (kRhsChunk + 1));
  const size_t gemm_smem = sizeof(T) * (kPanel * kPanel + kPanel * (kRhsChunk + 1));
  cudaError_t e = cudaFuncSetAttribute(
      k_fwd_step<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
      static_cast<int>(step_smem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bwd_step<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(step_smem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bwd_gemm<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(gemm_smem));
  if (e != cudaSuccess) return e;
  const T* fronts = static_cast<const T*>(P->fronts);
  const double nb = P->nbatch;
  for (size_t li = 0; li < P->fwd.launches.size(); ++li) {
    const Launch& L = P->fwd.launches[li];
    if (L.count <= 0) continue;
    if ((e = P->prof.begin(L.kind, P->fwd.flops[li] * k * nb,
                           (P->fwd.bytes[li] + P->fwd.bytes_rhs[li] * k) * nb,
                           st)) != cudaSuccess)
      return e;
    dim3 grid(static_cast<unsigned>(L.count), P->nbatch * nchunk);
    k_fwd_step<T><<<grid, kThreads, step_smem, st>>>(
        P->ds, P->fwd.d_tasks + L.first, fronts, P->front_stride, bufA, bufB, n,
        k, nchunk);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = P->prof.end(st)) != cudaSuccess) return e;
  }
  for (size_t li = 0; li < P->bwd.launches.size(); ++li) {
    const Launch& L = P->bwd.launches[li];
    if (L.count <= 0) continue;
    if ((e = P->prof.begin(L.kind, P->bwd.flops[li] * k * nb,
                           (P->bwd.bytes[li] + P->bwd.bytes_rhs[li] * k) * nb,
                           st)) != cudaSuccess)
      return e;
    dim3 grid(static_cast<unsigned>(L.count), P->nbatch * nchunk);
    if (L.kind == kBwdGemm)
      k_bwd_gemm<T><<<grid, kThreads, gemm_smem, st>>>(
          P->ds, P->bwd.d_tasks + L.first, fronts, P->front_stride, bufA, bufB,
          n, k, nchunk);
    else
      k_bwd_step<T><<<grid, kThreads, step_smem, st>>>(
          P->ds, P->bwd.d_tasks + L.first, fronts, P->front_stride, bufA, bufB,
          n, k, nchunk);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = P->prof.end(st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

// f64 plans: the permuted right-hand side is in `xa` (buffer A) and the
// solution is left there; P->bufB serves as buffer B.
cudaError_t run_solve_f64(dct_plan* P, double* xa, int k, cudaStream_t st) {
  return solve_impl<double>(P, xa, static_cast<double*>(P->bufB), k, st);
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
  dim3 g = grid1d(int64_t(n) * k, P->nbatch);
  k_residual<<<g, kThreads, 0, st>>>(
      P->ds, P->vals64, static_cast<int64_t>(P->sym.nnz_in), b, bstride, x, n, k,
      static_cast<float*>(P->bufA), P->resid_bits);
  return cudaGetLastError();
}

cudaError_t launch_ir_update(dct_plan* P, double* x, int k, int first,
                             cudaStream_t st) {
  const int64_t count = int64_t(P->nbatch) * P->sym.n * k;
  dim3 g = grid1d(count, 1);
  k_ir_update<<<g, kThreads, 0, st>>>(static_cast<const float*>(P->bufA), count,
                                      x, first);
  return cudaGetLastError();
}

}  // namespace dct
