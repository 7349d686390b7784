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
//    lower tile, C -= L_i L_j^T; in float32 plans 128x128 tensor-core tiles
//    fed from split panel images, update_tc.cu).
//
// A non-positive or NaN pivot is replaced by 1 so the factorization runs to
// the end, and the first such front is recorded in the status words; the host
// reports DCT_ERR_ZERO_PIVOT.  No device assert or trap is used.
#include <cuda_runtime.h>

#include "dct_internal.h"
#include "factor_diag.cuh"
#include "factor_lu.cuh"
#include "tile_mm.cuh"
#include "tc_common.cuh"

namespace dct {
namespace {

template <typename T>
__device__ __forceinline__ T load_val(const void* p, int dtype, int64_t i) {
  if constexpr (sizeof(T) == sizeof(cplx)) {
    if (dtype == DCT_C128) return static_cast<const cplx*>(p)[i];
  }
  return dtype == DCT_F64 ? T(static_cast<const double*>(p)[i])
                          : T(static_cast<const float*>(p)[i]);
}

// resident CTAs per SM the trailing-update kernel is compiled for: two for
// real values, one for complex (its 4 x 4 accumulators and tile copies are
// twice as wide)
template <typename T>
constexpr int kUpdMinBlocks = sizeof(T) > 8 ? 1 : 2;

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
// general plans (fronts2 non-null): the transposed entries, through the
// transpose map tr, go to the same positions of fronts2 (U^T's buffer)
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_large_scatter(DevSym S, const PanelTask* __restrict__ tasks, const void* vals,
                int vals_dtype, int64_t vals_stride, T* fronts,
                int64_t front_stride, T* fronts2, const int32_t* __restrict__ tr) {
  const int s = tasks[blockIdx.x].s;
  const int b = blockIdx.y;
  T* F = fronts + int64_t(b) * front_stride + S.front_off[s];
  T* F2 = fronts2 == nullptr ? nullptr : fronts2 + int64_t(b) * front_stride + S.front_off[s];
  const int64_t a0 = S.amap_ptr[s], a1 = S.amap_ptr[s + 1];
  for (int64_t q = a0 + threadIdx.x; q < a1; q += blockDim.x) {
    F[S.amap_pos[q]] = load_val<T>(vals, vals_dtype,
                                   int64_t(b) * vals_stride + S.amap_e[q]);
    if (F2 != nullptr)
      F2[S.amap_pos[q]] = load_val<T>(vals, vals_dtype,
                                      int64_t(b) * vals_stride + tr[S.amap_e[q]]);
  }
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
// task: s, p, t0 >= 1: the 64-row tile t0-1 below panel p becomes
// F_rows D_p^{-T}, using the inverse stored when the diagonal was factored.
// Float32 plans (im.img non-null) also write the rows' split image
// (hi = tf32(x), lo = x - hi) for the tensor-core trailing update; the
// image's padding rows and the columns beyond a narrow panel stay zero from
// the plan's creation.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_large_panel(DevSym S, const PanelTask* __restrict__ tasks, T* fronts,
              int64_t front_stride, const T* dinv, const int64_t* dinv_off,
              int64_t dinv_stride, ImgArgs im) {
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
  if constexpr (sizeof(T) == 4) {
    if (im.img != nullptr) {
      float* img = im.img + int64_t(b) * im.stride + im.off[im.pan_first[s] + tk.p];
      const int R0 = img_origin(tk.p, ns), G = img_groups(tk.p, ns, N);
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int c = ag + 16 * p;
        if (c >= w) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = jg + 16 * q;
          if (r >= nr) continue;
          const int gr = r0 + r - R0;
          const float v = float(acc[p][q]);
          const uint32_t h = tf32_rna(v);
          img[img_index(G, 0, c / kImgK, gr >> 3, c % kImgK, gr & 7)] = __uint_as_float(h);
          img[img_index(G, 1, c / kImgK, gr >> 3, c % kImgK, gr & 7)] = v - __uint_as_float(h);
        }
      }
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

// One tile update F_out[i, j] -= Fa_i Fb_j^T (K = w): rows ri.. of Fa and
// rj.. of Fb in the panel's columns, 4 x 4 outputs per thread.
template <typename T>
__device__ __forceinline__ void tile_update(const T* Fa, const T* Fb, T* Fo, int N, int c0,
                                            int w, int ri, int rj, int ni, int nj, T* As,
                                            T* Bs) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int idx = tid; idx < kPanel * kUT; idx += kThreads) {
    const int r = idx % kUT, k = idx / kUT;
    const bool kin = k < w;
    As[idx] = (kin && r < ni) ? Fa[(ri + r) + int64_t(c0 + k) * N] : T(0);
    Bs[idx] = (kin && r < nj) ? Fb[(rj + r) + int64_t(c0 + k) * N] : T(0);
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
      cur[p][q] = (cc < nj && rr < ni) ? Fo[(ri + rr) + int64_t(rj + cc) * N] : T(0);
    }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int cc = ag + 16 * p, rr = jg + 16 * q;
      if (cc < nj && rr < ni) Fo[(ri + rr) + int64_t(rj + cc) * N] = cur[p][q] - acc[p][q];
    }
}

// General plans (fronts2 non-null, float64): two products per tile, the lower
// part of the trailing block in F1 -= L_i U_j^T-rows and its upper part,
// transposed in F2, -= U^T_i L_j^T; diagonal blocks by lu_diag.
template <typename T>
__global__ void __launch_bounds__(kThreads, kUpdMinBlocks<T>)
k_large_update(DevSym S, const PanelTask* __restrict__ tasks, T* fronts,
               int64_t front_stride, T* dinv, const int64_t* dinv_off,
               int64_t dinv_stride, int* status, T* fronts2, T* dinv2, double pivot_floor) {
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
  T* F2 = nullptr;
  T* Dv2 = nullptr;
  if constexpr (sizeof(T) == 8) {
    if (fronts2 != nullptr) {
      F2 = fronts2 + int64_t(b) * front_stride + S.front_off[s];
      Dv2 = dinv2 + int64_t(b) * dinv_stride + dinv_off[s];
    }
  }
  // the diagonal block of panel q (Cholesky and inverse, or LU and both
  // inverses)
  auto diag = [&](int q) {
    const int cq = q * kPanel, wq = min(kPanel, ns - cq);
    if constexpr (sizeof(T) == 8) {
      if (F2 != nullptr) {
        lu_diag<kThreads>(reinterpret_cast<double*>(F), reinterpret_cast<double*>(F2), N, cq,
                          wq, reinterpret_cast<double*>(As),
                          reinterpret_cast<double*>(Dv + int64_t(q) * kPanel * kPanel),
                          reinterpret_cast<double*>(Dv2 + int64_t(q) * kPanel * kPanel),
                          status, s, b, pivot_floor);
        return;
      }
    }
    factor_diag<T, kThreads>(F, N, cq, wq, As, Dv + int64_t(q) * kPanel * kPanel, status, s, b);
  };
  if (tk.t0 < 0) {
    diag(tk.p);
    return;
  }
  const int ri = base + tk.t0 * kUT, rj = base + tk.t1 * kUT;
  const int ni = min(kUT, N - ri), nj = min(kUT, N - rj);
  if (F2 == nullptr) {
    tile_update<T>(F, F, F, N, c0, w, ri, rj, ni, nj, As, Bs);
  } else {
    tile_update<T>(F, F2, F, N, c0, w, ri, rj, ni, nj, As, Bs);
    __syncthreads();   // the operand tiles are reloaded
    tile_update<T>(F2, F, F2, N, c0, w, ri, rj, ni, nj, As, Bs);
  }
  if (tk.t0 == 0 && tk.t1 == 0 && base < ns) {
    __syncthreads();   // this CTA's updates of the block are complete
    diag(tk.p + 1);
  }
}

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
cudaError_t run_linv(dct_plan* P, cudaStream_t st, const void* fronts, const void* dinv,
                     void* linv) {
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
      k_linv_init<T><<<grid, kThreads, 0, st>>>(g, static_cast<const T*>(dinv),
                                               static_cast<T*>(linv));
    else if (L.kind == kLinvT)
      k_linv_t<T><<<grid, kThreads, smem, st>>>(g, static_cast<const T*>(fronts),
                                               static_cast<const T*>(linv),
                                               static_cast<T*>(P->ltmp));
    else
      k_linv_x<T><<<grid, kThreads, smem, st>>>(g, static_cast<const T*>(P->ltmp),
                                               static_cast<T*>(linv));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = P->prof.end(st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename T>
cudaError_t factor_impl(dct_plan* P, const void* vals, int vals_dtype,
                        int64_t vals_stride, cudaStream_t st) {
  T* fronts = static_cast<T*>(P->fronts);
  // general plans (float64 only): U^T's buffer
  const bool lu = sizeof(T) == 8 && P->lu != 0;
  T* fronts2 = lu ? static_cast<T*>(P->fronts2) : nullptr;
  const int nb = P->nbatch;
  cudaError_t e = cudaSuccess;
  const int small_max = P->tune.small_front_max;
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
  if constexpr (sizeof(T) == 8) {
    if (e == cudaSuccess && lu)
      e = cudaFuncSetAttribute(k_small_front_lu, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(small_smem));
  }
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
        if constexpr (sizeof(T) == 8) {
          if (lu) {
            k_small_front_lu<<<grid, kThreads, smem, st>>>(
                P->ds, t, static_cast<const double*>(vals), vals_stride, P->d_tr,
                reinterpret_cast<double*>(fronts), reinterpret_cast<double*>(fronts2),
                P->front_stride, P->status, P->pivot_floor);
            break;
          }
        }
        k_small_front<T><<<grid, kThreads, smem, st>>>(
            P->ds, t, vals, vals_dtype, vals_stride, fronts, P->front_stride,
            P->status);
        break;
      }
      case kLargeScatter:
        for (T* buf : {fronts, fronts2}) {
          if (buf == nullptr) continue;
          k_zero_lower<T><<<dim3(static_cast<unsigned>(L.count), nb * kZeroSplit), kThreads,
                            0, st>>>(P->ds, t, buf, P->front_stride);
        }
        k_large_scatter<T><<<grid, kThreads, 0, st>>>(
            P->ds, t, vals, vals_dtype, vals_stride, fronts, P->front_stride, fronts2,
            P->d_tr);
        break;
      case kLargeExtendAdd:
        for (T* buf : {fronts, fronts2}) {
          if (buf == nullptr) continue;
          k_large_extend_add<T><<<grid, kThreads, 0, st>>>(P->ds, t, buf, P->front_stride);
        }
        break;
      case kLargePanel:
        // general plans: L's rows take (U^T)^{-1} (L21 = A21 U11^{-1}), U^T's
        // rows take L^{-1} (U12^T = A12^T L11^{-T})
        e = launch_pdl(k_large_panel<T>, grid, dim3(kThreads), panel_smem, st, P->ds, t, fronts,
                       P->front_stride, static_cast<const T*>(lu ? P->dinv2 : P->dinv),
                       P->d_dinv_off, P->dinv_stride, sizeof(T) == 4 ? P->img : ImgArgs{});
        if (e == cudaSuccess && lu)
          e = launch_pdl(k_large_panel<T>, grid, dim3(kThreads), panel_smem, st, P->ds, t,
                         fronts2, P->front_stride, static_cast<const T*>(P->dinv),
                         P->d_dinv_off, P->dinv_stride, ImgArgs{});
        if (e != cudaSuccess) return e;
        break;
      case kLargeUpdate:
        if constexpr (sizeof(T) == 4) {
          e = launch_update_tc(
              P, t, L.count, li < P->update_nspec.size() ? P->update_nspec[li] : -1, st);
        } else {
          e = launch_pdl(k_large_update<T>, grid, dim3(kThreads), update_smem, st, P->ds, t,
                         fronts, P->front_stride, static_cast<T*>(P->dinv), P->d_dinv_off,
                         P->dinv_stride, P->status, fronts2, static_cast<T*>(P->dinv2),
                         P->pivot_floor);
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
    if (lu)
      k_panel_inverse<T><<<dim3(static_cast<unsigned>(ninv), nb), kThreads, inv_smem,
                           st>>>(P->ds, P->inv.d_tasks, fronts2, P->front_stride,
                                 static_cast<T*>(P->dinv2), P->d_dinv_off,
                                 P->dinv_stride);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = P->prof.end(st);
    if (e != cudaSuccess) return e;
  }
  e = run_linv<T>(P, st, P->fronts, P->dinv, P->linv);
  if (e == cudaSuccess && lu) e = run_linv<T>(P, st, P->fronts2, P->dinv2, P->linv2);
  return e;
}

}  // namespace

cudaError_t run_factor(dct_plan* P, const void* vals, int vals_dtype,
                       int64_t vals_stride, cudaStream_t st) {
  if (P->dtype == DCT_F64)
    return factor_impl<double>(P, vals, vals_dtype, vals_stride, st);
  if (P->dtype == DCT_C128)
    return factor_impl<cplx>(P, vals, vals_dtype, vals_stride, st);
  return factor_impl<float>(P, vals, vals_dtype, vals_stride, st);
}

}  // namespace dct
