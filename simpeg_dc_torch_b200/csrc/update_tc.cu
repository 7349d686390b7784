// Float32 trailing update of the large fronts on the tensor cores,
// F_ij -= L_i L_j^T over 128 x 128 tiles, with the operands streamed from
// the split panel images (see img_origin in dct_internal.h) that the panel
// TRSM writes once per panel.
//
// One CTA per output tile, warp-specialised:
//   warp 0    one thread issues the bulk copies (cp.async.bulk ... complete_tx)
//             of each K stage -- kImgK columns of the hi and lo images of the
//             tile's row block i and column block j, 16 KB each for 32
//             columns, contiguous in the images -- into a ring of stages that
//             fills kURingBytes (two stages of 64 KB), each stage guarded by
//             a "full" mbarrier (transaction bytes) and an "empty" one.
//             Deeper rings of smaller stages (16 columns: four or five stages
//             of 32 KB) measured slower on the 269,001-node benchmark (+1.5 %
//             / +6 % on this kernel): the copies' latency is not what bounds
//             it, the per-tile prologue and epilogue of one CTA per SM are;
//   warp 1    allocates TMEM and one thread issues tcgen05.mma kind::tf32 for
//             each stage (3xTF32: hi*hi + hi*lo + lo*hi; Markidis et al. 2018,
//             Ootomo & Yokota 2022), then commits to the stage's "empty"
//             barrier so the ring slot can be refilled;
//   warps 2-5 copy the output tile into shared memory (cp.async, one row
//             per thread) while the MMAs run, wait for the last commit, read
//             the accumulators from TMEM and store the difference.
// No thread converts or stages operands: the split happens once per panel,
// not once per tile and K stage.
//
// K is the column range [ka, base) of update_range: one panel for the
// narrow updates inside a block of panels, up to four for the update of the
// columns beyond the block.  Each panel accumulates in its own TMEM
// accumulator (128 columns; all 512) and the panels' products are
// subtracted one at a time, each rounded to float32, as in a
// panel-by-panel update.  Tiles start at R0 = base & ~7 (the 8-row grid of
// the images); rows and columns above `base` belong to the panel itself and
// are left untouched, as are columns at or beyond the update's end and, in
// diagonal tiles, the upper triangle.  The CTA of tile (0, 0) then factors
// the next panel's diagonal block.  Every wait is bounded (kTcWaitLimit
// polls): on timeout DCT_ERR_DEVICE_TIMEOUT is recorded and the CTA returns.
//
// Wide launches of one system (many tiles, few fronts; chosen when the plan
// is built) run persistent CTAs instead: the diagonal tiles come first in the
// launch's tasks and keep one CTA each, and one persistent CTA on every other
// SM loops over the remaining tiles (update_persistent), so that the copies
// and MMAs of the next tile overlap the epilogue of the current one.  On the
// 269,001-node benchmark this took the wide launches from 4.64 to 3.69 ms
// (serialised launch list) and the step by 0.24 ms.
#include <cuda_runtime.h>

#include <algorithm>

#include "dct_internal.h"
#include "factor_diag.cuh"
#include "tc_common.cuh"

namespace dct {
namespace {

#ifndef DCT_U_RING_KB
#define DCT_U_RING_KB 160
#endif
constexpr int kUThreads = 192;
constexpr int kUChunk = 128 * kImgK * 4;    // 128 rows x kImgK columns, hi or lo
constexpr int kUStageBytes = 4 * kUChunk;   // A hi, A lo, B hi, B lo
constexpr int kURingBytes = DCT_U_RING_KB * 1024;
constexpr int kUStages = kURingBytes / kUStageBytes;
constexpr uint32_t kULbo = 128, kUSbo = 32 * kImgK;
static_assert(kUStages >= 2, "at least two stages in the copy ring");
constexpr int kUAcc = 4;                    // accumulators: one per panel
constexpr int kUTileBytes = kTcM * kTcN * 4;   // the output tile, staged
constexpr int kUBarBytes = 256;             // mbarriers, TMEM address, abort word
constexpr size_t kUSmem = size_t(kUStages) * kUStageBytes + kUTileBytes + kUBarBytes;
static_assert(kUAcc * 128 <= 512, "TMEM columns of one SM");
static_assert(size_t(kUStages) * kUStageBytes >= sizeof(float) * kDiagSmemElems,
              "the ring also holds factor_diag's workspace");
static_assert(kUSmem <= 227 * 1024, "shared memory of one CTA");
static_assert((2 * kUStages + 2 * kUAcc + 1) * 8 + 8 <= kUBarBytes,
              "barriers, the TMEM slot and the abort word");

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// bulk global -> shared copy whose completion is counted on `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// one thread: bounded wait for phase `parity`
__device__ __forceinline__ bool mbar_wait1(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < kTcWaitLimit; ++it)
    if (mbar_try_wait_sleep(smem_u32(bar), parity)) return true;
  return false;
}

__device__ __forceinline__ void flag_timeout(int* status, int s, int b) {
  if (atomicCAS(&status[0], 0, DCT_ERR_DEVICE_TIMEOUT) == 0) {
    status[1] = s;
    status[2] = b;
  }
}

__device__ __forceinline__ void mbar_init_n(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// one thread: bounded wait for phase `parity` that also gives up once another
// role of the CTA has given up (*abort set); a timeout sets *abort
__device__ __forceinline__ bool mbar_wait_ab(uint64_t* bar, uint32_t parity,
                                             volatile int* abort) {
  for (uint32_t it = 0; it < kTcWaitLimit; ++it) {
    if (mbar_try_wait_sleep(smem_u32(bar), parity)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}

// geometry of one trailing-update tile (task tk)
struct UTile {
  int s, N, ns, base, ka, ri, rj, jn, np, nst, nacc;
  bool diag;
};

__device__ __forceinline__ UTile utile_of(const DevSym& S, const PanelTask& tk, int bpan) {
  UTile t;
  t.s = tk.s;
  t.N = S.front_n[tk.s];
  t.ns = S.sn_first[tk.s + 1] - S.sn_first[tk.s];
  const int c0 = tk.p * kPanel;
  t.base = c0 + min(kPanel, t.ns - c0);
  const UpdateRange R = update_range(tk.p, t.ns, t.N, bpan);
  t.ka = R.ka;
  const int R0 = t.base & ~7;
  t.ri = R0 + tk.t0 * kTcM;
  t.rj = R0 + tk.t1 * kTcN;
  t.diag = tk.t0 == tk.t1;
  t.jn = min(kTcN, R.cend - t.rj);   // tile columns that can be written
  t.np = (t.jn + 15) & ~15;          // MMA N: a multiple of 16
  t.nst = (t.base - R.ka + kImgK - 1) / kImgK;
  t.nacc = (t.base - R.ka + kPanel - 1) / kPanel;
  return t;
}

// the chunk of rows row0 .. row0 + 127, K stage st, hi (0) / lo (1) of tile t
__device__ __forceinline__ const float* uchunk(const ImgArgs& im, const float* img, int pan0,
                                               const UTile& t, int row0, int st, int hl) {
  const int kcol = t.ka + kImgK * st;
  const int q = kcol / kPanel;
  const int G = img_groups(q, t.ns, t.N);
  const int g0 = (row0 - img_origin(q, t.ns)) >> 3;
  return img + im.off[pan0 + q] + img_index(G, hl, (kcol % kPanel) / kImgK, g0, 0, 0);
}

// Persistent CTA (one system): the tiles nspec + c, nspec + c + P, ... of the
// launch, c = this CTA's index among the P persistent ones.  The copy ring
// and the four TMEM accumulators run on across tiles: warp 0 copies the next
// tile's stages while warp 1 still multiplies the current one, and the MMAs
// of panel g go to accumulator g % 4 once the epilogue has released it
// (mbarrier "free"), so the MMAs of the next tile overlap the epilogue of
// this one.  The epilogue warps subtract each panel's accumulator from the
// staged output tile as soon as it completes ("full"), panel by panel with
// float32 rounding as in the one-tile path, then store the tile.  A timeout
// in any role sets the CTA's abort word; the other roles stop at their next
// wait, MMAs and copies already issued are waited for, and
// DCT_ERR_DEVICE_TIMEOUT is recorded.
__device__ void update_persistent(const DevSym& S, const PanelTask* __restrict__ tasks,
                                  int64_t count, int nspec, float* fronts, int bpan,
                                  int* status, const ImgArgs& im, unsigned char* smem_raw) {
  float* Cs = reinterpret_cast<float*>(smem_raw + kUStages * kUStageBytes);   // [col][row]
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kUStages * kUStageBytes + kUTileBytes);
  uint64_t* empty = full + kUStages;
  uint64_t* accf = empty + kUStages;
  uint64_t* accr = accf + kUAcc;
  uint64_t* done = accr + kUAcc;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t first = blockIdx.x;                 // nspec + c
  const int64_t stride = int64_t(gridDim.x) - nspec;  // P

  if (warp == 1) tmem_alloc(tmem_slot, kUAcc * 128);
  if (tid == 0) {
    for (int i = 0; i < kUStages; ++i) {
      mbar_init(&full[i]);
      mbar_init(&empty[i]);
    }
    for (int a = 0; a < kUAcc; ++a) {
      mbar_init(&accf[a]);
      mbar_init_n(&accr[a], 4);   // one arrival per epilogue warp
    }
    mbar_init(done);
    *abort = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const float* img = im.img;
  bool ok = true;
  int bad_s = -1;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t gs = 0;   // stages issued by this CTA
      for (int64_t i = first; i < count && ok; i += stride) {
        const UTile t = utile_of(S, tasks[i], bpan);
        const int pan0 = im.pan_first[t.s];
        const uint32_t bytes = t.diag ? 2 * kUChunk : 4 * kUChunk;
        for (int st = 0; st < t.nst; ++st, ++gs) {
          const uint32_t slot = gs % kUStages;
          if (gs >= kUStages &&
              !mbar_wait_ab(&empty[slot], (gs / kUStages - 1) & 1u, abort)) {
            ok = false;
            bad_s = t.s;
            break;
          }
          unsigned char* dst = smem_raw + slot * kUStageBytes;
          mbar_expect_tx(&full[slot], bytes);
          bulk_g2s(dst, uchunk(im, img, pan0, t, t.ri, st, 0), kUChunk, &full[slot]);
          bulk_g2s(dst + kUChunk, uchunk(im, img, pan0, t, t.ri, st, 1), kUChunk, &full[slot]);
          if (!t.diag) {
            bulk_g2s(dst + 2 * kUChunk, uchunk(im, img, pan0, t, t.rj, st, 0), kUChunk,
                     &full[slot]);
            bulk_g2s(dst + 3 * kUChunk, uchunk(im, img, pan0, t, t.rj, st, 1), kUChunk,
                     &full[slot]);
          }
        }
      }
      // no copy may still be writing shared memory at exit: the last stages'
      // copies have landed once their barriers complete (copies always end)
      for (uint32_t g = gs > uint32_t(kUStages) ? gs - kUStages : 0u; g < gs; ++g)
        if (!mbar_wait1(&full[g % kUStages], (g / kUStages) & 1u)) ok = false;
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t gs = 0, gp = 0;   // stages consumed, panels accumulated
      for (int64_t i = first; i < count && ok; i += stride) {
        const UTile t = utile_of(S, tasks[i], bpan);
        const uint32_t idesc = umma_idesc_tf32(kTcM, t.np);
        uint32_t acc = tmem;
        for (int st = 0; st < t.nst; ++st, ++gs) {
          const uint32_t slot = gs % kUStages;
          const int kcol = t.ka + kImgK * st;
          const bool pfirst = kcol % kPanel == 0;
          const bool plast = st == t.nst - 1 || (kcol + kImgK) % kPanel == 0;
          if (pfirst) {
            const uint32_t a = gp % kUAcc;
            if (gp >= uint32_t(kUAcc) &&
                !mbar_wait_ab(&accr[a], (gp / kUAcc - 1) & 1u, abort)) {
              ok = false;
              bad_s = t.s;
              break;
            }
            acc = tmem + a * 128u;
          }
          if (!mbar_wait_ab(&full[slot], (gs / kUStages) & 1u, abort)) {
            ok = false;
            bad_s = t.s;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t ah = smem_u32(smem_raw + slot * kUStageBytes);
          const uint32_t al = ah + kUChunk;
          const uint32_t bh = t.diag ? ah : ah + 2 * kUChunk;
          const uint32_t bl = t.diag ? al : ah + 3 * kUChunk;
#pragma unroll
          for (int kk = 0; kk < kImgK / 8; ++kk) {
            const uint32_t ko = uint32_t(kk) * 2 * kULbo;
            const uint64_t dah = umma_desc(ah + ko, kULbo, kUSbo);
            const uint64_t dal = umma_desc(al + ko, kULbo, kUSbo);
            const uint64_t dbh = umma_desc(bh + ko, kULbo, kUSbo);
            const uint64_t dbl = umma_desc(bl + ko, kULbo, kUSbo);
            umma_tf32(acc, dah, dbh, idesc, (pfirst && kk == 0) ? 0u : 1u);
            umma_tf32(acc, dah, dbl, idesc, 1u);
            umma_tf32(acc, dal, dbh, idesc, 1u);
          }
          umma_commit(&empty[slot]);
          if (plast) {
            umma_commit(&accf[gp % kUAcc]);
            ++gp;
          }
        }
      }
      // tracks every MMA issued, also after an abort
      umma_commit(done);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 = tile rows; each
    // thread stages, updates and stores its own row of the tile, so the
    // staged tile needs no barrier between threads
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;
    uint32_t gp = 0;
    for (int64_t i = first; i < count && ok; i += stride) {
      const UTile t = utile_of(S, tasks[i], bpan);
      const int row = t.ri + r;
      const bool row_ok = row >= t.base && row < t.N;
      const int c_lo = max(0, t.base - t.rj);
      const int c_hi = row_ok ? min(t.jn, t.diag ? row - t.rj + 1 : t.jn) : 0;
      float* F = fronts + S.front_off[t.s];
      const float* src = F + min(row, t.N - 1) + int64_t(t.rj) * t.N;
      for (int c = c_lo; c < c_hi; ++c)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                         smem_u32(Cs + c * kTcM + r)),
                     "l"(src + int64_t(c) * t.N)
                     : "memory");
      asm volatile("cp.async.commit_group;" ::: "memory");
      asm volatile("cp.async.wait_all;" ::: "memory");
      for (int pa = 0; pa < t.nacc; ++pa, ++gp) {
        const uint32_t a = gp % kUAcc;
        int got = 1;
        if (lane == 0) got = mbar_wait_ab(&accf[a], (gp / kUAcc) & 1u, abort) ? 1 : 0;
        got = __shfl_sync(0xffffffffu, got, 0);
        if (!got) {
          ok = false;
          bad_s = t.s;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        for (int cb = 0; cb < t.np; cb += 32) {
          uint32_t v[32];
          tmem_ld32(tmem + (uint32_t(quarter * 32) << 16) + a * 128u + uint32_t(cb), v);
#pragma unroll
          for (int c = 0; c < 32; ++c) Cs[(cb + c) * kTcM + r] -= __uint_as_float(v[c]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&accr[a]);
      }
      if (!ok) break;
      float* dst = F + min(row, t.N - 1) + int64_t(t.rj) * t.N;
      for (int c = c_lo; c < c_hi; ++c) dst[int64_t(c) * t.N] = Cs[c * kTcM + r];
    }
  }
  if (!ok && (tid & 31) == 0) flag_timeout(status, bad_s, 0);
  // every MMA has completed before the accumulators are released (MMAs
  // always end, so this wait does not look at the abort word)
  if (warp == 1 && lane == 0 && !mbar_wait1(done, 0)) flag_timeout(status, -1, 0);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) tmem_dealloc(tmem, kUAcc * 128);
}

__global__ void __launch_bounds__(kUThreads, 1)
k_update_tc(DevSym S, const PanelTask* __restrict__ tasks, float* fronts,
            int64_t front_stride, float* dinv, const int64_t* dinv_off, int64_t dinv_stride,
            int bpan, int* status, ImgArgs im, int nspec, int64_t count) {
  pdl_wait();   // launched with launch_pdl: the predecessor's writes first
  pdl_trigger();
  // the bulk copies and the MMA descriptors need 16-byte alignment
  extern __shared__ __align__(128) unsigned char smem_raw[];
  if (nspec >= 0 && int(blockIdx.x) >= nspec) {
    update_persistent(S, tasks, count, nspec, fronts, bpan, status, im, smem_raw);
    return;
  }
  float* Cs = reinterpret_cast<float*>(smem_raw + kUStages * kUStageBytes);   // [col][row]
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kUStages * kUStageBytes + kUTileBytes);
  uint64_t* empty = full + kUStages;
  uint64_t* done = empty + kUStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);

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
  if (tk.t0 < 0) {
    factor_diag<float, kUThreads>(F, N, c0, w, reinterpret_cast<float*>(smem_raw),
                                  Dv + int64_t(tk.p) * kPanel * kPanel, status, s, b);
    return;
  }
  const UpdateRange R = update_range(tk.p, ns, N, bpan);
  const int R0 = base & ~7;
  const int ri = R0 + tk.t0 * kTcM, rj = R0 + tk.t1 * kTcN;
  const bool diag = tk.t0 == tk.t1;
  const int jn = min(kTcN, R.cend - rj);    // tile columns that can be written
  const int np = (jn + 15) & ~15;           // MMA N: a multiple of 16
  const int nst = (base - R.ka + kImgK - 1) / kImgK;
  const int nacc = (base - R.ka + kPanel - 1) / kPanel;

  if (warp == 1) tmem_alloc(tmem_slot, kUAcc * 128);
  if (tid == 0) {
    for (int i = 0; i < kUStages; ++i) {
      mbar_init(&full[i]);
      mbar_init(&empty[i]);
    }
    mbar_init(done);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const float* img = im.img + int64_t(b) * im.stride;
  const int pan0 = im.pan_first[s];
  // the 16 KB chunk of rows row0 .. row0 + 127, K stage st, hi (0) / lo (1)
  auto chunk = [&](int row0, int st, int hl) -> const float* {
    const int kcol = R.ka + kImgK * st;
    const int q = kcol / kPanel;
    const int G = img_groups(q, ns, N);
    const int g0 = (row0 - img_origin(q, ns)) >> 3;
    return img + im.off[pan0 + q] + img_index(G, hl, (kcol % kPanel) / kImgK, g0, 0, 0);
  };

  bool ok = true;
  if (warp == 0) {
    if (lane == 0) {
      const uint32_t bytes = diag ? 2 * kUChunk : 4 * kUChunk;
      int st = 0;
      for (; st < nst; ++st) {
        const int slot = st % kUStages;
        if (st >= kUStages && !mbar_wait1(&empty[slot], uint32_t(st / kUStages - 1) & 1u)) {
          ok = false;
          break;
        }
        unsigned char* dst = smem_raw + slot * kUStageBytes;
        mbar_expect_tx(&full[slot], bytes);
        bulk_g2s(dst, chunk(ri, st, 0), kUChunk, &full[slot]);
        bulk_g2s(dst + kUChunk, chunk(ri, st, 1), kUChunk, &full[slot]);
        if (!diag) {
          bulk_g2s(dst + 2 * kUChunk, chunk(rj, st, 0), kUChunk, &full[slot]);
          bulk_g2s(dst + 3 * kUChunk, chunk(rj, st, 1), kUChunk, &full[slot]);
        }
      }
      // no copy may still be writing this CTA's shared memory at exit: the
      // last stages' copies have landed once their barriers complete
      for (int t = max(0, st - kUStages); t < st; ++t)
        if (!mbar_wait1(&full[t % kUStages], uint32_t(t / kUStages) & 1u)) ok = false;
      if (!ok) flag_timeout(status, s, b);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_tf32(kTcM, np);
      for (int st = 0; st < nst; ++st) {
        const int slot = st % kUStages;
        if (!mbar_wait1(&full[slot], uint32_t(st / kUStages) & 1u)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t ah = smem_u32(smem_raw + slot * kUStageBytes);
        const uint32_t al = ah + kUChunk;
        const uint32_t bh = diag ? ah : ah + 2 * kUChunk;
        const uint32_t bl = diag ? al : ah + 3 * kUChunk;
        const int kcol = R.ka + kImgK * st;
        const uint32_t acc = tmem + uint32_t(((kcol - R.ka) / kPanel) * 128);
#pragma unroll
        for (int kk = 0; kk < kImgK / 8; ++kk) {
          const uint32_t ko = uint32_t(kk) * 2 * kULbo;
          const uint64_t dah = umma_desc(ah + ko, kULbo, kUSbo);
          const uint64_t dal = umma_desc(al + ko, kULbo, kUSbo);
          const uint64_t dbh = umma_desc(bh + ko, kULbo, kUSbo);
          const uint64_t dbl = umma_desc(bl + ko, kULbo, kUSbo);
          const bool fresh = (kcol % kPanel) == 0 && kk == 0;
          umma_tf32(acc, dah, dbh, idesc, fresh ? 0u : 1u);
          umma_tf32(acc, dah, dbl, idesc, 1u);
          umma_tf32(acc, dal, dbh, idesc, 1u);
        }
        umma_commit(&empty[slot]);
      }
      if (!ok) flag_timeout(status, s, b);
      // tracks every MMA issued before it, also after a timeout
      umma_commit(done);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 = tile rows.  The
    // thread's row of the tile is copied into shared memory (cp.async)
    // while the MMAs run, so its read latency hides behind the K loop.
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;
    const int row = ri + r;
    const bool row_ok = row >= base && row < N;
    // column c of the tile is written when in range and, in a diagonal
    // tile, on or below the diagonal
    const int c_lo = max(0, base - rj);
    const int c_hi = row_ok ? min(jn, diag ? row - rj + 1 : jn) : 0;
    const float* src = F + row + int64_t(rj) * N;
    for (int c = c_lo; c < c_hi; ++c)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(Cs + c * kTcM + r)),
                   "l"(src + int64_t(c) * N)
                   : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
    bool got = false;
    if (lane == 0) got = mbar_wait1(done, 0);
    got = __shfl_sync(0xffffffffu, got ? 1 : 0, 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (!got) {
      ok = false;
      if (lane == 0) flag_timeout(status, s, b);
    } else {
      float* dst = F + min(row, N - 1) + int64_t(rj) * N;
      for (int cb = 0; cb < np; cb += 32) {
        float cur[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) cur[c] = Cs[(cb + c) * kTcM + r];
        for (int a = 0; a < nacc; ++a) {
          uint32_t v[32];
          tmem_ld32(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(a * 128 + cb), v);
#pragma unroll
          for (int c = 0; c < 32; ++c) cur[c] -= __uint_as_float(v[c]);
        }
#pragma unroll
        for (int c = 0; c < 32; ++c)
          if (cb + c >= c_lo && cb + c < c_hi) dst[int64_t(cb + c) * N] = cur[c];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
  if (warp == 1) tmem_dealloc(tmem, kUAcc * 128);
  if (all_ok && tk.t0 == 0 && tk.t1 == 0 && base < ns) {
    __syncthreads();   // this CTA's updates of the block are complete
    factor_diag<float, kUThreads>(F, N, base, min(kPanel, ns - base),
                                  reinterpret_cast<float*>(smem_raw),
                                  Dv + int64_t(tk.p + 1) * kPanel * kPanel, status, s, b);
  }
}

}  // namespace

cudaError_t launch_update_tc(dct_plan* P, const PanelTask* tasks, int64_t count, int nspec,
                             cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(k_update_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kUSmem));
  if (e != cudaSuccess) return e;
  dim3 grid(static_cast<unsigned>(count), static_cast<unsigned>(P->nbatch));
  if (nspec >= 0) {
    // one CTA per diagonal task, persistent CTAs on the other multiprocessors
    // (one CTA per SM: shared memory), at most one per remaining tile
    const int64_t pers = std::min<int64_t>(P->sm_count - nspec, count - nspec);
    if (P->nbatch != 1 || pers < 1 || nspec > count) return cudaErrorInvalidValue;
    grid = dim3(static_cast<unsigned>(nspec + pers), 1);
  }
  return launch_pdl(k_update_tc, grid, dim3(kUThreads), kUSmem, st, P->ds, tasks,
                    static_cast<float*>(P->fronts), P->front_stride,
                    static_cast<float*>(P->dinv), P->d_dinv_off, P->dinv_stride,
                    P->update_bpan, P->status, P->img, nspec, count);
}

}  // namespace dct
