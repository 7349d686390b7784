// Float32 substitution products of the large supernodes on the tensor cores.
//
// Each of the four block products of the supernodal substitution is one
// launch kind of the same kernel, D (128 x N) = sum_k A[m, k] B[k, n], with
// the N right-hand sides (<= 256 per CTA) as the MMA's N dimension:
//
//   kFwdLinvTc  y_s   += L_ss^{-1}[rows m, k] b_s[k]        (B <- A rows)
//   kFwdBndTc   b_B   -= L_Bs[rows m, k] y_s[k]             (A rows, gathered)
//   kBwdGemmTc  y_s   -= L_Bs^T[cols m, k] x_B[k]           (B <- gathered A)
//   kBwdLinvTc  x_s   += L_ss^{-T}[cols m, k] y_s[k]        (A <- B rows)
//
// A task covers one 128-row tile of the output and a K range [k0, k1); every
// task adds its product into the destination rows -- one bulk f32 reduction
// per row (cp.reduce.async.bulk) when the rows are 16-byte aligned, float
// atomics otherwise -- so K ranges can be split over tasks, and the
// destination rows of the two inverse products are cleared before the pass
// that writes them (see solve.cu).  tcgen05.mma kind::tf32
// with the 3xTF32 split (hi*hi + hi*lo + lo*hi: Markidis et al. 2018; Ootomo
// and Yokota 2022) accumulates in TMEM.  Operands move in K stages of 16:
// cp.async copies the float32 values of stage i+2 into a two-deep raw ring
// in shared memory while stage i is split into the hi/lo operands and
// multiplied, so the global-memory latency of two stages is hidden without
// holding operands in registers.  256 threads per CTA and about 102 KB of
// shared memory let two CTAs share an SM and overlap each other's fixed
// per-task cost.
#include <cuda_runtime.h>

#include "dct_internal.h"
#include "tc_common.cuh"

namespace dct {
namespace {

constexpr int kStK = 16;                     // K per pipeline stage
#ifndef DCT_TC_RHS
#define DCT_TC_RHS 256
#endif
#ifndef DCT_TC_CTAS_PER_SM
#define DCT_TC_CTAS_PER_SM 2
#endif
constexpr int kStN = DCT_TC_RHS;             // right-hand sides per CTA
constexpr int kNT = 256;                     // threads per CTA
// split A operand (128 x 16), K-major: K-adjacent core matrices 160 B apart,
// so that the transposed converters (2 rows x 16 K per warp instruction) and
// the natural ones (8 rows x 4 K) both store to 32 distinct banks.
constexpr uint32_t kALbo = 160, kASbo = (kStK / 4 - 1) * kALbo + 128;   // 608
constexpr int kABytes = (kTcM / 8) * kASbo;                             // 9728
// split B operand (16 K x 256 N), K-major: N-groups of 8 kBSbo = 528 B apart
// (one 16 B slot of skew per group, so that the scalar stores of a warp that
// holds 8 consecutive float4 along N for 4 rows hit distinct banks)
constexpr uint32_t kBLbo = 128, kBSbo = (kStK / 4) * kBLbo + 16;       // 528
constexpr int kBBytes = (kStN / 8) * kBSbo;                            // 16896
constexpr int kSplitBytes = 2 * kABytes + 2 * kBBytes;
// sets of split operands: with two, stage i is split into one set while the
// MMAs of stage i - 1 still read the other
#ifndef DCT_TC_SPLIT_SETS
#define DCT_TC_SPLIT_SETS 1
#endif
constexpr int kSets = DCT_TC_SPLIT_SETS;
static_assert(kSets == 1 || kSets == 2, "one or two split sets");
// raw float32 stages as copied: A natural [k][m] with rows of kRawAld
// floats, A transposed [m][k] with rows of kStK floats, B [k][n] with rows of
// kRawBld floats (the padding keeps the converters' reads conflict-free)
#ifndef DCT_TC_RAW
#define DCT_TC_RAW 2
#endif
constexpr int kRaw = DCT_TC_RAW;
static_assert(kRaw >= 2 && kRaw <= 3, "two or three raw stages in flight");
constexpr int kRawAld = kTcM + 8;
constexpr int kRawABytes = kStK * kRawAld * 4;
constexpr int kRawBld = kStN + 8;
constexpr int kRawBBytes = kStK * kRawBld * 4;
constexpr int kRawBytes = kRawABytes + kRawBBytes;
constexpr size_t kSolveTcSmem = kSets * size_t(kSplitBytes) + kRaw * size_t(kRawBytes) + 64;
constexpr int kCtasPerSm = DCT_TC_CTAS_PER_SM;
// output rows leave by bulk reductions (1) or float atomics (0)
#ifndef DCT_TC_BULK_REDUCE
#define DCT_TC_BULK_REDUCE 1
#endif
constexpr bool kTcBulkReduce = DCT_TC_BULK_REDUCE != 0;
static_assert(kCtasPerSm * (kSolveTcSmem + 1024) <= 233472, "CTAs per SM");
static_assert(kRawABytes >= kTcM * kStK * 4, "raw A holds both layouts");
static_assert(64 * (kStN + 4) * 4 <= kSets * kSplitBytes + kRaw * kRawBytes,
              "64 staged output rows fit in the operand buffers");
static_assert(kASbo % 16 == 0 && kABytes % 16 == 0 && kBSbo % 16 == 0 &&
                  kBBytes % 16 == 0 && kRawABytes % 16 == 0 && (kRawBld * 4) % 16 == 0,
              "descriptor and copy alignment");

// cp.async of 4 or 16 bytes; src_bytes = 0 fills the destination with zeros
// and reads nothing
__device__ __forceinline__ void cp_async4(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)),
               "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)),
               "l"(src), "r"(src_bytes)
               : "memory");
}

enum TcMode { kModeFwdLinv = 0, kModeFwdBnd, kModeBwdGemm, kModeBwdLinv };

template <int MODE>
__global__ void __launch_bounds__(kNT, kCtasPerSm) k_solve_tc(SolveArgs<float> g) {
  pdl_wait();   // launched with launch_pdl: the predecessor's writes first
  pdl_trigger();
  // a finished refinement: the remaining correction launches do nothing
  if (g.skip != nullptr && *reinterpret_cast<const volatile int*>(g.skip) != 0) return;
  constexpr bool kTrans = MODE == kModeBwdGemm || MODE == kModeBwdLinv;
  constexpr bool kInv = MODE == kModeFwdLinv || MODE == kModeBwdLinv;
  constexpr int kWarps = kNT / 32;
  static_assert(kWarps % 4 == 0, "whole warpgroups: TMEM lane quarters");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // one mbarrier per split set: the commits of the MMAs that read it
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + kSets * kSplitBytes + kRaw * kRawBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + kSets);
  const PanelTask tk = g.tasks[blockIdx.x];
  const int b = blockIdx.y / g.nchunk;
  const int j0 = (blockIdx.y % g.nchunk) * kStN;
  const int kc = min(kStN, g.k - j0);
  const int np = (kc + 15) & ~15;
  const DevSym& S = g.S;
  const int s = tk.s;
  const int N = S.front_n[s], first = S.sn_first[s];
  const int ns = S.sn_first[s + 1] - first;
  const int k0 = tk.p, k1 = tk.t1;
  const int m0 = tk.t0 * kTcM;
  const int32_t* rows = S.rows + S.rows_ptr[s];
  const int mvalid = min(kTcM, (MODE == kModeFwdBnd ? N - ns : ns) - m0);
  // A source: column-major, leading dimension ld; natural A[m][k] =
  // M[(roff + m) + k ld], transposed A[m][k] = M[(roff + k) + (m0 + m) ld]
  const float* M;
  int ld, roff;
  if constexpr (kInv) {
    M = g.linv + int64_t(b) * g.linv_stride + g.linv_off[s];
    ld = ns;
    roff = kTrans ? 0 : m0;
  } else {
    M = g.fronts + int64_t(b) * g.front_stride + S.front_off[s];
    ld = N;
    roff = kTrans ? ns : ns + m0;
  }
  const float* X = (MODE == kModeFwdLinv || MODE == kModeBwdGemm ? g.A : g.B) +
                   int64_t(b) * g.n * g.k;
  float* Y = (MODE == kModeFwdLinv || MODE == kModeBwdGemm ? g.B : g.A) +
             int64_t(b) * g.n * g.k;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) tmem_alloc(tmem_slot, kStN);
  if (tid == 0)
    for (int q = 0; q < kSets; ++q) mbar_init(&mbar[q]);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc_tf32(kTcM, np);
  const int nst = (k1 - k0 + kStK - 1) / kStK;
  bool ok = true;
  constexpr int kPerA = kTcM * kStK / kNT;          // 8 values
  constexpr int kPerB = kStN * kStK / 4 / kNT;      // 4 float4
  const bool vec4 = (g.k & 3) == 0;   // 16-byte aligned rows
  // stage st's float32 values -> raw slot st % kRaw (one commit group)
  auto issue_stage = [&](int st) {
    unsigned char* raw = smem_raw + kSets * kSplitBytes + (st % kRaw) * kRawBytes;
    float* rA = reinterpret_cast<float*>(raw);
    float* rB = reinterpret_cast<float*>(raw + kRawABytes);
    const int kb = k0 + st * kStK;
    const int kw = min(kStK, k1 - kb);
#pragma unroll
    for (int u = 0; u < kPerA; ++u) {
      const int e = tid + u * kNT;
      int m, kl, d;
      if constexpr (kTrans) {
        m = e / kStK;
        kl = e % kStK;
        d = m * kStK + kl;
      } else {
        kl = e / kTcM;
        m = e % kTcM;
        d = kl * kRawAld + m;
      }
      const int kg = kb + kl;
      bool valid = m < mvalid && kl < kw;
      if constexpr (MODE == kModeFwdLinv) valid = valid && kg <= m0 + m;
      if constexpr (MODE == kModeBwdLinv) valid = valid && kg >= m0 + m;
      const int64_t idx = kTrans ? (roff + kg) + int64_t(m0 + m) * ld
                                 : (roff + m) + int64_t(kg) * ld;
      cp_async4(rA + d, valid ? M + idx : M, valid ? 4 : 0);
    }
    if (vec4) {
      // whole 16-byte quads: kc is a multiple of 4 when k is
#pragma unroll
      for (int u = 0; u < kStK * kStN / 4 / kNT; ++u) {
        const int q = tid + u * kNT;
        const int kl = q / (kStN / 4), n = (q % (kStN / 4)) * 4;
        const bool valid = kl < kw && n < kc;
        const float* src = X;
        if (valid) {
          const int kg = kb + kl;
          const int64_t row = MODE == kModeBwdGemm ? int64_t(__ldg(rows + ns + kg))
                                                   : int64_t(first + kg);
          src = X + row * g.k + j0 + n;
        }
        cp_async16(rB + kl * kRawBld + n, src, valid ? 16 : 0);
      }
    } else {
#pragma unroll 4
      for (int u = 0; u < kStK * kStN / kNT; ++u) {
        const int q = tid + u * kNT;
        const int kl = q / kStN, n = q % kStN;
        const bool valid = kl < kw && n < kc;
        const float* src = X;
        if (valid) {
          const int kg = kb + kl;
          const int64_t row = MODE == kModeBwdGemm ? int64_t(__ldg(rows + ns + kg))
                                                   : int64_t(first + kg);
          src = X + row * g.k + j0 + n;
        }
        cp_async4(rB + kl * kRawBld + n, src, valid ? 4 : 0);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // split slots of this thread: A element (m, kl) of slot u; B quad u with
  // rows kl = 4 (chunk / kNc) + lane % 4 and n = 4 (8 (chunk % kNc) + lane / 4)
  constexpr int kNc = kStN / 32;
  auto a_coord = [&](int u, int& m, int& kl) {
    const int gi = warp + u * kWarps;
    if constexpr (kTrans) {
      m = (gi % (kTcM / 2)) * 2 + (lane >> 4);
      kl = (gi / (kTcM / 2)) * 16 + (lane & 15);
    } else {
      m = (gi % (kTcM / 8)) * 8 + (lane >> 2);
      kl = (gi / (kTcM / 8)) * 4 + (lane & 3);
    }
  };
  auto b_coord = [&](int u, int& n, int& kl) {
    const int c = warp + u * kWarps;
    kl = (c / kNc) * 4 + (lane & 3);
    n = ((c % kNc) * 8 + (lane >> 2)) * 4;
  };
  for (int q = 0; q < kRaw && q < nst; ++q) issue_stage(q);
  for (int st = 0; st < nst; ++st) {
    // this thread's copies of stage st have landed (the groups of the
    // stages after it may still be in flight) ...
    const int pend = min(nst, st + kRaw) - st - 1;
    if (pend >= 2)
      asm volatile("cp.async.wait_group 2;" ::: "memory");
    else if (pend == 1)
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    else
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    // ... and everyone's (the barrier), and the MMAs of stage st - kSets,
    // which read this stage's split set, have completed (the set's
    // (st / kSets - 1)-th commit)
    const int set = st % kSets;
    if (st >= kSets) {
      ok = tc_wait(&mbar[set], uint32_t(st / kSets - 1) & 1u, g.status, DCT_ERR_DEVICE_TIMEOUT,
                   s, b);
      if (!ok) break;
    } else {
      __syncthreads();
    }
    unsigned char* Ahi = smem_raw + set * kSplitBytes;
    unsigned char* Alo = Ahi + kABytes;
    unsigned char* Bhi = Alo + kABytes;
    unsigned char* Blo = Bhi + kBBytes;
    const unsigned char* raw = smem_raw + kSets * kSplitBytes + (st % kRaw) * kRawBytes;
    const float* rA = reinterpret_cast<const float*>(raw);
    const float* rB = reinterpret_cast<const float*>(raw + kRawABytes);
    const int kw = min(kStK, k1 - (k0 + st * kStK));
#pragma unroll
    for (int u = 0; u < kPerA; ++u) {
      int m, kl;
      a_coord(u, m, kl);
      const float v = kTrans ? rA[m * kStK + kl] : rA[kl * kRawAld + m];
      tc_store_split(Ahi, Alo,
                     uint32_t(m >> 3) * kASbo + uint32_t(kl >> 2) * kALbo +
                         uint32_t(m & 7) * 16 + uint32_t(kl & 3) * 4,
                     v);
    }
#pragma unroll
    for (int u = 0; u < kPerB; ++u) {
      int n, kl;
      b_coord(u, n, kl);
      if (n < np) {   // columns at or beyond np are never read
        const float4 q4 = *reinterpret_cast<const float4*>(rB + kl * kRawBld + n);
        const float vv[4] = {q4.x, q4.y, q4.z, q4.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int nq = n + q;
          tc_store_split(Bhi, Blo,
                         uint32_t(nq >> 3) * kBSbo + uint32_t(kl >> 2) * kBLbo +
                             uint32_t(nq & 7) * 16 + uint32_t(kl & 3) * 4,
                         vv[q]);
        }
      }
    }
    // after this barrier no thread reads raw slot st % kRaw any more
    tc_publish_smem();
    if (tid == 0) {
      const uint32_t ah = smem_u32(Ahi), al = smem_u32(Alo);
      const uint32_t bh = smem_u32(Bhi), bl = smem_u32(Blo);
      for (int kk = 0; kk < (kw + 7) / 8; ++kk) {
        const uint64_t dah = umma_desc(ah + kk * 2 * kALbo, kALbo, kASbo);
        const uint64_t dal = umma_desc(al + kk * 2 * kALbo, kALbo, kASbo);
        const uint64_t dbh = umma_desc(bh + kk * 2 * kBLbo, kBLbo, kBSbo);
        const uint64_t dbl = umma_desc(bl + kk * 2 * kBLbo, kBLbo, kBSbo);
        umma_tf32(tmem, dah, dbh, idesc, (st > 0 || kk > 0) ? 1u : 0u);
        umma_tf32(tmem, dah, dbl, idesc, 1u);
        umma_tf32(tmem, dal, dbh, idesc, 1u);
      }
      umma_commit(&mbar[set]);
    }
    // the next copies after the MMA issue: gathered rows wait on an index load
    if (st + kRaw < nst) issue_stage(st + kRaw);
  }
  // no copy may still be writing this CTA's shared memory when it exits
  asm volatile("cp.async.wait_all;" ::: "memory");
  // the last commit tracks every MMA issued before it
  if (ok && nst > 0)
    ok = tc_wait(&mbar[(nst - 1) % kSets], uint32_t((nst - 1) / kSets) & 1u, g.status,
                 DCT_ERR_DEVICE_TIMEOUT, s, b);
  const float sgn = kInv ? 1.0f : -1.0f;
  // rows 16-byte aligned and kc a multiple of 4: every output row of the
  // tile goes out as one bulk reduction (cp.reduce.async.bulk .add.f32) from
  // a staging copy in shared memory -- the operand buffers, free once the
  // last MMA has completed -- instead of kc / 4 vector atomics per row.
  const bool bulk = kTcBulkReduce && (g.k & 3) == 0;
  if (ok && nst > 0 && bulk) {
    float* stage = reinterpret_cast<float*>(smem_raw);
    // row stride: a multiple of 4 floats with stride / 4 odd, so that the
    // float4 stores of 8 consecutive rows hit distinct banks
    int ld = (kc + 3) & ~3;
    if (((ld >> 2) & 1) == 0) ld += 4;
    // two rounds of 64 tile rows (TMEM lane quarters 2r and 2r + 1); rounds
    // and quarters wholly beyond the tile's valid rows are skipped
    for (int r = 0; r < 2 && 64 * r < mvalid; ++r) {
      if (((warp & 3) >> 1) == r && (warp & 3) * 32 < mvalid) {
        const int lr = (warp & 1) * 32 + lane;   // staging row
        for (int cb = (warp >> 2) * 32; cb < np; cb += (kWarps / 4) * 32) {
          uint32_t v[32];
          tmem_ld32(tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(cb), v);
#pragma unroll
          for (int c = 0; c < 32; c += 4)
            if (cb + c < kc)
              *reinterpret_cast<float4*>(stage + lr * ld + cb + c) =
                  make_float4(sgn * __uint_as_float(v[c]), sgn * __uint_as_float(v[c + 1]),
                              sgn * __uint_as_float(v[c + 2]), sgn * __uint_as_float(v[c + 3]));
        }
      }
      // generic-proxy stores -> the bulk copy engine, then everyone's rows
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid < 64) {
        const int m = 64 * r + tid;
        if (m < mvalid) {
          const int64_t row = MODE == kModeFwdBnd ? int64_t(rows[ns + m0 + m])
                                                  : int64_t(first + m0 + m);
          asm volatile(
              "cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;" ::"l"(
                  Y + row * g.k + j0),
              "r"(smem_u32(stage + tid * ld)), "r"(uint32_t(kc) * 4u)
              : "memory");
        }
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        // the staging rows are read before they are rewritten or released
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      }
      __syncthreads();
    }
  } else if (ok && nst > 0 && (warp & 3) * 32 < mvalid) {
    const int m = (warp & 3) * 32 + lane;
    float* dst = nullptr;
    if (m < mvalid) {
      const int64_t row = MODE == kModeFwdBnd ? int64_t(rows[ns + m0 + m])
                                              : int64_t(first + m0 + m);
      dst = Y + row * g.k + j0;
    }
    for (int cb = (warp >> 2) * 32; cb < np; cb += (kWarps / 4) * 32) {
      uint32_t v[32];
      tmem_ld32(tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(cb), v);
      if (dst != nullptr) {
#pragma unroll
        for (int c = 0; c < 32; c += 4) {
          if (cb + c + 4 <= kc && (g.k & 3) == 0) {
            atomicAdd(reinterpret_cast<float4*>(dst + cb + c),
                      make_float4(sgn * __uint_as_float(v[c]), sgn * __uint_as_float(v[c + 1]),
                                  sgn * __uint_as_float(v[c + 2]),
                                  sgn * __uint_as_float(v[c + 3])));
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (cb + c + q < kc) atomicAdd(dst + cb + c + q, sgn * __uint_as_float(v[c + q]));
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kStN);
}

}  // namespace

cudaError_t launch_solve_tc(int kind, const SolveArgs<float>& g0, int64_t count,
                            int nbatch, cudaStream_t st) {
  SolveArgs<float> g = g0;
  g.nchunk = (g.k + kStN - 1) / kStN;
  dim3 grid(static_cast<unsigned>(count), static_cast<unsigned>(nbatch * g.nchunk));
  const void* fn = nullptr;
  switch (kind) {
    case kFwdLinvTc: fn = reinterpret_cast<const void*>(k_solve_tc<kModeFwdLinv>); break;
    case kFwdBndTc: fn = reinterpret_cast<const void*>(k_solve_tc<kModeFwdBnd>); break;
    case kBwdGemmTc: fn = reinterpret_cast<const void*>(k_solve_tc<kModeBwdGemm>); break;
    case kBwdLinvTc: fn = reinterpret_cast<const void*>(k_solve_tc<kModeBwdLinv>); break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kSolveTcSmem));
  if (e != cudaSuccess) return e;
  switch (kind) {
    case kFwdLinvTc: return launch_pdl(k_solve_tc<kModeFwdLinv>, grid, dim3(kNT), kSolveTcSmem, st, g);
    case kFwdBndTc: return launch_pdl(k_solve_tc<kModeFwdBnd>, grid, dim3(kNT), kSolveTcSmem, st, g);
    case kBwdGemmTc: return launch_pdl(k_solve_tc<kModeBwdGemm>, grid, dim3(kNT), kSolveTcSmem, st, g);
    default: return launch_pdl(k_solve_tc<kModeBwdLinv>, grid, dim3(kNT), kSolveTcSmem, st, g);
  }
}

}  // namespace dct
