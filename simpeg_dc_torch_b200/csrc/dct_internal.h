// Internal declarations shared by the CUDA translation units of libdct.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/dct.h"
#include "cplx.cuh"
#include "symbolic.h"

namespace dct {

// Refinement state of one float32 solve, in device memory.  Iteration i adds
// the correction c_i to x; its size rho_i = max|c_i| / max|x_i| estimates the
// error of x_{i-1}, and rho_i * min(1, rho_i / rho_{i-1}) (rho_1^2 for the
// first) that of x_i.  `done` is set once the estimate is below the plan's
// tolerance, on stagnation (rho_i > rho_{i-1} / 2) or after the last allowed
// iteration; kernels of later correction solves then return at entry.
constexpr int kIrHistory = 16;
struct IrState {
  int done;                       // 1: no further corrections
  int iters;                      // corrections applied after the first solve
  int converged;                  // 1: estimate below the tolerance
  int pad;
  unsigned long long cmax, xmax;  // max|c|, max|x| of the last update (bits)
  unsigned long long rmax, bmax;  // max|b - A x|, max|b| of the last residual
  double est;                     // estimated relative error of x
  double rho[kIrHistory];         // rho_1 .. rho_iters
};

// Device copy of the symbolic structure (plain pointers, passed by value).
struct DevSym {
  const int32_t* sn_first;
  const int32_t* front_n;
  const int64_t* front_off;
  const int64_t* rows_ptr;
  const int32_t* rows;
  const int64_t* amap_ptr;
  const int32_t* amap_e;
  const int32_t* amap_pos;
  const int32_t* child_ptr;
  const int32_t* child;
  const int64_t* rel_ptr;
  const int32_t* rel;
  const int32_t* perm;
  const int32_t* iperm;
  const int32_t* crow;   // input pattern (refinement residuals)
  const int32_t* col;
};

// One launch of a factor or solve schedule: `count` tasks from `first`.
struct Launch {
  int kind;
  int level;
  int64_t first;
  int64_t count;
  int arg;         // small fronts: largest front order of the launch;
                   // panel steps: the panel; supernode inverses: the block
                   // width
};

enum LaunchKind : int {
  kSmallFront = 0,   // fused assemble + partial Cholesky, one CTA per front
  kLargeScatter,     // matrix entries into large fronts
  kLargeExtendAdd,   // one child slot into large fronts
  kLargePanel,       // TRSM of the rows below a factored diagonal block
  kLargeUpdate,      // trailing symmetric update tiles (+ next diagonal block)
  kPanelInverse,     // inverses of the diagonal blocks of single-CTA fronts
  kLinvInit,         // supernode inverses: diagonal 64-blocks from the panels
  kLinvT,            // supernode inverses, doubling step T = C A^{-1}
  kLinvX,            // supernode inverses, doubling step X = -D^{-1} T
  kFwdSmall,         // forward substitution of single-panel supernodes
  kFwdLinv,          // forward: y_s = L_ss^{-1} b_s, large supernodes (f64)
  kFwdBnd,           // forward: boundary rows -= L_Bs y_s (f64)
  kBwdSmall,         // backward substitution of single-panel supernodes
  kBwdGemm,          // backward: y_s -= L_Bs^T x_B (f64)
  kBwdLinv,          // backward: x_s = L_ss^{-T} y_s (f64)
  kFwdLinvTc,        // the four products above on tensor cores (f32),
  kFwdBndTc,         //   128-row output tiles, split K ranges
  kBwdGemmTc,
  kBwdLinvTc,
  kNumKinds
};

// Limits of the single-CTA front kernel (front fully in shared memory).
constexpr int kSmallFrontF64 = 160;
constexpr int kSmallFrontF32 = 224;
constexpr int kSmallFrontC128 = 112;
constexpr int kThreads = 256;
constexpr int kRhsChunk = 64;   // right-hand sides per CTA in the solves
constexpr int kUpdateTile = 64;   // trailing-update tile (rows = cols)
// float32 fronts group their panels in blocks of this many for the trailing
// update (see update_range); float64 fronts update after every panel
#ifndef DCT_UPDATE_BLOCK_PANELS
#define DCT_UPDATE_BLOCK_PANELS 4
#endif
constexpr int kUpdateBlockPanels = DCT_UPDATE_BLOCK_PANELS;

// Column ranges of the trailing update that follows panel p of a supernode
// with ns columns (front order N) when the panels are grouped in blocks of
// bpan (LAPACK-style blocked right-looking Cholesky with an inner panel
// loop): the last panel of a block, or of the supernode, updates the whole
// trailing block, columns [base, N), with all of the block's panels as K
// (columns [ka, base)); any other panel updates only the remaining columns
// of its own block, [base, cend), with its own kPanel columns.  base = the
// first column after panel p.  bpan = 1 is the plain right-looking update.
struct UpdateRange {
  int ka, cend;
};
__host__ __device__ inline UpdateRange update_range(int p, int ns, int N, int bpan) {
  const int npan = (ns + kPanel - 1) / kPanel;
  const int blk = p / bpan;
  const bool last = (p % bpan == bpan - 1) || (p == npan - 1);
  UpdateRange r;
  r.ka = (last ? blk * bpan : p) * kPanel;
  const int bend = (blk + 1) * bpan * kPanel;
  r.cend = last ? N : (bend < ns ? bend : ns);
  return r;
}

// Split images of the factor panels of large float32 fronts, the operands of
// the tensor-core trailing update (update_tc.cu).  Panel q of a supernode
// (columns c0 = 64 q .. c0 + w) has an image of the rows from
// R0 = c0 + (w & ~7) (8-aligned, at most 7 rows above the first row below
// the panel) down to the front's last row, in groups of 8 rows, plus 16
// groups of zero padding so that any 128-row window that starts below the
// front's last row lies inside it.  Each element is stored twice, hi =
// tf32(x) and lo = x - hi, in the tensor cores' K-major layout without
// swizzle: [hl][K stage of kImgK columns][8-row group][K core of 4][row of 8]
// [column of 4] floats, so 128 rows x kImgK columns of one of hi/lo are
// 128 * kImgK * 4 bytes contiguous (16 KB for 32 columns; core matrices
// 128 B apart along K, 8-row groups 32 * kImgK bytes apart).  The stage
// width is the K depth of one bulk copy of the trailing update.
#ifndef DCT_IMG_K
#define DCT_IMG_K 32
#endif
constexpr int kImgK = DCT_IMG_K;
static_assert(kImgK % 8 == 0 && kPanel % kImgK == 0, "image stages: 8 .. 64 columns");
__host__ __device__ inline int img_origin(int q, int ns) {
  const int c0 = q * kPanel;
  const int w = ns - c0 < kPanel ? ns - c0 : kPanel;
  return c0 + (w & ~7);
}
__host__ __device__ inline int img_groups(int q, int ns, int N) {
  return (N - img_origin(q, ns) + 7) / 8 + 16;
}
// float offset of (hl, K stage, group g, column k of the stage, row r8 of the
// group) in a panel image of G groups
__host__ __device__ inline int64_t img_index(int G, int hl, int stage, int g, int k, int r8) {
  return (int64_t(hl * (kPanel / kImgK) + stage) * G + g) * (8 * kImgK) + (k >> 2) * 32 +
         r8 * 4 + (k & 3);
}
// floats of one panel image of G groups (hi and lo, all stages)
__host__ __device__ inline int64_t img_floats(int G) { return int64_t(2) * kPanel * 8 * G; }
struct ImgArgs {
  float* img;                // nbatch * stride floats
  const int64_t* off;        // per panel (pan_first[s] + q): first float
  const int32_t* pan_first;  // per supernode: index of its first panel
  int64_t stride;            // floats per system
};

// Programmatic dependent launch for the long chains of dependent launches
// (panel TRSM <-> trailing update, the substitution products): a kernel
// launched with launch_pdl may be scheduled while its predecessor in the
// stream is still running, so it must call pdl_wait() before it touches
// memory that earlier work writes; pdl_trigger() lets this kernel's own
// successor be scheduled early.  Without the attribute both are no-ops.
#ifndef DCT_PDL
#define DCT_PDL 1
#endif
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = DCT_PDL ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

struct Schedule {
  std::vector<PanelTask> tasks;    // host copy
  PanelTask* d_tasks = nullptr;    // device copy
  std::vector<Launch> launches;
  // per launch, algorithmic work: factor launches give absolute flops and
  // bytes; solve launches give flops per right-hand side, bytes that do not
  // depend on k (factor reads) and bytes per right-hand side
  std::vector<double> flops;
  std::vector<double> bytes;
  std::vector<double> bytes_rhs;
};

// Optional per-launch event timing (dct_plan_profile).
struct Profiler {
  bool on = false;
  struct Rec {
    int kind;
    cudaEvent_t a, b;
    double flops, bytes;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  double ms[kNumKinds] = {0}, fl[kNumKinds] = {0}, by[kNumKinds] = {0};
  int64_t n[kNumKinds] = {0};
  std::vector<int> log_kind;     // every collected launch, in launch order
  std::vector<double> log_ms;
  cudaError_t begin(int kind, double flops, double bytes, cudaStream_t st);
  cudaError_t end(cudaStream_t st);
  cudaError_t collect();
  void reset();
};

}  // namespace dct

// The plan object behind the opaque handle of the C ABI.
struct dct_plan {
  dct::Symbolic sym;
  int device = 0;
  int nbatch = 1;
  int max_rhs = 1;
  int dtype = DCT_F64;             // factor / solve precision
  dct::DevSym ds{};
  std::vector<void*> owned;        // device allocations
  void* fronts = nullptr;          // nbatch * front_total elements of dtype
  int64_t front_stride = 0;
  dct::Schedule fact;              // factorization schedule
  dct::Schedule fwd;               // forward substitution schedule
  dct::Schedule bwd;               // backward substitution schedule
  dct::Schedule inv;               // diagonal-block inverses (one launch)
  void* dinv = nullptr;            // nbatch * dinv_stride elements of dtype
  int64_t dinv_stride = 0;         // per system: sum over panels of w^2
  const int64_t* d_dinv_off = nullptr;   // per supernode, first panel inverse
  dct::Schedule linv_sched;        // supernode-inverse doubling launches
  void* linv = nullptr;            // nbatch * linv_stride: L_ss^{-1}, ns x ns (ld ns)
  void* ltmp = nullptr;            // same size: doubling-step products
  int64_t linv_stride = 0;
  const int64_t* d_linv_off = nullptr;   // per supernode (-1 for one-panel ones)
  void* bufA = nullptr;            // dtype, nbatch*n*max_rhs (work buffer A)
  void* bufB = nullptr;            // dtype, nbatch*n*max_rhs (work buffer B)
  double* x64 = nullptr;           // f32 plans: refined solution (dct_solve)
  double* b64 = nullptr;           // f32 plans: permuted rhs (dct_solve)
  double* vals64 = nullptr;        // f32 plans: float64 values (residuals)
  int* status = nullptr;           // device: code, supernode, system
  unsigned long long* resid_bits = nullptr;  // device: max|r|, max|b|
  int factored = 0;
  int64_t stamp = 0;
  dct::ImgArgs img{};              // f32 plans: split panel images (large fronts)
  dct_tuning tune{};               // schedule shapes (resolved, no zero fields)
  int ir_iters = 2;                // most refinement iterations of f32 plans
  double ir_tol = 0.0;             // stop once the estimated error is below (0: fixed count)
  dct::IrState* ir = nullptr;      // device: refinement state of the last solve
  int update_bpan = 1;             // panels per trailing-update block
  int sm_count = 148;              // multiprocessors of the plan's device
  // per factor launch: for float32 trailing updates that run persistent CTAs,
  // the number of diagonal tasks moved to the front of the launch's tasks
  // (one CTA each); -1: one CTA per task
  std::vector<int32_t> update_nspec;
  dct::Profiler prof;
  // general (unsymmetric-valued) float64 plans, factored P A P^T = L U with
  // static pivoting: `fronts` holds L (unit diagonal) in the lower part,
  // `fronts2` holds U^T in the lower part, both with the same layout; the
  // inverses of L's diagonal blocks go to dinv / linv, those of U^T's to
  // dinv2 / linv2.  d_tr maps every pattern entry (i, j) to the entry (j, i).
  int lu = 0;
  void* fronts2 = nullptr;
  void* dinv2 = nullptr;
  void* linv2 = nullptr;
  const int32_t* d_tr = nullptr;
  double pivot_floor = 0.0;        // relative static-pivot threshold (x max|block|)
};

struct dct_symbolic {
  dct::Symbolic sym;
};

namespace dct {
// arguments of the substitution kernels (solve.cu, solve_tc.cu)
template <typename T>
struct SolveArgs {
  DevSym S;
  const PanelTask* tasks;
  const T* fronts;
  int64_t front_stride;
  const T* dinv;
  const int64_t* dinv_off;
  int64_t dinv_stride;
  T* A;
  T* B;
  int n, k, nchunk;
  int* status;
  const T* linv;
  const int64_t* linv_off;
  int64_t linv_stride;
  // float32 plans: refinement state; a set `done` word makes every kernel of
  // the remaining correction solves return at entry (null: never skip)
  const int* skip;
};
// one launch of a tensor-core substitution kind (kFwdLinvTc .. kBwdLinvTc)
cudaError_t launch_solve_tc(int kind, const SolveArgs<float>& g, int64_t count,
                            int nbatch, cudaStream_t st);
// one launch of the float32 trailing update (update_tc.cu); nspec >= 0:
// the first nspec tasks take one CTA each and persistent CTAs on the
// remaining multiprocessors share the others, nspec = -1: one CTA per task
cudaError_t launch_update_tc(dct_plan* P, const PanelTask* tasks, int64_t count, int nspec,
                             cudaStream_t st);
// records the message returned by dct_last_error() for this thread
void set_last_error(const char* msg);
cudaError_t run_factor(dct_plan* P, const void* vals, int vals_dtype,
                       int64_t vals_stride, cudaStream_t st);
cudaError_t run_solve_f64(dct_plan* P, double* xa, int k, cudaStream_t st,
                          bool transposed = false);
cudaError_t run_solve_f32(dct_plan* P, int k, cudaStream_t st);
// complex128 plans: the permuted right-hand side in xa (solution left there)
cudaError_t run_solve_c128(dct_plan* P, cplx* xa, int k, cudaStream_t st);
cudaError_t launch_perm_in_any(const void* b, int b_dtype, int64_t bstride,
                               const int32_t* perm, int n, int k, int nbatch,
                               void* dst, int dst_dtype, cudaStream_t st);
cudaError_t launch_perm_out_any(const void* src, int src_dtype,
                                const int32_t* perm, int n, int k, int nbatch,
                                void* x, int x_dtype, cudaStream_t st);
cudaError_t launch_convert_any(const void* src, int src_dtype, int64_t sstride,
                               int64_t count, int nbatch, void* dst,
                               int dst_dtype, cudaStream_t st);
cudaError_t launch_residual(dct_plan* P, const double* b, int64_t bstride,
                            const double* x, int k, cudaStream_t st);
cudaError_t launch_ir_update(dct_plan* P, double* x, int k, int first,
                             cudaStream_t st);
// decides after correction `iter` (1-based) whether to stop refining
cudaError_t launch_ir_decide(dct_plan* P, int iter, cudaStream_t st);
}  // namespace dct
