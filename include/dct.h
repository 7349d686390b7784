/*
 * dct.h -- C ABI of libdct, the B200 (sm_100a) sparse direct solver and DC
 * forward/adjoint kernels behind simpeg_dc_torch_b200.
 *
 * Conventions
 *   - Every entry point returns an int status (DCT_OK = 0).  On failure
 *     dct_last_error() returns a message for the calling thread.  No C++
 *     exception and no device trap crosses this boundary.
 *   - Pointers named d_* are device pointers on the plan's device; all other
 *     pointers are host pointers.  `stream` is a cudaStream_t (NULL = legacy
 *     default stream); work is enqueued asynchronously on it.
 *   - Dense right-hand sides are row-major (n, k) per system, k contiguous,
 *     the layout of a torch (n, k) tensor; batched ones are (nbatch, n, k).
 *   - "Permuted" buffers hold rows in the solver's elimination order
 *     (row i of the permuted buffer is row perm[i] of the user's ordering).
 *
 * Each declaration names the reference interface it replaces
 * (eacuellarq/SimPEG_DC_Torch, dctorch 0.2.0, path:line).
 */
#ifndef DCT_H
#define DCT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* value types: float64, float32, and complex128 (two doubles re, im; the
 * complex-symmetric systems of the complex-resistivity engine) */
enum { DCT_F64 = 0, DCT_F32 = 1, DCT_C128 = 2 };

enum {
  DCT_OK = 0,
  DCT_ERR_ARG = 1,              /* invalid argument */
  DCT_ERR_CUDA = 2,             /* a CUDA runtime call failed */
  DCT_ERR_OOM = 3,              /* device allocation failed */
  DCT_ERR_ZERO_PIVOT = 4,       /* non-positive pivot: matrix not SPD */
  DCT_ERR_IR_NOT_CONVERGED = 5, /* refinement residual above tolerance */
  DCT_ERR_BAD_PATTERN = 6,      /* pattern rejected by the analysis */
  DCT_ERR_NOT_FACTORED = 7,     /* solve before factorize */
  DCT_ERR_NO_DEVICE = 8,        /* no usable CUDA device */
  DCT_ERR_DEVICE_TIMEOUT = 9    /* a bounded on-device wait gave up */
};

typedef struct dct_symbolic dct_symbolic;
typedef struct dct_plan dct_plan;

typedef struct {
  int64_t n;             /* unknowns */
  int64_t nnz_in;        /* entries of the input pattern */
  int64_t nsuper;        /* supernodes (dense fronts) */
  int64_t nlevels;       /* levels of the assembly tree */
  int64_t max_front;     /* largest front order */
  int64_t max_ns;        /* largest supernode (pivot columns) */
  int64_t nnz_L;         /* stored factor entries, explicit zeros included */
  int64_t front_total;   /* front storage per system, in elements */
  double flops_factor;   /* dense flops of one numeric factorization */
} dct_symbolic_info;

int dct_version(void);
const char* dct_last_error(void);

/* ---- symbolic analysis (host only; no GPU needed) ------------------------
 * Nested-dissection ordering, assembly tree and front maps of a structurally
 * symmetric CSR pattern (int32 crow[n+1], col[nnz]).  coords (n x ndim
 * int32, may be NULL) are grid coordinates for geometric bisection.
 * Replaces the reordering + symbolic phase of DirectSolver(...).plan()
 * (dctorch/solver.py:103-109, 204-207). */
int dct_symbolic_create(int32_t n, const int32_t* crow, const int32_t* col,
                        const int32_t* coords, int32_t ndim, int32_t leaf_size,
                        dct_symbolic** out);
void dct_symbolic_destroy(dct_symbolic* sym);
int dct_symbolic_get_info(const dct_symbolic* sym, dct_symbolic_info* out);
/* Copies a named int32/int64 array of the analysis (perm, iperm, sn_first,
 * sn_parent, sn_level, front_n, front_off, rows_ptr, rows, child_ptr, child,
 * rel_ptr, rel, amap_ptr, amap_e, amap_pos) into dst.  With dst NULL only
 * *size_bytes is set. */
int dct_symbolic_get_array(const dct_symbolic* sym, const char* name,
                           void* dst, int64_t capacity_bytes,
                           int64_t* size_bytes);

/* Host-side copy of the launch schedule a plan of this dtype would run
 * (which: 0 factorization, 1 forward, 2 backward substitution, 3 panel
 * inverses, 4 supernode inverses), for
 * inspection and CPU-side replay in tests.  tasks: 4 int32 per task
 * (supernode, panel or K start, t0, t1 or K end); launches: 5 int64 per launch (kind, level,
 * first task, task count, arg).  With null outputs only the counts are set. */
int dct_symbolic_get_schedule(const dct_symbolic* sym, int32_t dtype,
                              int32_t which, int32_t* tasks, int64_t* ntasks,
                              int64_t* launches, int64_t* nlaunches);

/* ---- numeric plan: nbatch systems on one pattern, on one device -----------
 * dtype DCT_F64: plain float64 factor and solve.
 * dtype DCT_F32: float32 factor and solve, with iterative refinement whose
 *                residual b - A x is formed in float64.
 * dtype DCT_C128: complex-symmetric (A^T = A, not Hermitian) A = L L^T
 *                without conjugation, complex128 values and right-hand
 *                sides (dct_factorize / dct_solve with DCT_C128 buffers;
 *                dct_solve_permuted is float64 only).  Replaces cuDSS's
 *                "symmetric" matrix type (dctorch/solver.py:44-47,
 *                377-380) behind the complex-resistivity engine.
 * Replaces CuDSSSolver.__init__ (dctorch/solver.py:88-114) and
 * CuDSSBatchSolver.__init__ (dctorch/solver.py:187-213). */
int dct_plan_create(const dct_symbolic* sym, int32_t nbatch, int32_t max_rhs,
                    int32_t dtype, int32_t device, dct_plan** out);

/* Schedule shapes a plan is built with (the front tiles of its launches);
 * dct_tuning_default fills the measured defaults of the dtype.  Any field
 * <= 0 takes its default.
 *   small_front_max   largest front factored by one CTA in shared memory
 *                     (32 .. 224 float32, 32 .. 160 float64); larger fronts
 *                     take the panel / trailing-update path
 *   update_block      panels per block of the float32 trailing update (1..4;
 *                     the deferred update after a block has K = 64 x this)
 *   solve_target      float32 substitution: fewest tasks a launch is split
 *                     into (K ranges halved until reached)
 *   solve_split_max   float32 substitution: longest K piece of one task
 *   solve_split_min   float32 substitution: shortest K piece
 *   small_tc          single-panel supernodes on the tensor-core products:
 *                     1 yes, 2 no (CUDA-core one-CTA kernels), <= 0 decided
 *                     from where their work lies
 * The tuner of the Python package (simpeg_dc_torch_b200/tuning.py) times
 * candidate plans and keeps the fastest.  No counterpart in the reference:
 * cuDSS chooses its own (dctorch/solver.py:103-109). */
typedef struct {
  int32_t small_front_max;
  int32_t update_block;
  int32_t solve_target;
  int32_t solve_split_max;
  int32_t solve_split_min;
  int32_t small_tc;
} dct_tuning;
int dct_tuning_default(int32_t dtype, dct_tuning* out);
int dct_plan_create_tuned(const dct_symbolic* sym, int32_t nbatch, int32_t max_rhs,
                          int32_t dtype, int32_t device, const dct_tuning* tuning,
                          dct_plan** out);
/* the tuning a plan was built with (defaults resolved) */
int dct_plan_get_tuning(const dct_plan* plan, dct_tuning* out);
void dct_plan_destroy(dct_plan* plan);
/* Iterative refinement of float32 plans (no effect on float64 plans):
 * at most `iterations` corrections (default 2, at most 64) after the first
 * solve; each correction i adds c_i = A_32^{-1} (b - A x) with the residual
 * formed in float64.  rho_i = max|c_i| / max|x_i| estimates the relative
 * error of the previous iterate, so rho_i * min(1, rho_i / rho_{i-1})
 * (rho_1^2 for the first) estimates that of x_i.  With tol > 0 refinement
 * stops once that estimate is <= tol, and when the corrections stagnate
 * (rho_i > rho_{i-1} / 2) or the iterations run out above tol, the plan's
 * status words record DCT_ERR_IR_NOT_CONVERGED (read by dct_check_status,
 * `where` = -1).  tol = 0 (the default) runs the fixed number of
 * corrections, ending early only at a stall or at float64 rounding.  A NaN
 * correction is always recorded as DCT_ERR_IR_NOT_CONVERGED.  The decision is taken on the device: the
 * launches of corrections that are not needed return at entry and the host
 * never waits.  Replaces the fixed precision of CuDSSSolver's float32 solves
 * (dctorch/solver.py:122-135), which has no refinement. */
int dct_plan_set_refinement(dct_plan* plan, int32_t iterations);
int dct_plan_set_refinement_tolerance(dct_plan* plan, double tol);
/* The refinement record of the plan's last float32 solve (synchronises the
 * stream): corrections applied, whether the estimate reached the tolerance,
 * the estimated relative error and rho_1 .. rho_iters (first min(capacity,
 * iters, 16) of them). */
int dct_plan_refinement_info(dct_plan* plan, void* stream, int32_t* iters,
                             int32_t* converged, double* est_error, double* rho,
                             int32_t capacity);
/* device pointer to the plan's iperm (int32, n): user row -> permuted row */
int dct_plan_iperm(const dct_plan* plan, const int32_t** d_iperm);
/* bumped by every factorization (dctorch/solver.py:211-213, 221) */
int64_t dct_plan_stamp(const dct_plan* plan);

/* Numeric factorization of every system from its CSR values.
 * d_vals: nbatch rows of nnz values, row b at d_vals + b*vals_batch_stride,
 * float64 or float32 (vals_dtype).  Replaces CuDSSSolver.factorize
 * (dctorch/solver.py:116-120) and CuDSSBatchSolver.factorize (215-221). */
int dct_factorize(dct_plan* plan, const void* d_vals, int32_t vals_dtype,
                  int64_t vals_batch_stride, void* stream);

/* Solve every system for k <= max_rhs right-hand sides in the user's row
 * order.  d_b: (n, k) shared by all systems (b_batched = 0) or
 * (nbatch, n, k); d_x: (nbatch, n, k).  io_dtype gives the type of both.
 * Replaces CuDSSSolver.solve (dctorch/solver.py:122-135) and
 * CuDSSBatchSolver.solve (dctorch/solver.py:223-230). */
int dct_solve(dct_plan* plan, const void* d_b, int32_t io_dtype,
              int32_t b_batched, int32_t k, void* d_x, void* stream);

/* The same solve on float64 buffers already in permuted order:
 * d_bp (n, k) shared or (nbatch, n, k); d_xp (nbatch, n, k).  d_bp may alias
 * d_xp only when batched and only in float64 plans (a float32 plan forms its
 * refinement residuals from d_bp).  Used by the fused engine paths. */
int dct_solve_permuted(dct_plan* plan, const double* d_bp, int32_t b_batched,
                       int32_t k, double* d_xp, void* stream);

/* Per-launch-kind timing with CUDA events on the launch stream (off by
 * default).  While enabled, every factor/solve launch is bracketed by events;
 * dct_plan_profile_get synchronises and returns, for one launch kind
 * (0 small fronts, 1 large scatter, 2 extend-add, 3 panel TRSM, 4 trailing
 * update, 5 panel inverses, 6-8 supernode-inverse steps, 9 forward of
 * single-panel supernodes, 10 forward inverse products, 11 forward boundary
 * rows, 12 backward of single-panel supernodes, 13 backward boundary
 * product, 14 backward inverse products, 15-18 the products of 10, 11, 13
 * and 14 on tensor cores in float32 plans), the summed
 * device milliseconds, the launch count and the algorithmic flops and bytes
 * of those launches; reset clears the counters. */
int dct_plan_profile(dct_plan* plan, int32_t enable, int32_t reset);
int dct_plan_profile_get(dct_plan* plan, int32_t kind, double* ms,
                         int64_t* launches, double* flops, double* bytes);
/* The profiled launches one by one, in launch order since the last reset:
 * kind and device milliseconds of the first min(capacity, *count). */
int dct_plan_profile_log(dct_plan* plan, int64_t capacity, int32_t* kinds,
                         double* ms, int64_t* count);

/* Reads the device status words (synchronises the stream): the first error
 * code raised by a kernel since the last call, the supernode where it was
 * raised (or -1) and the last refinement residual ratio max|b-Ax|/max|b|. */
int dct_check_status(dct_plan* plan, void* stream, int32_t* code,
                     int32_t* where, double* residual);

/* ---- fused engine kernels (stateless; float64) ---------------------------- */

/* sigma = exp(-m) (nC) and vals = L sigma for a CSR L with nrows rows
 * (int64 row pointers).  Replaces the value build of TorchDC2D.dpred /
 * TorchDC3D.dpred: torch.sparse.mm(Lstack, exp(-m)) (dctorch/
 * simulation2d.py:391-392, simulation3d.py:203-204). */
int dct_sigma_values(int64_t nrows, const int64_t* d_L_ptr,
                     const int32_t* d_L_col, const double* d_L_val,
                     int64_t nC, const double* d_m, double* d_sigma,
                     double* d_vals, void* stream);

/* gm = -sigma * (Lt gv): the vjp of vals = L exp(-m), with Lt the CSR of L^T
 * (nC rows).  Replaces the autograd backward of torch.sparse.mm(Lstack, .)
 * and of exp (dctorch/simulation2d.py:391-392; simulation3d.py:25-41). */
int dct_values_vjp(int64_t nC, const int64_t* d_Lt_ptr, const int32_t* d_Lt_col,
                   const double* d_Lt_val, const double* d_sigma,
                   const double* d_gv, double* d_gm, void* stream);

/* dst(n, k) = 0, then dst[row[p]*k + src[p]] = sum over q in [ptr[p],
 * ptr[p+1]) of coef[q] * (d_g ? g[datum[q]] : 1).  Builds the permuted source
 * right-hand side (q, dctorch/simulation2d.py:231-234, 325-328) and the
 * adjoint right-hand side Pd^T G (the vjp of the projection/gather,
 * dctorch/simulation2d.py:395). */
int dct_scatter_rhs(int64_t n, int32_t k, int64_t npairs, const int64_t* d_ptr,
                    const int32_t* d_row, const int32_t* d_src,
                    const int32_t* d_datum, const double* d_coef,
                    const double* d_g, double* d_dst, void* stream);

/* d[i] = sum_b w[b] sum_{j in Pd row i} Pd[i,j] X[b, iperm[j], sidx[i]]:
 * wavenumber quadrature sum + receiver projection + per-datum source
 * gather, fused (dctorch/simulation2d.py:394-395; simulation3d.py:206).
 * X permuted (nbatch, n, k); d_w may be NULL (all ones). */
int dct_project_data(int32_t nbatch, int64_t n, int32_t k, int64_t nD,
                     const int32_t* d_Pd_ptr, const int32_t* d_Pd_col,
                     const double* d_Pd_val, const int32_t* d_sidx,
                     const int32_t* d_iperm, const double* d_w,
                     const double* d_X, double* d_out, void* stream);

/* gv[b, e] = -scale[b] * sum_r Y[b, iperm[row_e], r] X[b, iperm[col_e], r]:
 * the value gradient of the batched solve on the pattern
 * (dctorch/solver.py:268-276 with the quadrature weight of
 * simulation2d.py:394 folded in).  X, Y permuted (nbatch, n, k);
 * d_scale may be NULL (all ones). */
int dct_gather_contract(int32_t nbatch, int64_t n, int64_t nnz, int32_t k,
                        const int32_t* d_row, const int32_t* d_col,
                        const int32_t* d_iperm, const double* d_scale,
                        const double* d_Y, const double* d_X, double* d_gv,
                        void* stream);

/* Same contraction in the user's row order and dtype (DCT_F64, DCT_F32 or
 * DCT_C128, complex without conjugation), for the solver-level autograd op:
 * gv[b,e] = -sum_r Y[b,row_e,r] X[b,col_e,r] (dctorch/solver.py:160-170,
 * 268-276). */
int dct_gather_contract_plain(int32_t nbatch, int64_t n, int64_t nnz, int32_t k,
                              const int32_t* d_row, const int32_t* d_col,
                              int32_t dtype, const void* d_Y, const void* d_X,
                              void* d_gv, void* stream);

/* ---- linearised products of the 2.5-D engine (float64) ------------------- */

/* y = M x for a CSR matrix with int64 row pointers: the value perturbation
 * dvals = L (-sigma v) of a Jacobian-vector product.  Replaces
 * torch.sparse.mm(eng.Lstack, ...) in Linearization2D.Jvec
 * (dctorch/simulation2d.py:692-694). */
int dct_csr_spmv(int64_t nrows, const int64_t* d_ptr, const int32_t* d_col,
                 const double* d_val, const double* d_x, double* d_y, void* stream);

/* Y_b[iperm[i], :] = alpha * sum_e vals_b[e] X_b[iperm[col_e], :] over row i
 * of the pattern (crow/col in user order, X/Y permuted (nbatch, n, k),
 * X != Y): the right-hand sides -A_k(dvals) U_k.  Replaces the per-ky CSR
 * products of Linearization2D.Jvec (dctorch/simulation2d.py:697-703). */
int dct_pattern_spmm(int32_t nbatch, int32_t n, int32_t k, const int32_t* d_crow,
                     const int32_t* d_col, const int32_t* d_iperm, const double* d_vals,
                     int64_t nnz, double alpha, const double* d_X, double* d_Y,
                     void* stream);

/* gv[(b*nnz + e)*nb + r] = -scale[b] Y_b[iperm row_e, r] U_b[iperm col_e, sidx[r]]:
 * one adjoint column per datum contracted with that datum's own source field
 * (Y permuted (nbatch, n, nb), U permuted (nbatch, n, ns)).  Replaces the
 * per-ky gathers of TorchDC2D.Jmatrix (dctorch/simulation2d.py:502-505) and
 * Linearization2D._grad_vals_pairwise (808-818). */
int dct_gather_pairwise(int32_t nbatch, int64_t n, int64_t nnz, int32_t nb, int32_t ns,
                        const int32_t* d_row, const int32_t* d_col,
                        const int32_t* d_iperm, const double* d_scale,
                        const int32_t* d_sidx, const double* d_Y, const double* d_U,
                        double* d_gv, void* stream);

/* out[c, r] = -sigma[c] sum_q Lt_val[q] gv[Lt_col[q], r] for nb columns
 * (out (nC, nb), gv (rows of L, nb)): rows of the Jacobian through L^T.
 * Replaces torch.sparse.mm(Lstack.t(), ...) of TorchDC2D.Jmatrix
 * (dctorch/simulation2d.py:506-507) and Linearization2D._Lt (659-674). */
int dct_values_vjp_multi(int64_t nC, int32_t nb, const int64_t* d_Lt_ptr,
                         const int32_t* d_Lt_col, const double* d_Lt_val,
                         const double* d_sigma, const double* d_gv, double* d_out,
                         void* stream);

/* ---- allocation-free small solve -------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (hosts whose framework owns all device memory through its own pool,
 * loops that cannot take the device-wide synchronisation of
 * cudaMalloc/cudaFree): factors one SPD system given by its CSR pattern and
 * values (n <= 512; the lower triangle is read) and solves k <= 64
 * right-hand sides, b and x row-major (n, k) float64 on the current device.
 * Its only scratch is a fixed 2 MiB array in the library (held by every GPU
 * that loads the library until exit); sizes beyond the limits return
 * DCT_ERR_ARG.  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress) and caches it.  Calls share the array, so calls
 * that may overlap on the GPU race and must be ordered.  The call does not
 * wait for the GPU: a matrix that is not positive definite (a non-positive
 * or NaN pivot) makes every entry of x NaN rather than returning a status.
 * The pattern must be canonical (columns in [0, n), no duplicates: a
 * duplicate overwrites instead of adding); out-of-range columns and
 * decreasing row pointers are skipped. */
int dct_solve_small_noalloc(int32_t n, const int32_t* d_crow,
                            const int32_t* d_col, const double* d_vals,
                            const double* d_b, int32_t k, double* d_x,
                            void* stream);

/* ---- general (unsymmetric-valued) systems -----------------------------------
 * Replaces cuDSS's "general" matrix type (dctorch/solver.py:44-47, the
 * _MTYPE map: "general" -> GENERAL) for structurally symmetric patterns.
 * A float64 plan that factors P A P^T = L U on the same symbolic analysis
 * and schedules as the symmetric plans, without row exchanges: static
 * pivoting replaces a pivot smaller than sqrt(eps) x the largest entry of its
 * block (in magnitude) by that bound with the pivot's sign (counted, see
 * dct_plan_static_pivots); a non-finite pivot records DCT_ERR_ZERO_PIVOT.
 * Every pattern entry (i, j) needs its (j, i) (else DCT_ERR_BAD_PATTERN).
 * dct_factorize takes float64 values of the whole pattern; dct_solve and
 * dct_solve_permuted solve A x = b, dct_solve_transposed A^T x = b (the
 * adjoint of a general solve) on the same factors. */
int dct_plan_create_general(const dct_symbolic* sym, int32_t nbatch, int32_t max_rhs,
                            int32_t device, dct_plan** out);
int dct_solve_transposed(dct_plan* plan, const void* d_b, int32_t io_dtype,
                         int32_t b_batched, int32_t k, void* d_x, void* stream);
/* Number of pivots static pivoting replaced in the last factorization of a
 * general plan (synchronises the stream; dct_check_status leaves it). */
int dct_plan_static_pivots(dct_plan* plan, void* stream, int32_t* count);

/* ---- self-test of the bounded device waits ---------------------------------
 * No counterpart in the reference (failure detection).  Runs the kernels'
 * bounded mbarrier wait on a barrier that nothing arrives on, with a limit of
 * `polls` polls (1 .. 65536, each at most a few microseconds), on one CTA
 * with no asynchronous operation in flight, and synchronises the stream.
 * *code receives the status the wait recorded (DCT_ERR_DEVICE_TIMEOUT when
 * it gave up, as a real stalled wait does in a plan's status words) and
 * *completed (may be null) whether the wait saw its phase complete (0 here).
 * The context stays usable afterwards. */
int dct_selftest_wait_timeout(int32_t polls, int32_t* code, int32_t* completed,
                              void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DCT_H */
