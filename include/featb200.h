/*
 * featb200.h - C ABI of the B200 (sm_100a) geometric-multigrid Poisson path.
 *
 * Two seams, matching the two places where the reference's solve path can be replaced:
 *
 *  1. Op level: drop-in replacements of the reference's LAFEM::Arch backend kernels
 *     (kernel/lafem/arch/*.hpp).  Raw DEVICE pointers, element counts and scalars; no ownership
 *     transfer.  Each call is enqueued on `stream` (NULL = legacy default stream) and, like the
 *     reference's *_cuda functions, returns after the work is complete unless noted otherwise.
 *     Index variants: _u64 = the reference's default `Index` (unsigned long),
 *     _u32 = FEAT_INDEX_U32 builds.  Value variants: _f64, _f32.
 *
 *  2. Solver level: an opaque-handle PCG preconditioned by a geometric-multigrid V-cycle
 *     (kernel/solver/pcg.hpp + kernel/solver/multigrid.hpp), built from the same per-level data
 *     the reference's MultiGridHierarchy::push_level receives (system matrix, unit filter,
 *     prolongation and restriction matrices, kernel/solver/multigrid.hpp:612-690).  Host buffers
 *     in, uploaded once; solves run on the device without host round trips.
 *
 * Every function returns an fb_status (0 = success).  fb_last_error() returns a message for the
 * most recent failure on the calling thread.
 */
#ifndef FEATB200_H
#define FEATB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int fb_status;
#define FB_OK 0
#define FB_ERR_ARG 1          /* invalid argument (sizes, null pointers, aliasing) */
#define FB_ERR_CUDA 2         /* a CUDA runtime call failed */
#define FB_ERR_STATE 3        /* object not initialised / wrong order of calls */
#define FB_ERR_NOMEM 4        /* device allocation failed */
#define FB_ERR_UNSUPPORTED 5  /* option not supported for this configuration */

/* Solver status codes: the reference's Solver::Status (kernel/solver/base.hpp:48-64). */
#define FB_SOLVER_UNDEFINED 0
#define FB_SOLVER_PROGRESS 1
#define FB_SOLVER_SUCCESS 2
#define FB_SOLVER_ABORTED 3
#define FB_SOLVER_DIVERGED 4
#define FB_SOLVER_MAX_ITER 5
#define FB_SOLVER_STAGNATED 6

const char* fb_last_error(void);
/* Library version string and the compute capability it was built for. */
const char* fb_version(void);
/* Number of this library's kernels launched since load (all threads, all devices). */
uint64_t fb_kernel_launch_count(void);

/* ------------------------------------------------------------------------------------------ */
/* 1. Op level: LAFEM::Arch equivalents (device pointers)                                     */
/* ------------------------------------------------------------------------------------------ */

/* r = a * A * x + b * y, or r = a * A^T * x + b * y when transposed != 0.  |b| < eps(DT) means y
 * is not read (r is cleared first).  r may alias y, must not alias x.
 * Replaces Arch::Apply::csr (kernel/lafem/arch/apply.hpp:44-79; generic semantics
 * apply_generic.hpp:25-69; CUDA backend apply.cu:176-261).  Non-transposed rows are summed
 * in stored entry order without FMA contraction, so FP64 results equal the generic backend's
 * bit for bit. */
fb_status fb_apply_csr_f64_u64(double* r, double a, const double* x, double b, const double* y,
                               const double* val, const uint64_t* col_ind, const uint64_t* row_ptr,
                               uint64_t rows, uint64_t columns, uint64_t used_elements,
                               int transposed, void* stream);
fb_status fb_apply_csr_f64_u32(double* r, double a, const double* x, double b, const double* y,
                               const double* val, const uint32_t* col_ind, const uint32_t* row_ptr,
                               uint64_t rows, uint64_t columns, uint64_t used_elements,
                               int transposed, void* stream);
fb_status fb_apply_csr_f32_u64(float* r, float a, const float* x, float b, const float* y,
                               const float* val, const uint64_t* col_ind, const uint64_t* row_ptr,
                               uint64_t rows, uint64_t columns, uint64_t used_elements,
                               int transposed, void* stream);
fb_status fb_apply_csr_f32_u32(float* r, float a, const float* x, float b, const float* y,
                               const float* val, const uint32_t* col_ind, const uint32_t* row_ptr,
                               uint64_t rows, uint64_t columns, uint64_t used_elements,
                               int transposed, void* stream);

/* r = a * x + y; r may alias x or y.  Replaces Arch::Axpy::value (axpy.hpp:21-54, axpy.cu:18-75). */
fb_status fb_axpy_f64(double* r, double a, const double* x, const double* y, uint64_t n, void* stream);
fb_status fb_axpy_f32(float* r, float a, const float* x, const float* y, uint64_t n, void* stream);

/* *result = x^T y (FP64 accumulation for both value types); result is a HOST pointer and the
 * call synchronises `stream`.  Replaces Arch::DotProduct::value (dot_product.hpp:21, dot_product.cu:21-61). */
fb_status fb_dot_f64(double* result, const double* x, const double* y, uint64_t n, void* stream);
fb_status fb_dot_f32(float* result, const float* x, const float* y, uint64_t n, void* stream);

/* *result = x^T y like fb_dot_f64, but without allocating any device memory, for callers that
 * cannot allocate when they need the reduction: processes that give all device memory to their
 * own pool allocator at start-up, and loops that must not stall on cudaMalloc/cudaFree, which can
 * synchronise the device.  Its scratch is a fixed 32 KiB array in the library's device image, held
 * by every GPU that loads the library; n may be at most FB_DOT_NOALLOC_MAX_N (longer vectors are
 * rejected with FB_ERR_ARG).  Every call looks up the array's device address in the current
 * context.  Under CUDA's lazy module loading the first call on a device loads the library's module,
 * which takes device memory: call it once per device with n = 0 (x and y may be null; nothing is
 * launched) before a pool takes the device memory, and before any stream capture.  All calls share
 * the array and it keeps the last call's contents: calls that overlap on the GPU (several streams or
 * host threads) race.  No counterpart in the reference: an addition of this library. */
#define FB_DOT_NOALLOC_MAX_N 16777216ull
fb_status fb_dot_f64_noalloc(double* result, const double* x, const double* y, uint64_t n, void* stream);

/* *result = ||x||_2; HOST result, synchronises.  Replaces Arch::Norm2::value (norm.hpp:21, norm.cu:20-59). */
fb_status fb_norm2_f64(double* result, const double* x, uint64_t n, void* stream);
fb_status fb_norm2_f32(float* result, const float* x, uint64_t n, void* stream);

/* r_i = x_i * y_i.  Replaces Arch::ComponentProduct::value (component_product.cu:20-55; unlike the
 * reference's CUDA kernel, the FP64 product is not rounded through float). */
fb_status fb_component_product_f64(double* r, const double* x, const double* y, uint64_t n, void* stream);
fb_status fb_component_product_f32(float* r, const float* x, const float* y, uint64_t n, void* stream);

/* r_i = s / x_i.  Replaces Arch::ComponentInvert::value (component_invert.cu:19-64). */
fb_status fb_component_invert_f64(double* r, const double* x, double s, uint64_t n, void* stream);
fb_status fb_component_invert_f32(float* r, const float* x, float s, uint64_t n, void* stream);

/* r_i = s * x_i.  Replaces Arch::Scale::value (scale.hpp:21, scale.cu:17-58). */
fb_status fb_scale_f64(double* r, const double* x, double s, uint64_t n, void* stream);
fb_status fb_scale_f32(float* r, const float* x, float s, uint64_t n, void* stream);

/* v[idx[k]] = vals[k] (rhs/sol) and v[idx[k]] = 0 (def/cor).
 * Replaces Arch::UnitFilter::filter_rhs / filter_def (unit_filter.hpp:21-71, unit_filter.cu:19-91). */
fb_status fb_unit_filter_rhs_f64_u64(double* v, const double* vals, const uint64_t* idx, uint64_t ue, void* stream);
fb_status fb_unit_filter_def_f64_u64(double* v, const uint64_t* idx, uint64_t ue, void* stream);
fb_status fb_unit_filter_rhs_f32_u32(float* v, const float* vals, const uint32_t* idx, uint64_t ue, void* stream);
fb_status fb_unit_filter_def_f32_u32(float* v, const uint32_t* idx, uint64_t ue, void* stream);

/* diag[row] = position of the diagonal entry of `row`, or row_ptr[rows] when the row has none.
 * Replaces Arch::Diagonal::csr (diagonal.cu:18-62). */
fb_status fb_diagonal_csr_u64(uint64_t* diag, const uint64_t* col_ind, const uint64_t* row_ptr,
                              uint64_t rows, void* stream);

/* r_i = value for i < n.  Replaces Util::cuda_set_memory (cuda_util.cu:202-219), which
 * MemoryPool::set_memory calls for the cuda backend (memory_pool.hpp:179-199). */
fb_status fb_set_memory_f64(double* r, double value, uint64_t n, void* stream);
fb_status fb_set_memory_f32(float* r, float value, uint64_t n, void* stream);
fb_status fb_set_memory_u64(uint64_t* r, uint64_t value, uint64_t n, void* stream);
fb_status fb_set_memory_u32(uint32_t* r, uint32_t value, uint64_t n, void* stream);

/* r[k] = val[k] * x[row] for every entry k of every row (r may alias val).  Replaces
 * Arch::ScaleRows::csr (scale_row_col.hpp, generic semantics scale_row_col_generic.hpp:19-31). */
fb_status fb_scale_rows_csr_f64_u64(double* r, const double* val, const uint64_t* row_ptr, const double* x,
                                    uint64_t rows, void* stream);

/* Precision conversion (MemoryPool::convert / Util::cuda_convert, cuda_util.cu:228-262). */
fb_status fb_convert_f64_to_f32(float* dst, const double* src, uint64_t n, void* stream);
fb_status fb_convert_f32_to_f64(double* dst, const float* src, uint64_t n, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* 2. Solver level: PCG + geometric multigrid                                                  */
/* ------------------------------------------------------------------------------------------ */

typedef struct fb_hierarchy fb_hierarchy;
typedef struct fb_solver fb_solver;

/* A CSR matrix in HOST memory with the reference's default index type (SparseMatrixCSR<double,
 * Index>, kernel/lafem/sparse_matrix_csr.hpp:280-302): row_ptr[rows+1], col_ind[nnz], val[nnz]. */
typedef struct
{
  uint64_t rows, columns, used_elements;
  const uint64_t* row_ptr;
  const uint64_t* col_ind;
  const double* val;
} fb_csr_host;

/* Create an empty hierarchy of `num_levels` levels on the current CUDA device.
 * Levels are numbered finest = 0 as in MultiGridHierarchy (kernel/solver/multigrid.hpp:419). */
fb_status fb_hierarchy_create(fb_hierarchy** out, int num_levels);

/* Set level `level` (0 = finest).  A: system matrix; filter_idx/filter_val[nf]: unit-filter
 * (Dirichlet) DOFs and values (UnitFilter, kernel/lafem/unit_filter.hpp:30); P: prolongation
 * level <- level+1 and R: restriction level+1 <- level (LAFEM::Transfer, kernel/lafem/transfer.hpp;
 * both NULL on the coarsest level).  Mirrors MultiGridHierarchy::push_level
 * (kernel/solver/multigrid.hpp:633-690).  Data is copied; the host buffers may be freed after. */
fb_status fb_hierarchy_set_level(fb_hierarchy* h, int level, const fb_csr_host* A,
                                 const uint64_t* filter_idx, const double* filter_val, uint64_t nf,
                                 const fb_csr_host* P, const fb_csr_host* R);

void fb_hierarchy_destroy(fb_hierarchy* h);

/* Precision of the multigrid preconditioner. */
#define FB_PREC_F64 0        /* plain FP64 (the reference's path; parity mode) */
#define FB_PREC_F32 1        /* FP32 V-cycle inside FP64 PCG (iterative refinement) */
#define FB_PREC_F32_BF16 2   /* as FB_PREC_F32, with BF16 matrix values in the V-cycle */

/* DOF ordering used on the device. */
#define FB_ORDER_NATIVE 0    /* the caller's numbering */
#define FB_ORDER_RCM 1       /* reverse Cuthill-McKee per level (host, at setup); vectors are
                                permuted on the way in and out of fb_solver_solve */

#define FB_CYCLE_V 0
#define FB_CYCLE_F 1
#define FB_CYCLE_W 2
/* coarse-grid correction of the multigrid (MultiGridAdaptCGC, kernel/solver/multigrid.hpp:39-50) */
#define FB_CGC_FIXED 0        /* x += P x_c */
#define FB_CGC_MIN_ENERGY 1   /* x += w P x_c, w = (d, c) / (A c, c) */
#define FB_CGC_MIN_DEFECT 2   /* x += w P x_c, w = (d, A c) / (A c, A c) */
/* the preconditioner of the Richardson smoother (JacobiPrecond, SORPrecond, SSORPrecond:
 * kernel/solver/jacobi_precond.hpp, sor_precond.hpp:179-224, ssor_precond.hpp) */
#define FB_SMOOTHER_JACOBI 0
#define FB_SMOOTHER_SOR 1
#define FB_SMOOTHER_SSOR 2
/* the order of the SOR / SSOR sweeps */
#define FB_SWEEP_SEQUENTIAL 0 /* the rows' dependency levels: the reference's generic sequential sweep, bit for bit */
#define FB_SWEEP_COLOURED 1   /* greedy colours by ascending size: the reference's coloured CUDA sweeps (sor_precond.cu:26-41) */

typedef struct
{
  int precision;        /* FB_PREC_* */
  int ordering;         /* FB_ORDER_* */
  double omega;         /* Jacobi damping (JacobiPrecond omega; 0.7 in the configured problems) */
  int smooth_steps;     /* Richardson min_iter = max_iter for pre- and post-smoothing (2 = V(2,2)) */
  double tol_rel;       /* PCG relative tolerance (IterativeSolver tol_rel) */
  double tol_abs;       /* PCG absolute tolerance (default 1/eps^2) */
  int max_iter;         /* PCG max_iter (default 100) */
  int min_iter;         /* PCG min_iter (default 0) */
  int use_graph;        /* capture the whole solve in one CUDA graph (1) or launch per kernel (0) */
  int rows_per_block;   /* batch solver: rows (threads) per block of the V-cycle passes, a multiple
                           of 32 up to 512; 0 = picked per level by the autotuner at creation */
  int tail_rows;        /* levels (below the finest) with at most this many rows, down to the
                           coarsest, run in one single-block kernel per visit of the cycle (a
                           V-cycle bottom, or an F/W sub-cycle with its peak smoothing); 0 = off */
  int tma_rows;         /* levels with at least this many rows use the TMA-staged persistent
                           passes (bulk copies into shared memory); 0 = off */
  int cluster_rows;     /* levels (below the finest) with at most this many rows, down to the
                           coarsest, run in one kernel on a cluster of 8 thread blocks (8 SMs) per
                           V-cycle, passes separated by the cluster barrier; takes precedence over
                           tail_rows; V-cycle only; 0 = off (default: measured slower than the
                           single-block tail on B200 for every threshold) */
  int cycle;            /* FB_CYCLE_V (default), FB_CYCLE_F or FB_CYCLE_W: the multigrid cycle of
                           MultiGrid::_apply_cycle_v/_f/_w (kernel/solver/multigrid.hpp:1350-1440) */
  int tma_window;       /* the window of the gathered vector that a TMA-staged chunk reads:
                           0 (default) = neither: the row sums gather from global memory;
                           1 = staged in shared memory with the chunk; 2 = bulk-prefetched into L2
                           when the chunk's copies are issued.  Both measured slower on B200 */
  int diagonal;         /* 1 (default): a level's system matrix whose entries lie on at most 27
                           diagonals of the device numbering, with strictly increasing columns in
                           every row (structured grids numbered lexicographically), is stored as
                           its diagonals without column indices (row sums keep the stored order;
                           missing diagonals hold zeros); 0 = always sliced ELL.  The multi-RHS
                           solver (fb_msolver_*) uses, for diagonal != 0, a stencil form for system
                           matrices whose stored rows all have the same 9 or 27 column offsets in
                           triplets (o-1, o, o+1); 0 = always CSR (measured as fast there) */
  int pdl;              /* 1 (default): the solve's kernels are launched with programmatic stream
                           serialisation, so each one's launch and its matrix prologue overlap the
                           end of its predecessor; 0 = plain stream order */
  int adapt_cgc;        /* FB_CGC_FIXED (default), FB_CGC_MIN_ENERGY or FB_CGC_MIN_DEFECT: the
                           coarse-grid correction is scaled by the step length that minimises the
                           energy or the defect, and the post-smoother starts from the defect
                           updated with A P x_c (MultiGrid::_apply_prol, multigrid.hpp:1880-1960) */
  int fused;            /* levels with at most this many rows (default 70000; 0 = never) that are
                           structured 2D grids (lexicographic 9-point operator in diagonal storage,
                           local restriction) run, in a V(2,2) cycle with the fixed coarse-grid
                           correction, pre-smoothing + defect + restriction as one pass and
                           prolongation + post-smoothing as another (tiles with halos recomputed in
                           shared memory); results are bitwise those of one pass per step */
  int smoother;         /* FB_SMOOTHER_JACOBI (default; damping `omega`), FB_SMOOTHER_SOR or FB_SMOOTHER_SSOR:
                           the Richardson smoother's preconditioner; SOR / SSOR need FB_ORDER_NATIVE and the
                           fixed coarse-grid correction, and run without the tail kernels */
  double smoother_omega;/* SOR / SSOR damping (SORPrecond omega; default 1) */
  int sweep_colouring;  /* FB_SWEEP_SEQUENTIAL (default) or FB_SWEEP_COLOURED */
  int streamed;         /* structured 2D levels with more rows than `fused` and at least this many
                           (0 = never) run the same two fused passes swept row by row through
                           tiles of whole coarse-row bands, their rows staged in shared memory by
                           the bulk-copy engine; results are bitwise those of one pass per step */
} fb_solver_config;

/* Fill `cfg` with the reference's defaults: FP64, native order, omega 0.7, V(2,2), tol_rel 1e-8,
 * tol_abs 1/eps^2, max_iter 100, min_iter 0, graph on, autotuned blocks, single-block tail for
 * levels of at most 300 rows, TMA-staged passes from 1000 rows (both thresholds tuned on B200). */
void fb_solver_config_default(fb_solver_config* cfg);

typedef struct
{
  int status;           /* FB_SOLVER_* */
  int iterations;
  double def_init;      /* initial defect norm */
  double def_final;     /* final defect norm */
  double solve_ms;      /* device time of the solve (CUDA events) */
  uint64_t kernel_launches;  /* kernels of this library launched by the solve */
  double bytes_moved;   /* algorithmic bytes of every launched kernel */
} fb_solve_info;

/* Build the solver: uploads every level, forms the Jacobi inverse diagonals, the exact coarse
 * inverse and (for FB_PREC_F32*) the low-precision copies.  Mirrors MultiGridHierarchy::init +
 * PCG::init.  The hierarchy must stay alive while the solver exists. */
fb_status fb_solver_create(fb_solver** out, fb_hierarchy* h, const fb_solver_config* cfg);
void fb_solver_destroy(fb_solver* s);

/* PCG::correct semantics (kernel/solver/pcg.hpp:159-170): sol holds the initial guess on entry
 * and the solution on return.  HOST buffers of the finest level's size; copies in and out are
 * part of the call.  Synchronous. */
fb_status fb_solver_solve(fb_solver* s, double* sol, const double* rhs, fb_solve_info* info);

/* As fb_solver_solve with DEVICE buffers in the caller's numbering, enqueued on `stream`;
 * returns after the solve completed. */
fb_status fb_solver_solve_device(fb_solver* s, double* sol, const double* rhs, void* stream,
                                 fb_solve_info* info);

/* One application of the preconditioner (MultiGrid::apply, kernel/solver/multigrid.hpp:1270):
 * cor = V-cycle(def).  HOST buffers of the finest level's size. */
fb_status fb_solver_vcycle(fb_solver* s, double* cor, const double* def);

/* Kernels that fb_solver_time_kernel can time in isolation. */
#define FB_KERNEL_PCG_SPMV 0   /* q = F(A p) with q.p, finest level, FP64 (the PCG matrix product) */
#define FB_KERNEL_MG_DEFECT 1  /* d = F(b - A x), finest level, in the V-cycle's precision */
#define FB_KERNEL_MG_TAIL 2    /* the coarse-level tail kernel (one launch; needs a tail level) */
#define FB_KERNEL_MG_CYCLE 3   /* one whole multigrid cycle from the finest level (all its launches) */
#define FB_KERNEL_MG_SMOOTH 4  /* pre-smoothing step 2 x' = x + F(D F(b - A x)), finest level */
#define FB_KERNEL_MG_POST1 5   /* post-smoothing step 1: d = F(b - A x), c = F(D d), ||d||, finest level */
#define FB_KERNEL_MG_POST2 6   /* post-smoothing step 2 with the PCG's z = x + c' and r.z, finest level */
#define FB_KERNEL_MG_RESTRICT 7 /* restriction b_c = F(R d) with sol1_c = F(D_c b_c), finest to next level */
#define FB_KERNEL_MG_PROLONG 8 /* prolongation x += F(P x_c), next level to finest */
#define FB_KERNEL_MG_DOWN 9    /* fused pre-smoothing step 2 + defect + restriction, finest level (structured grids,
                                  whatever the `fused` row threshold) */
#define FB_KERNEL_MG_UP 10     /* fused prolongation + post-smoothing with the PCG's z and r.z, finest level */
#define FB_KERNEL_MG_SDOWN 11  /* FB_KERNEL_MG_DOWN in its streamed form (whatever the `streamed` threshold) */
#define FB_KERNEL_MG_SUP 12    /* FB_KERNEL_MG_UP in its streamed form */

/* Launches kernel `which` `reps` times on the solver's stream, timing each launch with CUDA events
 * on that stream (the finest level's pass kernels need a finest level above the coarse-level tail);
 * with flush_l2 != 0 a 256 MiB buffer is overwritten and another 256 MiB buffer read
 * before each launch (outside the timed interval), so every launch starts with an L2 that holds
 * none of its data and no dirty lines.  Returns the mean launch time and the
 * kernel's bytes per launch as stored on the device (matrix as stored + gathered vector + row-wise
 * vector reads and writes + Dirichlet mask; 0 for the tail and the whole cycle).  No counterpart in the reference: a measurement aid for the SpMV roofline. */
fb_status fb_solver_time_kernel(fb_solver* s, int which, int reps, int flush_l2, double* avg_ms,
                                double* bytes_per_launch);

/* Per-level sizes after upload: rows, nnz of A, nnz of P (as stored on the device, explicit zeros
 * removed).  `out` holds 3 * num_levels entries. */
fb_status fb_solver_level_info(const fb_solver* s, uint64_t* out);

/* How a solver would store a matrix on the device (host only, no device touched).  kind: 0 sliced
 * ELL, 1 uniform-width ELL, 2 diagonal storage; width: entries per row (the widest slice for sliced
 * ELL); narrow: column indices as int16 offsets from the row; diagonals: the number of diagonals
 * (kind 2); entries: stored slots including padding.  rcm != 0: in reverse Cuthill-McKee order (the
 * solver's FB_ORDER_RCM); allow_diag != 0: diagonal storage allowed (the solver's `diagonal`, for
 * system matrices).  Rows listed in empty_rows (Dirichlet rows, NULL for none) are stored empty. */
typedef struct
{
  int kind, narrow;
  uint32_t width, diagonals;
  uint64_t entries;
} fb_storage_plan;
fb_status fb_matrix_storage_plan(const fb_csr_host* M, const uint64_t* empty_rows, uint64_t num_empty, int rcm,
                                 int allow_diag, fb_storage_plan* out);

/* Events of one multigrid cycle, as a solver with this cycle and coarse-grid correction runs them */
#define FB_EV_PRE 0        /* pre-smoothing steps 2.. on a level (step 1 comes with the restriction) */
#define FB_EV_DEF 1        /* defect on a level */
#define FB_EV_RES 2        /* restriction from a level to the next coarser one */
#define FB_EV_CRS 3        /* coarse solve */
#define FB_EV_PRO 4        /* prolongation into a level (x += P x_c) */
#define FB_EV_POST 5       /* post-smoothing (also the peak smoother) on a level */
#define FB_EV_POST_TOP 6   /* the finest level's last post-smoothing (forms the PCG's z and r.z) */
#define FB_EV_PROC 7       /* prolongation with adaptive coarse-grid correction */
#define FB_EV_POSTC 8      /* post-smoothing from the defect that FB_EV_PROC updated */
#define FB_EV_POSTC_TOP 9  /* as FB_EV_POST_TOP after FB_EV_PROC */

/* The event list of one cycle over num_levels levels (finest = level 0): MultiGrid::_apply_cycle_v,
 * _f, _w with _apply_rest, _apply_prol and _apply_smooth_peak (kernel/solver/multigrid.hpp:1335-1990).
 * Writes at most `capacity` (op, level) pairs into ops[] / levels[]; *count receives the full
 * number of events.  Host only (no device is touched). */
fb_status fb_multigrid_cycle_events(int cycle, int adapt_cgc, int num_levels, uint8_t* ops, uint8_t* levels,
                                    uint64_t capacity, uint64_t* count);

/* New stopping tolerances for the following solves (IterativeSolver::set_tol_rel/set_tol_abs,
 * kernel/solver/iterative.hpp): converged when ||d|| <= tol_abs and ||d|| <= tol_rel * ||d_0||. */
fb_status fb_solver_set_tolerances(fb_solver* s, double tol_rel, double tol_abs);

/* New iteration limits for the following solves (IterativeSolver::set_min_iter / set_max_iter,
 * kernel/solver/iterative.hpp): max_iter may not exceed the max_iter of the configuration the
 * solver was created with. */
fb_status fb_solver_set_iteration_limits(fb_solver* s, int min_iter, int max_iter);

/* New values for the system matrix of `level` (0 = finest): `values` is a DEVICE array of the
 * level's used_elements doubles in the pattern and entry order passed to fb_hierarchy_set_level
 * (the pattern must not change).  Rewrites the stored values (and the FP64 copy of the finest level
 * in FB_PREC_F32* modes), recomputes the level's Jacobi inverse diagonal omega / a_ii on the device
 * and, for the coarsest level, the exact coarse inverse on the host.  Ordered on `stream`; returns
 * after it completed.  Counterpart of re-running init_numeric() of the hierarchy after the
 * matrices' values changed (kernel/solver/multigrid.hpp:776-790, JacobiPrecond::init_numeric
 * kernel/solver/jacobi_precond.hpp:136-165).  The host copies in the fb_hierarchy keep the old
 * values. */
fb_status fb_solver_update_matrix(fb_solver* s, int level, const double* values, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* 3. Solver level, many right-hand sides: K = 32 or 64 systems with one hierarchy              */
/* ------------------------------------------------------------------------------------------ */

typedef struct fb_msolver fb_msolver;

/* Like fb_solver_create for num_rhs (32 or 64) right-hand sides solved together: every right-hand
 * side runs its own PCG + V-cycle (own scalars, stopping test and smoother skip flags); each matrix
 * entry is read once per pass for all of them.  FB_PREC_F64 or FB_PREC_F32, smooth_steps >= 2.
 * Counterpart of solving with DenseVectorBlocked<double, Index, num_rhs> vectors (the reference's
 * multi-vector CSR kernel, kernel/lafem/arch/apply.cu:109-135, handles up to 3 per row). */
fb_status fb_msolver_create(fb_msolver** out, fb_hierarchy* h, const fb_solver_config* cfg, int num_rhs);
void fb_msolver_destroy(fb_msolver* s);

/* sol/rhs: HOST arrays of rows * num_rhs doubles, right-hand side index fastest (x[row*num_rhs+j]);
 * sol holds the initial guesses.  info: NULL or num_rhs entries (per right-hand side). */
fb_status fb_msolver_solve(fb_msolver* s, double* sol, const double* rhs, fb_solve_info* info);
/* As fb_msolver_solve with DEVICE arrays, ordered on `stream`. */
fb_status fb_msolver_solve_device(fb_msolver* s, double* sol, const double* rhs, void* stream, fb_solve_info* info);

/* ------------------------------------------------------------------------------------------ */
/* 4. Solver level, batches: many independent systems of uneven size                           */
/* ------------------------------------------------------------------------------------------ */

typedef struct fb_batch fb_batch;

/* A batch of num independent PCG + V-cycle solves, one hierarchy each (any number of levels, at
 * least 2).  Every V-cycle pass runs as ONE launch over all instances present at that level
 * (levels aligned from the coarsest); each instance keeps its own scalars, stopping test and
 * skip flags, and converged instances stop working.  The reference solves such families one
 * system after the other. */
fb_status fb_batch_create(fb_batch** out, int num, fb_hierarchy* const* hierarchies, const fb_solver_config* cfg);
void fb_batch_destroy(fb_batch* b);
/* top_rows[num]: finest-level size of every instance (the packed vector is their concatenation) */
fb_status fb_batch_sizes(const fb_batch* b, uint64_t* top_rows);
/* sol/rhs: HOST packed arrays (instances concatenated in order, each in its caller numbering);
 * sol holds the initial guesses.  info: NULL or num entries. */
fb_status fb_batch_solve(fb_batch* b, double* sol, const double* rhs, fb_solve_info* info);
/* As fb_batch_solve with DEVICE packed arrays, ordered on `stream`. */
fb_status fb_batch_solve_device(fb_batch* b, double* sol, const double* rhs, void* stream, fb_solve_info* info);
/* Rows per block of the V-cycle passes per global level (finest first; rows_per_block may be NULL to
 * query num_levels): the autotuner's choice at creation, or cfg.rows_per_block.  No counterpart in
 * the reference. */
fb_status fb_batch_rows_per_block(const fb_batch* b, int* rows_per_block, int* num_levels);

/* ------------------------------------------------------------------------------------------ */
/* 5. Set-up on the device: Q1 assembly on the uniformly refined unit square                    */
/* ------------------------------------------------------------------------------------------ */

/* The step before the solve path.  Vertices of level L are numbered lexicographically (x fastest),
 * (2^L+1)^2 of them; the reference assembles the same operators on the host
 * (assemble_bilinear_operator_matrix_1 with a LaplaceOperator / kappa-weighted operator,
 * kernel/assembly/domain_assembler_helpers.hpp, common_operators.hpp:36, the load vector
 * int f phi_i of common_functionals.hpp:33; cubature "auto-degree:5" = 3x3 Gauss). */

/* The row-sorted 9-point CSR pattern of level L (HOST arrays; row_ptr (2^L+1)^2+1 entries, col_ind
 * nnz entries).  Pass NULL arrays to query nnz first.  0 <= level <= 13. */
fb_status fb_q1_pattern_2d(int level, uint64_t* nnz, uint64_t* row_ptr, uint64_t* col_ind);

/* Stiffness values of -div(kappa grad u) in that pattern and/or the load vector (Dirichlet
 * boundary entries set to 0), DEVICE arrays, ordered on `stream`, synchronous on return.
 * kappa = exp(g), g(x,y) = s sum_{i,j<K} (xi[i*K+j] cos t + eta[i*K+j] sin t) / (kx_i^2 + ky_j^2),
 * t = 2 pi (kx_i x + ky_j y), kx_i = i - K/2, ky_j = j - K/2, the (0,0) mode left out; kmodes = 0
 * gives kappa = 1 (xi, eta unused).  f = sum_g a_g exp(-|x - c_g|^2 / (2 w_g^2)) with
 * gauss[4g..4g+3] = (c_x, c_y, w, a) (DEVICE array).  row_ptr: DEVICE copy of the pattern's row
 * pointer (needed with values).  values or rhs may be NULL. */
fb_status fb_q1_assemble_2d(int level, int kmodes, const double* xi, const double* eta, double s, int ngauss,
                            const double* gauss, const uint64_t* row_ptr, double* values, double* rhs,
                            void* stream);

/* The Q1 prolongation from level-1 to `level` (1 <= level <= 13) on the lexicographic vertices
 * (weights 1, 1/2, 1/4; entries in ascending coarse index), written into DEVICE arrays (row_ptr
 * (2^level+1)^2+1, col_ind and values nnz entries); with all three NULL only nnz is returned.  The
 * reference assembles it on the host (assemble_prolongation_direct,
 * kernel/assembly/grid_transfer.hpp:353-430); R = P^T. */
fb_status fb_q1_prolongation_2d(int level, uint64_t* nnz, uint64_t* row_ptr, uint64_t* col_ind, double* values,
                                void* stream);

/* The 3D counterparts for the Laplacian on the unit cube refined to level L (hexahedral Q1, 3x3x3
 * Gauss rule, (2^L+1)^3 vertices numbered lexicographically, x fastest; L <= 8): the row-sorted
 * 27-point pattern (host), the stiffness values in that pattern and / or the load vector of a sum
 * of Gaussians (DEVICE gauss[ngauss][5] = c_x, c_y, c_z, w, a; boundary entries zeroed), and the
 * prolongation level L-1 -> L (weights 1, 1/2, 1/4, 1/8, DEVICE arrays of nnz entries).
 * Replace the reference's host assembly on RefinedUnitCubeFactory meshes
 * (kernel/assembly/common_operators.hpp:36, kernel/assembly/grid_transfer.hpp:353-430 in 3D) in
 * lexicographic numbering. */
fb_status fb_q1_pattern_3d(int level, uint64_t* nnz, uint64_t* row_ptr, uint64_t* col_ind);
fb_status fb_q1_assemble_3d(int level, int ngauss, const double* gauss, const uint64_t* row_ptr, double* values,
                            double* rhs, void* stream);
fb_status fb_q1_prolongation_3d(int level, uint64_t* nnz, uint64_t* row_ptr, uint64_t* col_ind, double* values,
                                void* stream);

/* f (sum of Gaussians, as above) and g = log kappa at the vertices of level L (DEVICE arrays of
 * (2^L+1)^2 doubles, lexicographic; either may be NULL): the inputs of the learned warm start. */
fb_status fb_q1_sample_2d(int level, int kmodes, const double* xi, const double* eta, double s, int ngauss,
                          const double* gauss, double* f, double* g, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* 6. Learned warm start: a convolutional U-Net on vertex grids (no counterpart in the reference) */
/* ------------------------------------------------------------------------------------------ */

/* Maps (f, log kappa) sampled on a G x G vertex grid (G = 2^k + 1, k >= 3) to an approximation of
 * u on the same grid; the solve path prolongates it to the finest level as the PCG initial guess.
 * 8 convolutions (channels 16/32/64/64, 3x3, zero padding): three injection subsamplings on the way
 * down, bilinear vertex upsampling + concatenation with the encoder activations on the way up, ReLU
 * everywhere but the last layer.  BF16 activations and GEMM operands, FP32 accumulation (tensor
 * cores), FP32 master parameters with Adam.  Parameter order: per layer W[co][tap][ci]
 * (tap = (dy+1)*3 + dx+1, dy along the slow grid axis), then b[co]. */
typedef struct fb_unet fb_unet;

fb_status fb_unet_create(fb_unet** out, int grid, int max_batch);
void fb_unet_destroy(fb_unet* u);
fb_status fb_unet_num_params(const fb_unet* u, uint64_t* n);
/* HOST arrays of num_params floats; set_params also resets the Adam moments */
fb_status fb_unet_set_params(fb_unet* u, const float* params);
fb_status fb_unet_get_params(const fb_unet* u, float* params);
fb_status fb_unet_get_grads(const fb_unet* u, float* grads);
/* in: DEVICE [batch][2][G][G] FP32 (channel 0 = f, 1 = log kappa, caller-scaled);
 * out: DEVICE [batch][G][G] FP32.  Keeps the activations for fb_unet_backward. */
fb_status fb_unet_forward(fb_unet* u, const float* in, float* out, int batch, void* stream);
/* dout: DEVICE [batch][G][G] FP32 = d loss / d out of the last forward (same batch); writes (or,
 * with accumulate != 0, adds) the parameter gradients. */
fb_status fb_unet_backward(fb_unet* u, const float* dout, int batch, int accumulate, void* stream);
/* One Adam step (t = 1, 2, ...) with the stored gradients. */
fb_status fb_unet_adam(fb_unet* u, float lr, float beta1, float beta2, float eps, int t, void* stream);
/* loss (DEVICE double) = mean (y - t)^2 over n entries; grad (DEVICE, or NULL) = 2 (y - t) / n */
fb_status fb_unet_mse(fb_unet* u, const float* y, const float* t, uint64_t n, float* grad, double* loss,
                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FEATB200_H */
