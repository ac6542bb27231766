/*
 * gipb200 -- B200 (sm_100a) kernels and device-resident solvers for GIP's algebraic
 * fractional-step Navier-Stokes timestep, behind a plain C ABI.
 *
 * Conventions
 *  - Every entry point returns an int status (GIPB200_OK = 0).  On error
 *    gipb200_last_error() returns a message for the calling thread.
 *  - Pointers named d_* are device pointers; h_* are host pointers owned by the
 *    caller.  Handles own their device memory until *_destroy.
 *  - `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).
 *  - Integer indices are 0-based int32, values float64, as in GIP's CSR files.
 *  - SpMV follows GIP's CPU Specification: a row with rowptr[i]==rowptr[i+1] leaves
 *    y[i] untouched, and every row sums its nonzeros sequentially in stored order, so
 *    float64 products match GIP's CPU build bit for bit.
 *
 * GIP's own device library is `extern "C++"` with void returns and default-stream
 * blocking reductions (src/Specifications/Cuda/Headers/GIP_gpu.h:4-46); each
 * declaration below names the routine it replaces.
 */
#ifndef GIPB200_H
#define GIPB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  GIPB200_OK = 0,
  GIPB200_ERR_ARG = 1,        /* invalid argument or inconsistent sizes            */
  GIPB200_ERR_CUDA = 2,       /* a CUDA runtime call failed                        */
  GIPB200_ERR_BREAKDOWN = 3,  /* PCG: p.Ap <= 0 or a non-finite scalar             */
  GIPB200_ERR_TIMEOUT = 4,    /* a bounded device wait gave up                     */
  GIPB200_ERR_NOMEM = 5,      /* device or host allocation failed                  */
  GIPB200_ERR_NOT_CONVERGED = 6,
  GIPB200_ERR_STATE = 7       /* call not valid in the object's current state       */
};

/* ------------------------------------------------------------------ library */
int gipb200_version(void);                 /* major*10000 + minor*100 + patch */
const char* gipb200_status_string(int status);
const char* gipb200_last_error(void);

/* GIP_cudaSetDevice (src/Specifications/Cuda/Libs/libgpu.cu:237-240) */
int gipb200_set_device(int device);
/* GIP_cudaMallocDouble / GIP_cudaMallocInt (libgpu.cu:18-26) */
int gipb200_malloc(void** d_ptr, size_t bytes);
/* GIP_cudaFree (libgpu.cu:52-55) */
int gipb200_free(void* d_ptr);
/* GIP_cudaMemcpyDToGpu / IToGpu (libgpu.cu:29-39) */
int gipb200_memcpy_h2d(void* d_dst, const void* h_src, size_t bytes, void* stream);
/* GIP_cudaMemcpyDToCpu / IToCpu (libgpu.cu:41-49) */
int gipb200_memcpy_d2h(void* h_dst, const void* d_src, size_t bytes, void* stream);
/* The same copy enqueued on `stream` without waiting for it (h_dst pinned for the copy to
 * overlap work on other streams; read it after the stream has passed it). */
int gipb200_memcpy_d2h_async(void* h_dst, const void* d_src, size_t bytes, void* stream);
/* GIP_cudaDcopy (libgpu.cu:68-71): d_dst[0:n) = d_src[0:n) */
int gipb200_dcopy(int n, double* d_dst, const double* d_src, void* stream);
int gipb200_stream_sync(void* stream);
/* GIP_cudaEventCreate / Record / Synchronize / ElapsedTime / Destroy (libgpu.cu:206-235) */
int gipb200_event_create(void** event);
int gipb200_event_record(void* event, void* stream);
int gipb200_event_elapsed_ms(void* start, void* stop, float* ms); /* waits for stop */
int gipb200_event_destroy(void* event);

/* ------------------------------------------------------------------ raw-pointer kernels */
/* GIP_cudaDCsrSpMV (libgpu.cu:89-96 and 113-120).  mode 0: y = A x; mode 1:
 * y = alpha A x + beta y.  Empty rows keep y (GIP's CPU semantics, not libgpu's). */
int gipb200_dcsr_spmv(int nrows, const int* d_rowptr, const int* d_col, const double* d_val,
                      const double* d_x, double* d_y, double alpha, double beta, int mode,
                      void* stream);
/* GIP_cudaDaxpy (libgpu.cu:133-139): y += alpha x */
int gipb200_daxpy(int n, double* d_y, const double* d_x, double alpha, void* stream);
/* GIP_cudaDaxpy(alpha,beta) (libgpu.cu:152-158): y = alpha x + beta y */
int gipb200_daxpby(int n, double* d_y, const double* d_x, double alpha, double beta,
                   void* stream);
/* GIP_VectorCuda::operator=(int) (GIP_VectorCuda.cpp:190-195): y[0:n) = value */
int gipb200_dfill(int n, double* d_y, double value, void* stream);
/* GIP_Topo::pack (src/BasicInterfaces/GIP_Topo.cpp:109-115) in device memory:
 * d_buf[k] = d_x[d_idx[k]] for k < n (the interface cells a neighbour reads). */
int gipb200_gather(int n, const int* d_idx, const double* d_x, double* d_buf, void* stream);
/* GIP_Topo::unpack (GIP_Topo.cpp:116-122) in device memory: d_x[d_idx[k]] = d_buf[k]
 * (the halo cells received); indices must be distinct. */
int gipb200_scatter(int n, const int* d_idx, const double* d_buf, double* d_x, void* stream);
/* GIP_cudaDdot (libgpu.cu:160-203): *h_result = sum x[i]*y[i], one pass, deterministic
 * two-level order; blocks until the result is on the host. */
int gipb200_ddot(int n, const double* d_x, const double* d_y, double* h_result, void* stream);
/* GIP_gpuNormi (libgpu.cu:337-393): *h_result = max |x[i]| */
int gipb200_dnorminf(int n, const double* d_x, double* h_result, void* stream);
/* GIP_gpuGetCFL (libgpu.cu:244-334) with GIP's CPU expression order
 * (GIP_NonLinearMulticore.cpp:3-55): *h_dt = min(0.1, 0.8*min_i(...)) over [0,n). */
int gipb200_cfl(int n, const double* d_u, const double* d_v, const double* d_w,
                const double* d_dxs, double gamma, double rho, double* h_dt, void* stream);

/* ------------------------------------------------------------------ matrix handles */
typedef struct gipb200_matrix_s* gipb200_matrix;

/* GIP_MatrixCuda::postConstruct (src/Specifications/Cuda/GIP_MatrixCuda.cpp:14-53):
 * uploads a host CSR and builds the device layouts (CSR plus 32-row sliced ELL).
 * Every column index must lie in [0, ncols): x vectors passed to the products must hold
 * ncols entries (at one rank GIP's operators satisfy this with ncols = cells or faces). */
int gipb200_matrix_create(int nrows, int ncols, int nnz, const int* h_rowptr, const int* h_col,
                          const double* h_val, gipb200_matrix* out);
int gipb200_matrix_destroy(gipb200_matrix A);
int gipb200_matrix_info(gipb200_matrix A, int* nrows, int* ncols, int* nnz, int64_t* padded_slots);
/* GIP_MatrixCuda::spmv(x,b[,alpha,beta]) (GIP_MatrixCuda.cpp:83-91) */
int gipb200_matrix_spmv(gipb200_matrix A, const double* d_x, double* d_y, double alpha,
                        double beta, int mode, void* stream);
/* GIP_MatrixCuda::spmv(x,GIP_Matrix*[,alpha,beta]) (GIP_MatrixCuda.cpp:93-100): row k of A
 * writes value k of `target` (A has one row per nonzero of target). */
int gipb200_matrix_spmv_values(gipb200_matrix A, const double* d_x, gipb200_matrix target,
                               double alpha, double beta, int mode, void* stream);
/* Copies the target's current values (stored order) to the host. */
int gipb200_matrix_get_values(gipb200_matrix A, double* h_val);
/* GIP_MatrixCuda::setUpDiagonal (GIP_MatrixCuda.cpp:143-184): d_dinv[i] = 1/A_ii;
 * *missing = rows without a diagonal entry (their dinv is 0). */
int gipb200_matrix_inverse_diagonal(gipb200_matrix A, double* d_dinv, int* missing);

/* ------------------------------------------------------------------ fused CG operations */
/* For hosts that drive GIP's solver loop themselves (GIP_LinearSolver.h:85-116): one
 * iteration is gipb200_matrix_spmv_dot, gipb200_cg_update_dot, gipb200_cg_direction --
 * three launches in place of GIP's SpMV, two dots, diagonal SpMV and three axpys
 * (libgpu.cu:75-203), with every scalar kept in device memory so the host never waits.
 * Element arithmetic follows GIP's CPU rounding; the dots sum in a fixed two-level
 * order.  Calls that share a matrix handle share its reduction scratch: order them on
 * one stream. */
typedef struct {
  double rz;     /* r.z: the previous value on entry to cg_update_dot, the new one after */
  double pAp;    /* p.Ap (point gipb200_matrix_spmv_dot's d_dot here)                    */
  double alpha;  /* rz / pAp, written by cg_update_dot                                   */
  double beta;   /* new rz / previous rz, written by cg_update_dot                       */
  double rr;     /* r.r after the update                                                 */
} gipb200_cg_scalars;
/* GIP_cudaDCsrSpMV + GIP_cudaDdot (libgpu.cu:89-96, 187-203), the pair at
 * GIP_LinearSolver.h:89-91: y = A x (rows without nonzeros keep y) and
 * *d_dot = sum_{i < n_dot} x_i y_i, written to DEVICE memory.  x and y must not alias. */
int gipb200_matrix_spmv_dot(gipb200_matrix A, const double* d_x, double* d_y, int n_dot,
                            double* d_dot, void* stream);
/* GIP_cudaDaxpy x2 + diagonal SpMV + GIP_cudaDdot (libgpu.cu:133-139, 89-96, 187-203), the
 * sequence at GIP_LinearSolver.h:93-111: alpha = rz/pAp; x += alpha p; r -= alpha q;
 * z = dinv r; then rz (new), rr = r.r, beta and alpha into *d_sc.  n <= rows of A (A
 * supplies only the reduction scratch).  A row whose dinv is 0 gets z = 0. */
int gipb200_cg_update_dot(gipb200_matrix A, int n, double* d_x, double* d_r, double* d_z,
                          const double* d_p, const double* d_q, const double* d_dinv,
                          gipb200_cg_scalars* d_sc, void* stream);
/* GIP_cudaDaxpy(alpha,beta) (libgpu.cu:152-158) at GIP_LinearSolver.h:113:
 * p = 1.0 z + beta p with beta read from *d_sc on the device. */
int gipb200_cg_direction(int n, double* d_p, const double* d_z, const gipb200_cg_scalars* d_sc,
                         void* stream);

/* ------------------------------------------------------------------ PCG */
typedef struct gipb200_pcg_s* gipb200_pcg;

enum {
  GIPB200_PCG_FIXED = 0,  /* exactly maxit iterations: GIP_LinearSolver.h:85-116          */
  GIPB200_PCG_TOL = 1,    /* stop when ||r||_2 <= tol ||b||_2 (r recursive)                */
  GIPB200_PCG_MIXED = 2   /* FP32 PCG with FP64 residual replacement (iterative refinement
                             that keeps the Krylov direction), stop at tol                  */
};

typedef struct {
  int mode;          /* GIPB200_PCG_*                                                */
  int maxit;         /* FIXED: iterations; TOL/MIXED: cap on (inner) iterations      */
  double tol;        /* TOL/MIXED: relative 2-norm residual target                   */
  double inner_tol;  /* MIXED: the FP64 true residual replaces the FP32 one when the
                        FP32 residual has fallen by this factor (reliable update)   */
  int inner_maxit;   /* MIXED: unused (kept for layout)                              */
  int max_outer;     /* MIXED: cap on residual replacements                          */
  int precond;       /* GIPB200_PRECOND_*: GIP's Jacobi (0); TOL/MIXED may take AMG  */
} gipb200_pcg_params;

/* Preconditioners.  JACOBI is GIP's (GIP_LinearSolver.h:70-80).  AMG (no counterpart in
 * the reference; TOL and MIXED): a smoothed-aggregation multigrid V-cycle, its hierarchy
 * built on the host once at create time — in FP32 from the Jacobi-scaled operator for
 * MIXED, in FP64 from the operator itself for TOL. */
enum { GIPB200_PRECOND_JACOBI = 0, GIPB200_PRECOND_AMG = 1 };

typedef struct {
  int iterations;        /* FIXED/TOL: PCG iterations; MIXED: inner iterations summed */
  int outer;             /* MIXED: FP64 residual replacements                         */
  int status;            /* GIPB200_OK / BREAKDOWN / NOT_CONVERGED                    */
  double rr;             /* r.r at exit (MIXED: true FP64 residual)                   */
  double bb;             /* b.b                                                       */
} gipb200_pcg_result;

/* GIP_LinearSolver::setUp (src/Algorithms/GIP_LinearSolver.h:31-42) */
int gipb200_pcg_create(gipb200_matrix L, int n_all, const gipb200_pcg_params* params,
                       gipb200_pcg* out);
int gipb200_pcg_destroy(gipb200_pcg S);
/* GIP_LinearSolver::solve (GIP_LinearSolver.h:44-117): x (n_all) = PCG(b) from x0. */
int gipb200_pcg_solve(gipb200_pcg S, const double* d_b, double* d_x, const double* d_x0,
                      void* stream, gipb200_pcg_result* h_result);

/* No counterpart in the reference: launches a kernel whose shared-memory barrier wait can
 * never complete and writes the status it reported (GIPB200_ERR_TIMEOUT after about one
 * second of SM clock).  Checks on the device that the library's bounded barrier wait gives
 * up instead of hanging; the context stays usable. */
int gipb200_check_bounded_wait(void* stream, int* h_status);

/* No counterpart in the reference: how the solver stores its operator. */
typedef struct {
  int pin_row;                 /* MIXED: detected pinned-Neumann row (-1: none)           */
  int compressed;              /* MIXED: FP32 operator packed (see value_table)           */
  int value_table;             /* MIXED: bits of a packed row's value-table index (4, 8)  */
  double compressed_fraction;  /* MIXED: share of the operator's slots in packed slices   */
  int amg_levels;              /* AMG: levels of the hierarchy (0: no AMG)                */
  double amg_complexity;       /* AMG: operator nonzeros of all levels / of the finest     */
  double amg_setup_s;          /* AMG: host setup time                                    */
  int packed_residual;         /* MIXED: FP64 residual from the packed columns (1) or L   */
} gipb200_pcg_info;
int gipb200_pcg_get_info(gipb200_pcg S, gipb200_pcg_info* info);
/* No counterpart in the reference: times `reps` launches of the solver's SpMV-dot kernel
 * (FP64 forms: the FP64 kernel; MIXED: the FP32 kernel of its operator layout) on its
 * current search direction, with CUDA events on `stream`; returns the mean launch time and
 * the kernel's streamed bytes per launch.  Solve once first so the direction is set. */
int gipb200_pcg_kernel_time(gipb200_pcg S, int reps, void* stream, double* avg_ms,
                            double* bytes);

/* No counterpart in the reference (GIP has no multigrid): per-kernel profile of the AMG
 * preconditioner.  Runs `reps` V-cycles on the solver's current residual after one
 * untimed cycle, with a CUDA event on `stream` before every kernel, and reports each
 * kernel of one cycle in launch order: its level, its kind (GIPB200_CYCLE_*), its mean
 * time in ms and its algorithmic bytes (stored operator words once, every vector read
 * or written once).  At most `cap` kernels are written; *n_kernels = kernels per cycle.
 * Leaves the solution untouched; solve once first so the residual is set. */
enum {
  GIPB200_CYCLE_JACOBI0 = 0,   /* x = D^-1 b (pre-smoothing from zero)           */
  GIPB200_CYCLE_RESIDUAL = 1,  /* t = b - A x                                    */
  GIPB200_CYCLE_RESTRICT = 2,  /* b_coarse = R t                                 */
  GIPB200_CYCLE_DENSE = 3,     /* coarsest level: x = A^-1 b (dense inverse)     */
  GIPB200_CYCLE_PROLONG = 4,   /* x += P x_coarse                                */
  GIPB200_CYCLE_SMOOTH = 5,    /* x + D^-1 (b - A x) (level 0: with r.z)         */
  GIPB200_CYCLE_TAIL = 6       /* the small levels and the coarsest, one launch  */
};
int gipb200_pcg_vcycle_profile(gipb200_pcg S, int reps, void* stream, int cap, int* n_kernels,
                               int* h_level, int* h_kind, double* h_ms, double* h_bytes);
/* The form each kernel of the last profiled cycle ran its product in (GIPB200_FORM_*), in
 * the same order; at most `cap` written, *n_kernels = kernels per cycle.
 * GIPB200_ERR_STATE before a profile. */
enum {
  GIPB200_FORM_PACKED = 0,     /* level 0 from the packed FP32 operator (k_amgp_spmv)     */
  GIPB200_FORM_SLICED = 1,     /* sliced, a lane per row (k_amg_spmv)                     */
  GIPB200_FORM_PIPELINED = 2,  /* sliced, software-pipelined (k_amg_spmv_pf)              */
  GIPB200_FORM_CSR = 3,        /* CSR, several lanes per row (k_amg_csr)                  */
  GIPB200_FORM_DENSE = 4,      /* dense inverse of the coarsest level (k_amg_dense)       */
  GIPB200_FORM_VECTOR = 5,     /* element-wise (k_amg_jacobi0)                            */
  GIPB200_FORM_TAIL = 6,       /* the coarse tail in one launch (k_amg_tail)              */
  GIPB200_FORM_SMOOTH_DOT = 7  /* level-0 smoothing with r.z, plain layout                */
};
int gipb200_pcg_vcycle_forms(gipb200_pcg S, int cap, int* n_kernels, int* h_form);

/* No counterpart in the reference.  A Jacobi-PCG solve for callers that cannot allocate
 * device memory at solve time (a framework-owned arena or caching allocator, code that
 * must not call cudaMalloc because it synchronises the device, embedders without
 * library handles).  The caller passes a device CSR operator (n rows), b (n), x and x0
 * (n_all = inner plus ghost cells, ghosts copied from x0), and d_stats (4 doubles out:
 * iterations, r.r, b.b, status).  mode: GIPB200_PCG_FIXED (exactly maxit iterations, as
 * GIP's solver) or GIPB200_PCG_TOL (stops on the device at tol; the host reads the stop
 * flag every 32 iterations, waiting on `stream` each time).  Every column index must be
 * below n_all; a row without a diagonal entry gets a zero Jacobi entry, as in
 * gipb200_pcg_solve.  The solver's vectors and reductions use one file-scope device array
 * of 8 MiB that every GPU loading the library keeps until exit: n_all above 262144 is
 * rejected with GIPB200_ERR_ARG.  All calls share that array, so calls that overlap on
 * the GPU race; serialise them.  Each call clears the array's reduction counter on its own
 * stream.  The first call on a device (with that device current) resolves the array's
 * address; make that first call before any stream capture. */
int gipb200_pcg_solve_static(int n, int n_all, const int* d_rowptr, const int* d_col,
                             const double* d_val, const double* d_b, double* d_x,
                             const double* d_x0, int mode, int maxit, double tol,
                             double* d_stats, void* stream);

/* Host-side setup of the AMG preconditioner alone (no counterpart in the reference, whose
 * solver is Jacobi-PCG; no device work, so it runs without a GPU): builds the hierarchy
 * that precond = GIPB200_PRECOND_AMG builds for the n x n host CSR operator (columns < n)
 * with near-null vector z (singular != 0: the operator annihilates z), coarse operators
 * sparsified at `drop` (0: plain Galerkin), and reports its first min(levels, max_levels)
 * levels: rows[l], nnz[l], and checks[3 l + 0..2] = max |a_ij - a_ji| / max |a| (1 when
 * the pattern is not symmetric), max |(A z)_i| / (max |a| max |z|), and the smallest
 * diagonal entry.  *levels = levels reported. */
int gipb200_amg_host_levels(int n, const int* rowptr, const int* col, const double* val,
                            const double* z, int singular, double drop, int max_levels,
                            int* levels, int* rows, long long* nnz, double* checks);

/* ------------------------------------------------------------------ timestep engine */
typedef struct gipb200_dns_s* gipb200_dns;

typedef struct {
  int nrows, ncols, nnz;
  const int* rowptr;
  const int* col;
  const double* val;
} gipb200_host_csr;

/* The operators GIP_DNS loads (src/Algorithms/GIP_DNS.h:143-238), host memory. */
typedef struct {
  gipb200_host_csr D, Ec, L, Lb, Mx, My, Mz, Mres, Gx, Gy, Gz, SFx, SFy, SFz, SO;
  int n_inner, n_owned, n_faces;
} gipb200_dns_ops;

typedef struct {
  double rho;                  /* GIP_DNS.h:133 (1.0)                             */
  double gamma;                /* GIP_DNS.h:137 (1/Re; enters only the CFL limit)  */
  gipb200_pcg_params pcg;      /* GIP_DNS.h:180-185 (FIXED, maxit 100)             */
  int use_graph;               /* capture each timestep in a CUDA graph            */
  int reorder;                 /* 1: renumber cells (breadth-first from a peripheral cell)
                                  and faces (by adjacent cell) inside the engine for
                                  gather locality; every row keeps its nonzero order, so
                                  each product is unchanged bit for bit.  Fields cross the
                                  API in the caller's numbering. */
} gipb200_dns_params;

/* GIP_DNS::setUp (GIP_DNS.h:116-125): uploads operators and the initial fields u,v,w,dxs
 * (n_owned each); every other GIP_DNS vector starts at 0, C's values at D's. */
int gipb200_dns_create(const gipb200_dns_ops* ops, const double* h_u, const double* h_v,
                       const double* h_w, const double* h_dxs, const gipb200_dns_params* params,
                       gipb200_dns* out);
int gipb200_dns_destroy(gipb200_dns E);
/* GIP_DNS::integrate (GIP_DNS.h:99-113): advances nsteps timesteps on `stream`; the first
 * call also computes the initial dt.  No host synchronisation inside. */
int gipb200_dns_advance(gipb200_dns E, int nsteps, void* stream);
/* Per-step history of all steps so far (host arrays of length >= steps taken, any may
 * be NULL): time, dt used, massr (GIP_DNS.h:399-404), PCG iterations (MIXED: FP32
 * iterations), final r.r, MIXED residual replacements (FP64 true-residual updates), and
 * the library kernels the step launched (kernels that found their solve finished and
 * returned at once included). */
int gipb200_dns_history(gipb200_dns E, int* steps_taken, double* h_time, double* h_dt,
                        double* h_massr, int* h_iters, double* h_rr, int* h_outer,
                        int* h_kernels);
/* Per-phase timing report (what a GIP_TimerB200 channel per phase would give): advances
 * one timestep with host-driven loops (no graph) and CUDA events on `stream` between
 * GIP_DNS's phases, and writes their durations in ms to h_ms[7]: predictor (Ec, D/C
 * products, AB2; GIP_DNS.h:309-338), Poisson right-hand side (:341-348), PCG, ghost copy
 * (:350-354), velocity correction (:357-376), mass fluxes (:379-391), massr and CFL
 * (:394-414).  The step is a real step (state and history advance). */
int gipb200_dns_step_phases(gipb200_dns E, void* stream, double* h_ms);
/* Per-phase timing of every step, graph-launched steps included (GIP_Timer channels per
 * phase, src/AbstractInterfaces/GIP_Timer.h, kept on the device): with `on` set, each
 * step also launches 8 one-thread kernels that store the device clock (%globaltimer, ns)
 * at the phase boundaries of gipb200_dns_step_phases; the captured step graph is rebuilt
 * at the next advance.  Off by default. */
int gipb200_dns_phase_stamps(gipb200_dns E, int on);
/* The 7 phase durations (ms, same order as gipb200_dns_step_phases) of the first
 * min(steps taken, max_steps) steps into h_ms[step * 7 + phase]; NaN for steps taken
 * with stamps off.  *steps_out (may be NULL) = steps written.  Synchronises the device. */
int gipb200_dns_phase_history(gipb200_dns E, int max_steps, double* h_ms, int* steps_out);
/* Copies a field to the host: "u","v","w","p","p0","mf","ax0","ay0","az0","gpx",... */
int gipb200_dns_get_field(gipb200_dns E, const char* name, double* h_out, int n);
/* Copies h_in[0:n) into a field at `offset` on `stream` (no host synchronisation; the
 * host buffer must stay valid until the stream reaches the copy).  Used to feed
 * boundary values (e.g. the lid's ghost velocities) between steps. */
int gipb200_dns_set_field(gipb200_dns E, const char* name, const double* h_in, int offset, int n,
                          void* stream);
/* Device pointer of a field (valid until destroy), in the engine's internal numbering
 * (the caller's numbering unless `reorder` is set). */
int gipb200_dns_field_ptr(gipb200_dns E, const char* name, double** d_ptr, int* n);
/* Device-to-device copy of a field in the caller's numbering, on `stream`. */
int gipb200_dns_copy_field(gipb200_dns E, const char* name, double* d_out, int n, void* stream);
/* GIP_DNS's `time` member (GIP_DNS.h:400): sets the engine's simulated time, so an engine
 * built from a GIP_DNS state continues GIP's clock; ordered on `stream`, returns once the
 * value is on the device. */
int gipb200_dns_set_time(gipb200_dns E, double time, void* stream);
/* Current dt, sigma=1/dt and simulated time. */
int gipb200_dns_scalars(gipb200_dns E, double* dt, double* sigma, double* time);

typedef struct {
  int reordered;               /* engine runs in its breadth-first numbering            */
  int pin_row;                 /* MIXED: detected pinned-Neumann row of L (-1: none)     */
  int compressed;              /* MIXED: FP32 operator stored compressed                 */
  int value_table;             /* MIXED: bits of a packed row's value-table index (4, 8) */
  double compressed_fraction;  /* MIXED: share of L's slots in packed slices             */
  long long slots_L;           /* sliced slots of L (stored nonzeros plus padding)       */
  long long nnz_L;
  int amg_levels;              /* AMG: levels of the hierarchy (0: no AMG)               */
  double amg_complexity;       /* AMG: operator nonzeros of all levels / of the finest    */
  double amg_setup_s;          /* AMG: host setup time                                   */
  double iteration_bytes;      /* algorithmic bytes of one PCG iteration (with V-cycle)   */
  double replacement_bytes;    /* MIXED: bytes of one FP64 residual replacement           */
  int packed_residual;         /* MIXED: FP64 residual from the packed columns (1) or L   */
  int value_tables;            /* phase kernels (of 4: D/C products, right-hand side,     */
                               /* massr, C's values) reading their operators' values      */
                               /* through 8-bit value tables                              */
} gipb200_dns_info;
int gipb200_dns_get_info(gipb200_dns E, gipb200_dns_info* info);

/* Device-side checkpoint of the whole timestep state (every GIP_DNS vector, C's values,
 * dt, sigma, time, step counter): restore = 0 saves, 1 restores the last save.  Steps
 * taken after a restore overwrite the history from the saved step on. */
int gipb200_dns_snapshot(gipb200_dns E, int restore, void* stream);

/* Launch shape of the PCG kernels (SpMV+dot grid, vector-kernel grid; 0 = default,
 * at most 8192 blocks of 256 threads).  A different shape changes the order of the
 * dot-product partial sums (results stay deterministic for a given shape).  The next
 * step re-captures its graph. */
int gipb200_dns_set_launch(gipb200_dns E, int spmv_blocks, int vec_blocks);

/* Algorithmic bytes of each phase of one timestep, in the order of
 * gipb200_dns_step_phases (h_bytes[7]; stored operator values and indices once, gathered
 * vectors once, written vectors once).  The PCG entry is 0: a solve moves iterations x
 * iteration_bytes plus replacements x replacement_bytes (gipb200_dns_get_info). */
int gipb200_dns_phase_bytes(gipb200_dns E, double* h_bytes);
/* Host seconds the engine's creation took: h_seconds[0] checks and renumbering, [1] the
 * operators' device layouts and the fields, [2] the pressure solver (FP32 operator,
 * packing, AMG hierarchy), [3] the whole of gipb200_dns_create. */
int gipb200_dns_setup_profile(gipb200_dns E, double* h_seconds);
/* gipb200_pcg_vcycle_profile for the engine's pressure solver (precond = AMG). */
int gipb200_dns_vcycle_profile(gipb200_dns E, int reps, void* stream, int cap, int* n_kernels,
                               int* h_level, int* h_kind, double* h_ms, double* h_bytes);
/* gipb200_pcg_vcycle_forms for the engine's pressure solver. */
int gipb200_dns_vcycle_forms(gipb200_dns E, int cap, int* n_kernels, int* h_form);

/* Number of this library's kernels the engine has launched so far (a graph launch counts
 * the kernels it holds). */
int gipb200_dns_launch_count(gipb200_dns E, long long* count);

enum {
  GIPB200_KERNEL_PCG_SPMV_DOT = 0,   /* FP64 PCG: Ap = L p fused with p.Ap              */
  GIPB200_KERNEL_MIXED_SPMV_DOT = 1, /* FP32 inner PCG: Ap = (S L S) p fused with p.Ap  */
  GIPB200_KERNEL_MIXED_UPDATE = 2    /* FP32 inner PCG: y += alpha p, r -= alpha Ap, r.r */
};
/* Times `reps` back-to-back launches of one PCG kernel on the engine's resident operator
 * with CUDA events on `stream`; returns the mean launch time and the kernel's compulsory
 * bytes per launch (stored values and indices read once, the vector read once, the
 * product written once).  Leaves the engine's fields untouched. */
int gipb200_dns_kernel_time(gipb200_dns E, int kernel, int reps, void* stream, double* avg_ms,
                            double* bytes);

/* ------------------------------------------------------------------ batched cavities */
/* No counterpart in the reference.  Many independent cases (uneven sizes, own Reynolds
 * numbers and parameters) advanced together: each timestep is one CUDA graph launch whose
 * parallel branches are the instances' steps; every branch keeps its own device-decided
 * PCG loops, so each instance stops at its own convergence (per-instance masks). */
typedef struct gipb200_batch_s* gipb200_batch;
int gipb200_batch_create(int n, const gipb200_dns_ops* const* ops, const double* const* h_u,
                         const double* const* h_v, const double* const* h_w,
                         const double* const* h_dxs, const gipb200_dns_params* params,
                         gipb200_batch* out);
int gipb200_batch_destroy(gipb200_batch B);
/* Instance i as an engine handle (history, fields, launch shape); owned by the batch. */
int gipb200_batch_instance(gipb200_batch B, int i, gipb200_dns* out);
/* nsteps timesteps of every instance, one graph launch each, on `stream`. */
int gipb200_batch_advance(gipb200_batch B, int nsteps, void* stream);
/* How the batch solves its pressure systems.  persistent = 0 (the default): inside each
 * instance's graph branch, as a single instance does.  persistent = 1: one cooperative
 * launch per timestep solves every instance's system, the launch's CTAs split into one
 * group per instance (shares set by gipb200_batch_balance); each group runs its instance's
 * mixed-form Jacobi-PCG and leaves when that instance has converged.  Needs every instance
 * in GIPB200_PCG_MIXED with GIPB200_PRECOND_JACOBI.  block: threads per CTA (128, 256 or
 * 512); rows_per_warp: 32 (one 32-row slice per warp pass) or 64 (two slices in flight);
 * threads_per_sm: 1024 (64 registers a thread) or 1536 (40; 0 = 1024), the occupancy the
 * kernel is compiled for.
 * The step graph is captured again at the next advance. */
int gipb200_batch_set_solver(gipb200_batch B, int persistent, int block, int rows_per_warp,
                             int threads_per_sm);
/* CTA shares of the persistent solve: weights[i] >= 0 is instance i's expected work (for
 * example rows times iterations of the last step); null restores the default, rows times
 * the cube root of rows (Jacobi-PCG iterations grow with the grid edge).  Waits for the
 * device; a captured step graph keeps working (same grid, new tables). */
int gipb200_batch_balance(gipb200_batch B, const double* weights);
/* The persistent solve's grid and each instance's CTAs (h_ncta: one per instance, or
 * null); 0 when the batch solves inside its branches. */
int gipb200_batch_layout(gipb200_batch B, int* grid, int* h_ncta);
/* *h_err = nonzero when a group barrier of the persistent solve gave up waiting (about 2 s)
 * since the last call, which clears it; the instances' results are then not valid.
 * Synchronises `stream`. */
int gipb200_batch_solver_status(gipb200_batch B, void* stream, int* h_err);
/* Runs one persistent-solve launch whose group barrier waits for a CTA that does not exist:
 * *h_status = GIPB200_ERR_TIMEOUT when the wait gave up (about 2 s) and the kernel returned
 * with the error recorded, as designed; the context stays usable.  Synchronises `stream`. */
int gipb200_batch_check_bounded_wait(void* stream, int* h_status);

/* ------------------------------------------------------------------ discrete adjoint */
/* No counterpart in the reference (GIP has no derivatives).  FP64 discrete adjoint of
 * the timestep above with the CFL steps frozen: J = 1/2 sum_i vol_i |u_i|^2 over the
 * inner cells after `nsteps` steps; gradients with respect to the lid's ghost velocities
 * (u on the listed ghost cells) and the viscosity nu = nu_scale * nu0 (D scales with
 * nu).  The forward keeps checkpoints every `checkpoint_every` steps; the backward
 * recomputes each segment and applies the transposed step: transposed SpMVs over CSR
 * transposes built at creation, one adjoint Poisson solve per step with the same PCG
 * (L is symmetric), and the convective adjoint dJ/dmf = -Ec^T z. */
typedef struct gipb200_adjoint_s* gipb200_adjoint;

typedef struct {
  double rho;            /* density                                                  */
  double gamma;          /* CFL viscosity parameter (dt is frozen after the forward)  */
  double nu0;            /* viscosity baked into D                                    */
  double tol;            /* relative tolerance of every Poisson solve (forward, adjoint) */
  int maxit;             /* PCG iteration cap                                         */
  int checkpoint_every;  /* forward checkpoint spacing, in steps                      */
  int precond;           /* GIPB200_PRECOND_* of the forward and adjoint Poisson solves */
} gipb200_adjoint_params;

int gipb200_adjoint_create(const gipb200_dns_ops* ops, const double* h_u0, const double* h_v0,
                           const double* h_w0, const double* h_dxs, const double* h_volume,
                           const int* h_lid_cells, int n_lid, const gipb200_adjoint_params* prm,
                           gipb200_adjoint* out);
int gipb200_adjoint_destroy(gipb200_adjoint A);
/* Forward from the initial fields with the lid values applied.  dt_given = 1: use the
 * nsteps steps in h_dt; dt_given = 0: GIP's CFL chooses them and they are written to h_dt
 * when it is not NULL.  *h_J = kinetic energy after the last step. */
int gipb200_adjoint_forward(gipb200_adjoint A, const double* h_lid, double nu_scale, int nsteps,
                            double* h_dt, int dt_given, double* h_J);
/* Gradients of the last forward's J: h_grad_lid[n_lid], *h_grad_nu. */
int gipb200_adjoint_backward(gipb200_adjoint A, double* h_grad_lid, double* h_grad_nu);

#ifdef __cplusplus
}
#endif
#endif /* GIPB200_H */
