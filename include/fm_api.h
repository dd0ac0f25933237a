/*
 * fm_api.h — C ABI of the B200 FlexMesh hot path (libflexmesh_b200.so).
 *
 * One Newton iteration of FlexMesh's finite-strain solve, on one GPU:
 *   compressible Neo-Hookean force + 12x12 tangent per tetrahedron,
 *   scatter into a CSR global stiffness (no atomics: each CSR row block is
 *   written once by the warp that owns its node),
 *   Dirichlet elimination, ILU(0) factorization and ILU(0)-preconditioned CG
 *   (SpMV + dependency-ordered triangular solves), Newton load stepping,
 *   and the adjoint for per-element material gradients.
 *
 * Conventions
 *   - Plain C; no exceptions cross the boundary; every call returns fm_status.
 *   - Host arrays are caller-owned and only read/written during the call.
 *     Arguments named *_dev are device pointers on the context's device.
 *   - Node coordinates and DOF vectors are interleaved per node:
 *     xyz[3*n+d], u[3*n+d] (the reference's MeshNode order, DOF 3n+d).
 *     Connectivity is conn[4*e+v].
 *   - All device work is ordered on the context's stream; calls that return
 *     scalars (iteration counts, norms, status) synchronize that stream.
 *   - A context is not thread-safe; use one context per host thread.
 *   - Kernels never trap: device-side problems set a status word that the
 *     calls translate into FM_ERR_* codes (see fm_last_error for text).
 *
 * Every entry point cites the reference interface it replaces
 * (file:line in the FlexMesh sources).
 */
#ifndef FM_API_H
#define FM_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fm_ctx fm_ctx;

typedef enum {
    FM_OK = 0,
    FM_ERR_ARG = 1,            /* bad argument or call order */
    FM_ERR_CUDA = 2,           /* CUDA runtime error */
    FM_ERR_OOM = 3,            /* device allocation failed */
    FM_ERR_NONFINITE = 4,      /* NaN/Inf produced (element or solver) */
    FM_ERR_ZERO_PIVOT = 5,     /* reserved: pivots are perturbed, not fatal */
    FM_ERR_INVERTED = 6,       /* reserved: det F <= 0 is reported as a flag */
    FM_ERR_TIMEOUT = 7,        /* a bounded device wait expired */
    FM_ERR_NOT_CONVERGED = 8,  /* Newton/PCG stopped at its iteration cap */
    FM_ERR_LIMITS = 9,         /* mesh valence or size beyond the kernels' limits */
    FM_ERR_DIVERGED = 10       /* Newton stopped by the divergence test */
} fm_status;

typedef enum { FM_FP64 = 0, FM_MIXED = 1 } fm_precision;

/* FM_PATTERN_REFERENCE: the reference's CSR exactly as its builder writes it
 * (FEM/adaptive_fem_engine.hpp:1069-1120, including its column-fill defect).
 * FM_PATTERN_SOLVE: same row_ptr, every row of node n lists all 3|nb(n)|
 * columns ascending (the fill the Newton/PCG path needs). */
typedef enum { FM_PATTERN_REFERENCE = 0, FM_PATTERN_SOLVE = 1 } fm_pattern;

/* Device status flags accumulated since the last fm_clear_flags. */
enum {
    FM_FLAG_NONFINITE = 1u << 0, /* NaN/Inf in an element or solver value */
    FM_FLAG_INVERTED = 1u << 1,  /* det F <= 0 met in an element */
    FM_FLAG_J_CLAMPED = 1u << 2, /* det F < 0.01, ln J clamped as the reference does */
    FM_FLAG_PIVOT = 1u << 3,     /* an ILU(0) pivot was perturbed (|u_ii| < 1e-12) */
    FM_FLAG_TIMEOUT = 1u << 4,   /* a bounded dependency wait expired */
    FM_FLAG_BREAKDOWN = 1u << 5  /* PCG |p.Ap| < 1e-60 */
};

/* Kernel classes of the built-in profiler. */
enum {
    FM_PROF_ASSEMBLE = 0, /* element evaluation + CSR scatter (incl. residual-only) */
    FM_PROF_ILU = 1,      /* ILU(0) factorization */
    FM_PROF_TRSV = 2,     /* preconditioner apply: forward + backward solve */
    FM_PROF_SPMV = 3,     /* K x */
    FM_PROF_VECTOR = 4,   /* PCG/Newton vector updates and reductions */
    FM_PROF_STATES = 5,   /* element state update */
    FM_PROF_KINDS = 8
};
typedef struct {
    double ms[FM_PROF_KINDS];       /* device time per class (CUDA events, ms) */
    uint64_t calls[FM_PROF_KINDS];  /* launch groups per class */
    uint64_t kernels[FM_PROF_KINDS];/* kernel launches per class */
} fm_profile;

/* ---- context ----------------------------------------------------------- */
/* cuda_stream: a cudaStream_t, or NULL to let the context create its own. */
fm_status fm_create(fm_ctx** ctx, int device, void* cuda_stream);
void fm_destroy(fm_ctx* ctx);
/* Text of the last error on this context (always NUL-terminated). */
fm_status fm_last_error(const fm_ctx* ctx, char* buf, size_t len);
fm_status fm_get_flags(fm_ctx* ctx, uint32_t* flags);
/* After FM_ERR_TIMEOUT the flag also stops every later wait at once (so a
 * kernel whose dependency never arrives ends quickly): clear it before the
 * next solve. */
fm_status fm_clear_flags(fm_ctx* ctx);
/* Bounded device waits (no reference counterpart: the reference's solves are
 * serial loops).  Every dependency wait of the context's kernels (ILU(0)
 * factorization, triangular solves) gives up after `cycles` SM clock cycles
 * without progress, raises FM_FLAG_TIMEOUT and lets its kernel finish; the
 * call then returns FM_ERR_TIMEOUT and the context stays usable.  cycles is
 * rounded up to a multiple of 1024; 0 restores the default 2e9 cycles
 * (about 1 s at B200 clocks). */
fm_status fm_set_wait_limit(fm_ctx* ctx, uint64_t cycles);
/* Health check of that path: one warp waits, under the context's wait
 * limit, on a device flag that nothing sets, and the call returns
 * FM_ERR_TIMEOUT (FM_FLAG_TIMEOUT raised) once the limit has passed. */
fm_status fm_check_wait(fm_ctx* ctx);
/* Size queries after fm_set_mesh: DOFs, CSR nonzeros, node neighbours. */
fm_status fm_sizes(const fm_ctx* ctx, uint32_t* n_nodes, uint32_t* n_elems, uint32_t* n_dofs,
                   uint64_t* nnz);
/* Built-in profiler (no reference counterpart; the reference times whole
 * phases with wall clocks, FEM/adaptive_fem_engine.hpp:1251-1273).
 * Launch groups and kernel launches are always counted per class;
 * fm_profile_enable(ctx, on) zeroes all counters, and with on = 1 also
 * records a CUDA event pair around every kernel group launched afterwards
 * (device time per class).  fm_profile_read synchronizes the stream and
 * returns the totals. */
fm_status fm_profile_enable(fm_ctx* ctx, int on);
fm_status fm_profile_read(fm_ctx* ctx, fm_profile* out);

/* ---- A1: unit-cube generator (host only) ---------------------------------
 * Replaces generate_unit_cube_mesh, FEM/adaptive_fem_engine.hpp:2219-2294:
 * (N+1)^3 nodes numbered k(N+1)^2 + j(N+1) + i, 6 tets per hex (one of them
 * the zero-volume sliver the reference's split contains). */
fm_status fm_unit_cube_sizes(int N, uint32_t* n_nodes, uint32_t* n_elems);
fm_status fm_unit_cube(int N, double* xyz, uint32_t* conn);

/* ---- mesh, pattern, material, boundary conditions (host arrays) ---------
 * fm_set_mesh replaces the MeshTopology hand-over to the assembly
 * (FEM/fem_types.hpp:168-211).  elem_volume, if given, is the stored
 * TetraElement::volume: elements with volume < 1e-30 are skipped exactly as
 * assemble_global_threadlocal skips them (FEM/adaptive_fem_engine.hpp:1169);
 * NULL uses |det J|/6 of the given coordinates.  Builds the node->tet
 * incidence, the node neighbour sets, the ILU(0) dependency levels and
 * schedules and the assembly's scatter structure on the device (the
 * reference builds its neighbour sets per node with std::set, :1076-1085),
 * and the triangular-solve plan on the host.  Clears the flags. */
fm_status fm_set_mesh(fm_ctx* ctx, uint32_t n_nodes, const double* xyz, uint32_t n_elems,
                      const uint32_t* conn, const double* elem_volume);

/* Replaces MeshColoring::compute (FEM/adaptive_fem_engine.hpp:1549-1602)
 * (host only): greedy first-fit element colouring in element order, tets
 * sharing a node get different colours; the same colours as the
 * reference's all-pairs construction in time linear in the incidences.
 * colors[n_elems]; *n_colors = 1 + the largest colour (0 for no tets). */
fm_status fm_mesh_coloring(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn,
                           uint32_t* colors, uint32_t* n_colors);

/* Replaces build_csr_sparsity_pattern_rigorous (FEM/adaptive_fem_engine.hpp:1069)
 * and the element->CSR lookup it feeds (:1141-1150).  Any output may be NULL.
 * row_ptr_out[n_dofs+1], col_idx_out[nnz], slot_map_out[n_elems*144] with
 * slot[e][(i*3+di)*12 + j*3+dj] = CSR index of (3n_i+di, 3n_j+dj); for the
 * reference pattern the last duplicate wins and missing entries are -1. */
fm_status fm_build_pattern(fm_ctx* ctx, fm_pattern kind, uint32_t* row_ptr_out,
                           uint32_t* col_idx_out, int32_t* slot_map_out);

/* Material, replaces ProblemDescriptor{E, nu} (FEM/fem_types.hpp:241-256) and
 * NeoHookeanParameters (FEM/constitutive_models.hpp:30-46).  E_elem (nullable)
 * gives a per-element Young's modulus with the global nu; mu and lambda are
 * derived per element as the reference derives them (:81-82). */
fm_status fm_set_material(fm_ctx* ctx, double E, double nu, const double* E_elem);
/* Per-element Lame parameters (independent mu_e, lambda_e, as the adjoint's
 * parameters); nu only enters the tangent's volumetric factor
 * lambda / (J max(1-2nu, 0.1)) (:170). */
fm_status fm_set_material_lame(fm_ctx* ctx, const double* mu_elem, const double* lambda_elem,
                               double nu);

/* Dirichlet data, replaces BoundaryConditions::dirichlet_bcs
 * (FEM/fem_types.hpp:258-264): dof_mask[n_dofs] (1 = constrained) and the
 * value at full load (NULL = all zero).  Elimination as in
 * FEM/nonlinear_solver.hpp:329-334, 388-396: constrained rows/columns of K
 * are zeroed with a unit diagonal and their residual entries are zero. */
fm_status fm_set_bc(fm_ctx* ctx, const uint8_t* dof_mask, const double* dof_value_full_load);

/* ---- A5: batched element kernel -------------------------------------------
 * Replaces tet_element_stiffness_rigorous (FEM/adaptive_fem_engine.hpp:511-701)
 * for n independent tets: x_dev[12n] (4 nodes xyz), u_dev[12n], E_dev[n];
 * outputs K_dev[144n] (row-major (i*3+p)*12 + j*3+q) and f_dev[12n]. */
fm_status fm_elements(fm_ctx* ctx, uint32_t n, const double* x_dev, const double* u_dev,
                      const double* E_dev, double nu, double* K_dev, double* f_dev);

/* ---- A10/A11/A12: assembly ------------------------------------------------
 * Replaces assemble_global_threadlocal (FEM/adaptive_fem_engine.hpp:1126-1233)
 * on the solve pattern.  K_vals_dev: nnz doubles (FM_FP64) or floats
 * (FM_MIXED), NULL = the context's own buffer (used by fm_ilu0/fm_pcg).
 * f_int_dev: n_dofs doubles (FP64 in both precisions), may be NULL.
 * apply_bc != 0 also eliminates the Dirichlet rows/columns in K. */
fm_status fm_assemble(fm_ctx* ctx, const double* u_dev, void* K_vals_dev, double* f_int_dev,
                      fm_precision prec, int apply_bc);
/* Same with host buffers (copies inside the call): the drop-in for callers
 * holding std::vector data.  K_vals_host: nnz doubles. */
fm_status fm_assemble_host(fm_ctx* ctx, const double* u_host, double* K_vals_host,
                           double* f_int_host);
/* Replaces assemble_global_residual_only (FEM/adaptive_fem_engine.hpp:990-1059). */
fm_status fm_residual(fm_ctx* ctx, const double* u_dev, double* f_int_dev);
/* Reference-pattern assembly (the reference's CSR with its fill defect,
 * last-duplicate-wins slot map), FP64, for structural parity only. */
fm_status fm_assemble_reference_pattern(fm_ctx* ctx, const double* u_dev, double* K_vals_dev,
                                        double* f_int_dev);

/* ---- A15: ILU(0) level sets (host arrays) ---------------------------------
 * True dependency levels of the solve pattern at DOF granularity:
 * depth_L(i) = 1 + max depth_L(j) over j < i in row i, depth_U likewise
 * from the bottom; rows of a level ascend.  (The reference's own schedule
 * is natural order, level[i] = i: FEM/adaptive_fem_engine.hpp:327-349.)
 * fwd_ptr/bwd_ptr need n_dofs+1 entries of room, *_rows n_dofs. */
fm_status fm_levels(fm_ctx* ctx, uint32_t* fwd_ptr, uint32_t* fwd_rows, uint32_t* bwd_ptr,
                    uint32_t* bwd_rows, uint32_t* n_fwd, uint32_t* n_bwd);

/* ---- A13/A14: ILU(0) factorization of the context's K ---------------------
 * Replaces ILU0Preconditioner::factorize (FEM/adaptive_fem_engine.hpp:305-470);
 * same values as the reference's natural-order Doolittle elimination with
 * pivot perturbation (|u_ii| < 1e-12 -> +-1e-8).  Export with fm_get_ilu0. */
fm_status fm_ilu0(fm_ctx* ctx, fm_precision prec);
/* Copies out LU (L multipliers on lower slots, U on upper slots, the matrix
 * value on the diagonal slot as the reference's U_val keeps it) and pivots. */
fm_status fm_get_ilu0(fm_ctx* ctx, double* LU_host, double* diag_host);
/* Replaces ILU0Preconditioner::solve (:473-504): y = U^-1 L^-1 r. */
fm_status fm_ilu0_apply(fm_ctx* ctx, const double* r_dev, double* y_dev);
/* No counterpart in the reference.  fm_ilu0_apply for callers that must not
 * allocate device memory during the call (an application whose HBM belongs
 * to another allocator, where a cudaMalloc can fail, or that cannot take
 * the device-wide synchronization of cudaFree): the intermediate L^-1 r and
 * the wait-status word live in one file-scope device array of the library
 * (FM_NOALLOC_MAX_DOFS doubles = 8 MiB, held by every GPU that loads the
 * library until exit), not in context buffers.  Meshes with more than
 * FM_NOALLOC_MAX_DOFS DOFs are rejected with FM_ERR_LIMITS.  The first call
 * on a device looks the array up (cudaGetSymbolAddress, with that device
 * made current for the lookup and the caller's current device restored).
 * Every context on a device shares the array: calls that overlap on the GPU
 * race, so issue one at a time per device.  Output is bit-identical to
 * fm_ilu0_apply's.  Every call synchronizes the context's stream to read the
 * wait status, so no call can be made while that stream is capturing. */
#define FM_NOALLOC_MAX_DOFS (1u << 20)
fm_status fm_ilu0_apply_noalloc(fm_ctx* ctx, const double* r_dev, double* y_dev);

/* ---- A17/A18: SpMV and PCG on the context's K -----------------------------
 * fm_spmv replaces SparseCSR::matvec (FEM/fem_types.hpp:310-319).
 * fm_pcg replaces pcg_solve_ilu0 (FEM/adaptive_fem_engine.hpp:1283-1341) with
 * the same stop tests; the factorization from fm_ilu0 is reused (call
 * fm_ilu0 first, as the reference refactors on entry).  *iters = iterations
 * (max_iter when not converged), *relres = sqrt(r.z / b.b) at exit. */
fm_status fm_spmv(fm_ctx* ctx, const double* x_dev, double* y_dev);
fm_status fm_pcg(fm_ctx* ctx, const double* b_dev, double* x_dev, double tol, int max_iter,
                 int* iters, double* relres, fm_precision prec);

/* ---- generic CSR PCG-ILU(0) (host arrays) ---------------------------------
 * Drop-in for pcg_solve_ilu0(const SparseCSR&, b, x, N, tol, max_iter)
 * (FEM/adaptive_fem_engine.hpp:1283) on any square CSR matrix (columns in any
 * order; ILU works on the sorted pattern as the reference's symbolic phase
 * does).  x is in/out. */
fm_status fm_csr_pcg_ilu0(fm_ctx* ctx, uint32_t n, const uint32_t* row_ptr,
                          const uint32_t* col_idx, const double* val, const double* b, double* x,
                          double tol, int max_iter, int* iters, double* relres);

/* Drop-in for ILU0Preconditioner::factorize on any CSR (host arrays):
 * LU_out[nnz] in the caller's column order (L multipliers on lower slots,
 * U on upper, a_ii kept on the diagonal slot), diag_out[n] the pivots. */
fm_status fm_csr_ilu0(fm_ctx* ctx, uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                      const double* val, double* LU_out, double* diag_out);

/* ---- A19/A20: Newton load stepping ----------------------------------------
 * fm_newton_step: one load level (NonlinearNewtonSolver::solve(u, load, cfg),
 * FEM/nonlinear_solver.hpp:87): constrained DOFs of u are set to
 * load_frac * value, then Newton iterations run until
 * ||R|| < newton_rtol ||R_0|| or ||R|| < newton_atol (R_0: first iteration
 * of this call).  line_search > 0 enables Armijo backtracking on ||R||
 * (accept alpha when ||R(u + alpha du)|| <= (1 - ls_c alpha) ||R(u)||,
 * alpha halved up to line_search times; FEM/adaptive_fem_engine.hpp:933-985
 * with ls_c = 1e-4, FEM/nonlinear_solver.hpp:156-187 with ls_c = 0.1).
 * Equals fm_newton_step_cfg with fm_newton_config_default's divergence test
 * (growth > 10x stops with FM_ERR_DIVERGED; the slow-rate count is off),
 * predictor_tol = inner_tol and the line search given here. */
fm_status fm_newton_step(fm_ctx* ctx, double* u_dev, double load_frac, double newton_rtol,
                         double newton_atol, double inner_tol, int max_newton, int max_pcg,
                         int line_search, double ls_c, fm_precision prec, int* newton_iters,
                         int* pcg_iters, double* final_relres);

/* Host-buffer form of fm_newton_step: u_host (n_dofs doubles, in/out) is
 * copied to the device, solved and copied back inside the call - the shape
 * of NonlinearNewtonSolver::solve(Solution& u, ...) whose Solution is a
 * host std::vector<double>. */
fm_status fm_newton_step_host(fm_ctx* ctx, double* u_host, double load_frac, double newton_rtol,
                              double newton_atol, double inner_tol, int max_newton, int max_pcg,
                              int line_search, double ls_c, fm_precision prec, int* newton_iters,
                              int* pcg_iters, double* final_relres);

/* ---- Newton configuration, result and per-iteration history ---------------
 * fm_newton_config gathers NewtonSolverConfig (FEM/nonlinear_solver.hpp:23-34)
 * and the Newton fields of AdaptiveFEMEngine::Config
 * (FEM/adaptive_fem_engine.hpp:2306-2324); fm_newton_config_default fills
 * the defaults below.
 *   predictor_tol  PCG tolerance of the load step's Dirichlet predictor
 *                  solve (<= 0: inner_tol).  The predictor carries the whole
 *                  prescribed increment into the body, so an inexact
 *                  predictor leaves it in the elements next to the loaded
 *                  face.
 *   line_search    Armijo backtracking as armijo_line_search_true
 *                  (FEM/adaptive_fem_engine.hpp:933-985): alpha = 1, 1/2, ...
 *                  accepted when ||R(u + alpha du)|| <= (1 - ls_c alpha)
 *                  ||R(u)|| + 1e-14, at most line_search trials; when none
 *                  is accepted alpha = 2^-line_search ("best effort").
 *   divergence     the reference's test (:2561-2572): from the fourth
 *                  iteration on, rate = ||R|| / ||R_prev||; rate >
 *                  diverge_rate counts a slow iteration; stop when more than
 *                  diverge_count were slow or when ||R|| > diverge_growth *
 *                  ||R_prev||.  diverge_rate <= 0 or diverge_growth <= 0
 *                  turns that half off.  Where the reference breaks out of
 *                  the load step silently, the call returns FM_ERR_DIVERGED.
 *   inner_tol_min  > 0: when an iteration fails to reduce ||R|| by
 *                  diverge_rate the next corrections use a 10x tighter inner
 *                  tolerance, down to inner_tol_min (no reference
 *                  counterpart: the reference's inner solve is tight). */
/* Defaults (fm_newton_config_default): newton_rtol 1e-10, newton_atol 0,
 * inner_tol 1e-12, predictor_tol 0 (= inner_tol), inner_tol_min 0 (off),
 * max_newton 200, max_pcg 5000, line_search 10 with ls_c 1e-4 (the engine's
 * armijo_line_search_true(..., line_search_c = 1e-4, 10), :2314, :2581),
 * diverge_rate 0 (off), diverge_count 3, diverge_growth 10, FP64, ilu_every 1,
 * initial_guess 0. */
typedef struct {
    double newton_rtol;    /* stop when ||R|| < newton_rtol ||R_0|| */
    double newton_atol;    /* ... or ||R|| < newton_atol */
    double inner_tol;      /* PCG tolerance of the Newton corrections */
    double predictor_tol;  /* PCG tolerance of the Dirichlet predictor (<= 0: inner_tol) */
    double inner_tol_min;  /* adaptive inner tolerance floor (<= 0: fixed inner_tol) */
    int max_newton;        /* Newton iterations per load step (predictor included) */
    int max_pcg;           /* PCG iterations per solve */
    int line_search;       /* Armijo trials (0: full steps) */
    double ls_c;           /* Armijo constant */
    double diverge_rate;   /* slow-iteration rate (reference 0.9; <= 0: off) */
    int diverge_count;     /* slow iterations tolerated (reference 3) */
    double diverge_growth; /* growth factor that stops at once (reference 10; <= 0: off) */
    int precision;         /* fm_precision */
    int ilu_every;         /* refactorize the ILU(0) preconditioner at every ilu_every-th
                              solve of a load step (1: every solve, as pcg_solve_ilu0
                              does; k > 1: an earlier tangent's factors precondition
                              the current tangent, which PCG still solves) */
    int initial_guess;     /* mixed precision: 1 starts each Newton correction's PCG from
                              gamma x_prev, the previous correction (per ||R||) scaled by
                              the energy-norm projection gamma = x_prev.b / x_prev.K x_prev;
                              0 starts from zero as pcg_solve_ilu0's callers do.  FP64
                              ignores it: its PCG keeps the reference's absolute early
                              exit (||b - A x0|| < tol 1e-3) on the unscaled R, which a
                              good x0 would trigger before any iteration */
} fm_newton_config;

typedef struct {
    int newton_iters;      /* predictor + Newton iterations */
    int pcg_iters;         /* PCG iterations over all solves */
    int backtracks;        /* Armijo halvings over all iterations */
    uint32_t flags;        /* device flags (FM_FLAG_*) at exit */
    double rnorm0;         /* ||R_0||: the predictor's right-hand side, else the first ||R|| */
    double rnorm;          /* ||R|| at exit */
    double final_relres;   /* rnorm / rnorm0 */
} fm_newton_result;

/* One entry per solve of the latest fm_newton_step(_cfg) call on the
 * context, the data the reference prints per Newton iteration
 * (FEM/adaptive_fem_engine.hpp:2548-2550).  kind 0: the Dirichlet
 * predictor (rnorm = norm of its right-hand side), 1: a Newton iteration. */
typedef struct {
    int kind;
    int pcg_iters;
    double rnorm;          /* ||R|| before the solve (free DOFs) */
    double alpha;          /* step length taken */
    double inner_tol;      /* PCG tolerance used */
    uint32_t flags;        /* device flags after this iteration's assembly */
    uint32_t pad;
} fm_newton_record;

fm_status fm_newton_config_default(fm_newton_config* cfg);
/* fm_newton_step with a configuration; result (nullable) filled on every
 * return, also on FM_ERR_NOT_CONVERGED / FM_ERR_DIVERGED / FM_ERR_NONFINITE. */
fm_status fm_newton_step_cfg(fm_ctx* ctx, double* u_dev, double load_frac,
                             const fm_newton_config* cfg, fm_newton_result* result);
/* Host-buffer form of fm_newton_step_cfg (u_host copied in and out inside
 * the call, as fm_newton_step_host). */
fm_status fm_newton_step_cfg_host(fm_ctx* ctx, double* u_host, double load_frac,
                                  const fm_newton_config* cfg, fm_newton_result* result);
/* Copies up to cap records of the latest Newton call; *count = records kept
 * (at most 4096 per call). */
fm_status fm_newton_history(const fm_ctx* ctx, fm_newton_record* out, int cap, int* count);

/* fm_newton_step_cfg over load steps first_step..n_load_steps (load
 * fraction s / n_load_steps); result totals the counts, its norms are the
 * last step's.  A step that hits max_newton does not stop the path (the
 * call returns FM_ERR_NOT_CONVERGED at the end); any other error does. */
fm_status fm_newton_solve_cfg(fm_ctx* ctx, double* u_dev, int first_step, int n_load_steps,
                              const fm_newton_config* cfg, fm_newton_result* result);

/* fm_newton_solve: load steps first_step..n_load_steps of a load path.
 * Replaces NonlinearNewtonSolver::solve (FEM/nonlinear_solver.hpp:87-238)
 * with the engine's mathematics (FEM/adaptive_fem_engine.hpp:2476-2592):
 * for load step s = 1..n_load_steps the constrained DOFs of u are set to
 * (s/n) * value; then repeat {assemble, eliminate, R = -f_int,
 * stop when ||R|| < newton_rtol * ||R at the step's first iteration||
 * (or < newton_atol), ILU(0), PCG to inner_tol, u += alpha du with the
 * engine's Armijo line search (10 trials, c = 1e-4, :2581)}.
 * FM_MIXED: tangent, ILU(0) and PCG in FP32; det F, ln J, f_int, R and u in
 * FP64 (the Newton loop is the iterative refinement).
 * newton_iters/pcg_iters (nullable) receive totals over all steps. */
fm_status fm_newton_solve(fm_ctx* ctx, double* u_dev, int first_step, int n_load_steps,
                          double newton_rtol, double newton_atol, double inner_tol,
                          int max_newton, int max_pcg, fm_precision prec, int* newton_iters,
                          int* pcg_iters, double* final_relres);

/* ---- element state update --------------------------------------------------
 * Replaces update_element_states_rigorous (FEM/adaptive_fem_engine.hpp:
 * 2716-2794).  For every tet whose reference Jacobian is invertible
 * (|det| >= 1e-30, as the reference tests it): F = I + grad u,
 * F_sl3 = sl3_retraction(F, 0) = exp(log F) rescaled to det 1
 * (CORE/lie_operator.cpp:300), and the Neo-Hookean Mandel stress of F_sl3
 * (neo_hookean_response, :79-129, with J = det F_sl3: the reference passes
 * an uninitialized J there, :2784-2785).  F_dev[9e .. 9e+8]: F_sl3 as
 * ElementState::F_data holds it; stress_dev[6e .. 6e+5]: Voigt (S11, S22,
 * S33, sqrt2 S12, sqrt2 S13, sqrt2 S23).  Other tets keep their values
 * (initialize them as ElementState::initialize does: F = I, stress = 0).
 * det_violations (nullable): tets with |det F_sl3 - 1| > 1e-8, the count of
 * RuntimeInvariantMonitor::check_sl3_element (CORE/lie_operator.hpp:244).
 * nonfinite (nullable): tets whose state is not finite (under node jitter
 * the split's sliver tets have a tiny nonzero reference Jacobian; the
 * reference updates them too and their F can overflow).  Neither count is
 * an error.  The engine's J2 return after it (:2109) is an empty stub and
 * not run. */
fm_status fm_element_states(fm_ctx* ctx, const double* u_dev, double* F_dev, double* stress_dev,
                            uint32_t* det_violations, uint32_t* nonfinite);
/* Attach state arrays to the Newton calls: with both non-NULL every
 * fm_newton_step(_cfg) / fm_newton_solve(_cfg) updates them after each
 * update of u (the predictor's and every Newton iteration's), as the
 * engine does after each Newton iteration (:2589).  NULL, NULL detaches. */
fm_status fm_set_state_output(fm_ctx* ctx, double* F_dev, double* stress_dev);

/* ---- restart files (host only) ---------------------------------------------
 * Replaces CheckpointFile::save / load (FEM/adaptive_fem_engine.hpp:
 * 1347-1452) with the same byte layout, so files interchange with the
 * reference's: header u32 load_step, adapt_iter, n_nodes, n_elements, n_dofs;
 * per node f64 x, y, z, u, v, w; per element u32 nodes[4], f64 volume,
 * jacobian_det, quality_metric; per element state f64 F[9], stress[6],
 * eps_plastic[6], kappa, gamma_p; then n_dofs f64 of the solution.
 * Array pointers are host arrays of the sizes the counts give; on save a
 * NULL array is written as ElementState::initialize / zero-filled values
 * (xyz, conn and, when n_dofs > 0, u are required); on load a NULL array is
 * skipped.  fm_checkpoint_header reads the five header words, so the
 * caller can size its arrays; fm_checkpoint_load then needs the same
 * counts in *ck.  I/O failures return FM_ERR_ARG. */
typedef struct {
    uint32_t load_step, adapt_iter;
    uint32_t n_nodes, n_elems, n_dofs;
    double* xyz;           /* 3 n_nodes: MeshNode x, y, z */
    double* node_disp;     /* 3 n_nodes: MeshNode u, v, w */
    uint32_t* conn;        /* 4 n_elems */
    double* volume;        /* n_elems */
    double* jacobian_det;  /* n_elems */
    double* quality;       /* n_elems */
    double* F;             /* 9 n_elems: ElementState::F_data */
    double* stress;        /* 6 n_elems */
    double* eps_plastic;   /* 6 n_elems */
    double* kappa;         /* n_elems */
    double* gamma_p;       /* n_elems */
    double* u;             /* n_dofs */
} fm_checkpoint;
fm_status fm_checkpoint_save(const char* path, const fm_checkpoint* ck);
fm_status fm_checkpoint_header(const char* path, fm_checkpoint* ck);
fm_status fm_checkpoint_load(const char* path, fm_checkpoint* ck);

/* ---- A9/A21: exact Jacobian and adjoint (no reference counterpart) --------
 * fm_exact_apply: y = K_exact v (transpose = 0) or K_exact^T v (1), the
 * derivative of the element forces f_int(u) at u (not the reference's
 * heuristic tangent), matrix-free.
 * fm_adjoint: at a converged u solves K_exact^T w = dL/du on the free DOFs
 * (defect correction preconditioned by the reference tangent's ILU(0)-PCG)
 * and writes dL/dmu_e = -w_e . df_e/dmu_e and dL/dlambda_e likewise
 * (L depends on u only; the residual is R = f_ext - f_int).
 * w_dev (nullable) receives the adjoint vector. */
fm_status fm_exact_apply(fm_ctx* ctx, const double* u_dev, const double* v_dev, double* y_dev,
                         int transpose);
fm_status fm_adjoint(fm_ctx* ctx, const double* u_dev, const double* dLdu_dev,
                     double* dLdmu_dev, double* dLdlambda_dev, double* w_dev, double tol,
                     double inner_tol, int max_sweeps, fm_precision prec, int* sweeps,
                     int* pcg_iters);

#ifdef __cplusplus
}
#endif
#endif /* FM_API_H */
