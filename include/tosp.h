/*
 * tosp.h - C ABI of the B200 (sm_100a) equilibrium-solve library for
 * TopOpt-SLP-3D ("tosp").
 *
 * The entry points replace, one for one, the MATLAB functions on the
 * reference's per-iteration solve path.  Paths are relative to the reference
 * project; "I/" abbreviates its "Implementation/" folder.  A MEX gateway keeps
 * the MATLAB names and argument lists; heavy MATLAB arguments (A, P, M, R,
 * perm, kv, W) become state held by an opaque handle.
 *
 * Conventions
 *   - Node numbering, dof numbering and element order are the reference's:
 *     node = (z*nx + x)*ny + y (y is the vertical axis), dof = 3*node + c.
 *   - Index arrays crossing the ABI are 1-based int64 (MATLAB convention).
 *   - Vectors are float64.  Every pointer argument may be host memory or CUDA
 *     device memory of the handle's device (detected per call); device
 *     pointers avoid host<->device copies.  Device memory of another GPU is
 *     refused with TOSP_ERR_BAD_ARG.
 *   - Every call returns a status code (TOSP_OK = 0); tosp_last_error() gives
 *     the message of the last failing call on a handle.
 *   - Calls on one handle are serialised on that handle's CUDA stream and
 *     return after their results are written.  Distinct handles are
 *     independent and may be used from different host threads.
 */
#ifndef TOSP_H
#define TOSP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------- */
#define TOSP_OK               0
#define TOSP_NOT_CONVERGED    1   /* iteration cap reached (the reference returns silently) */
#define TOSP_ERR_BAD_ARG     -1
#define TOSP_ERR_CUDA        -2
#define TOSP_ERR_OOM         -3   /* device allocation failed / over the HBM budget */
#define TOSP_ERR_BREAKDOWN   -4   /* non-finite or non-positive curvature in CG */
#define TOSP_ERR_UNSUPPORTED -5
#define TOSP_ERR_STATE       -6   /* call order: e.g. solve before setup */
#define TOSP_ERR_CANCELLED   -7
#define TOSP_ERR_TIMEOUT     -8

/* ---- precision of the multigrid preconditioner ------------------------ */
#define TOSP_PREC_FP64   0   /* every level in FP64 (the reference's arithmetic) */
#define TOSP_PREC_MIXED  1   /* V-cycle in FP32 with BF16 SIMP factors; outer CG,
                                 coarsest solve, Grad and filter in FP64 */

typedef struct tosp_handle tosp_handle;

/* The fields of the reference's `str` struct used on the solve path
 * (I/EnterData.m, I/StartMR.m) plus the SIMP/filter scalars that StrSLP
 * passes to GlobalStiffMatrix/KelemProd/Grad/ApplyFilter. */
typedef struct tosp_problem {
    int32_t nelx, nely, nelz;      /* str.nelx/nely/nelz (displacement mesh)        */
    double  el, eh, ew;            /* str.el/eh/ew element sizes                    */
    double  E, nu;                 /* str.E, str.nu                                  */
    double  p, emin;               /* SIMP exponent, void Young's modulus           */
    int32_t mr_n;                  /* mr.n density sub-elements per direction (1 = mr.op false) */
    int32_t opfilter;              /* 0 none, 1 Gaussian, 2 hat (I/ElemNeighborhood.m) */
    double  rmin;                  /* filter radius, physical units                 */
    const int64_t *freedofs;       /* str.freedofs, 1-based, ascending              */
    int64_t nfree;
    const int64_t *fixed_dens;     /* fixed elements of the density (= design) mesh, 1-based; may be NULL */
    int64_t nfixed_dens;
    const int64_t *free_dens_g;    /* str.freeDensG: displacement elements with sensitivities,
                                      1-based; NULL = all elements                   */
    int64_t nfree_dens_g;
} tosp_problem;

/* mg.* fields of I/TopOpt3D.m:171-190 used by the geometric multigrid. */
typedef struct tosp_mg_params {
    int32_t ngrids;        /* mg.ngrids (raised by the nmaxchol rule like I/StartStrSLP.m:123-133) */
    int32_t cycle;         /* 0 V, 1 W, 2 full-multigrid V (mg.cycle)                  */
    int32_t smoother;      /* 0 damped Jacobi (the only smoother of the matrix-free path) */
    double  omega;         /* mg.omega                                                 */
    int32_t smoothiter1;   /* pre-smoothing sweeps                                     */
    int32_t smoothiter2;   /* post-smoothing sweeps                                    */
    double  tolMG;         /* relative residual tolerance                             */
    int32_t maxiterMG;     /* iteration cap                                            */
    int32_t nmaxchol;      /* largest coarsest-grid system for the direct solve        */
    int32_t flexible;      /* 0: beta = rho/rho_old as in I/SolveMG.m:43-46 (default);
                              1: flexible (Polak-Ribiere) beta = r'(s - s_old)/rho_old,
                              robust to a preconditioner that varies between applications
                              (FP32 V-cycle with atomics)                                    */
    int32_t maxstall;      /* 0: off (the reference runs to maxiterMG); k > 0: stop with
                              TOSP_NOT_CONVERGED when the best relative residual has not
                              halved within k iterations (used by the serving loop to fall
                              back from a stalling mixed-precision solve)                    */
    int32_t warp_stencil_max; /* coarse levels with at most this many nodes store their 27-point
                              stencil node-major and apply it with one warp per node (small
                              levels are latency-bound with one thread per node); 0: 65536,
                              -1: never.  A tuning knob with no reference counterpart.       */
    int32_t small_cycle_max; /* 0: off (default); k > 0: V/W cycles below the first coarse level
                              with at most k nodes run as one persistent cooperative kernel
                              (one launch per visit instead of one per sweep and transfer).
                              Measured slower than the graph-replayed launches on a B200, so
                              off by default.  A tuning knob with no reference counterpart.   */
    int32_t cg_product;    /* product K d of the CG recurrence (I/SolveMG.m:37-38):
                              0: FP64 operator every iteration (default, the reference's PCG);
                              1 (TOSP_PREC_MIXED with the tensor-core operator, n * nely even):
                              the tensor-core operator with FP32 SIMP factors and the blocks
                              in three FP16 pieces (about 1e-7 of |K||d|), every CG vector,
                              dot and update still FP64;
                              the recurrence residual is replaced by the FP64 residual
                              f - K u (FP64 operator) whenever its norm has fallen by the
                              factor replace_drop since the last replacement, and before
                              convergence is accepted, so the tolerance holds for the true
                              residual.  Served FP64 requests ignore it.                       */
    double  replace_drop;  /* replacement factor of cg_product 1, in (0, 1); 0: 0.1            */
    int32_t opchol;        /* mg.opchol: 0 (default) add grids while the coarsest system exceeds
                              nmaxchol and solve it directly; 1 PCG on the coarsest grid
                              (I/VCycle.m:28-35).  With 0, a coarsest system above nmaxchol
                              on a mesh that cannot take another grid switches to 1, as
                              I/StartStrSLP.m:122-132 does.                                  */
    int32_t opcond;        /* mg.opcond, the coarsest PCG's preconditioner in the reference
                              (0 diag, 1 ichol); the GPU PCG always uses the diagonal
                              (Jacobi) preconditioner and stops on the same tolerance        */
    double  tolPCG;        /* pcgp.tolPCG: the coarsest PCG's relative residual tolerance     */
    int32_t maxiterPCG;    /* pcgp.maxiterPCG: its iteration cap                              */
} tosp_mg_params;

/* Statistics of the last tosp_solve_mg call. */
typedef struct tosp_solve_stats {
    int32_t it;            /* the reference's `it` (iterations + 1)                   */
    double  relres;        /* final ||f - K u|| / ||f|| as tracked by CG (cg_product 1:
                              computed with the FP64 operator)                        */
    double  ms_setup;      /* device time of the last setup (tosp_setup_gmg)          */
    double  ms_solve;      /* device time of the last solve                           */
    int32_t replacements;  /* cg_product 1: residual replacements (FP64 products)     */
} tosp_solve_stats;

/* Library version string. */
const char *tosp_version(void);

/* Fill *mg with the reference defaults of I/TopOpt3D.m:171-190 (W-cycle,
 * Jacobi, omega 0.5, 1+1 sweeps, tol 1e-8, 5000 iterations, nmaxchol 60000,
 * ngrids 3). */
void tosp_default_mg_params(tosp_mg_params *mg);

/* Create a solver for one problem on the current CUDA device.  Builds the
 * sub-element stiffness blocks (I/ElemStiffMatrixGQMR.m:1), the dof/density
 * maps (I/DegreesOfFreedom.m:1, I/StartMR.m:58-83), the filter weights
 * (I/ElemNeighborhood.m:1) and the multigrid geometry (I/SetupGMG.m:16-44).
 * `precision` is TOSP_PREC_FP64 or TOSP_PREC_MIXED. */
int tosp_create(const tosp_problem *prob, const tosp_mg_params *mg, int32_t precision,
                tosp_handle **out);

/* Free a handle and all its device memory. */
int tosp_destroy(tosp_handle *h);

/* Message of the last failing call on `h` (or of the last failing
 * tosp_create on this thread when h == NULL). */
const char *tosp_last_error(const tosp_handle *h);

/* Effective number of grids and coarsest-grid system size after the level rules. */
int tosp_info(const tosp_handle *h, int32_t *ngrids, int64_t *ncoarse, int64_t *device_bytes);

/* Replace the free dofs (and the load vector's support) after Elem2Fix fixes
 * displacements: replaces the resetup of I/StrSLP.m:196-203.  The hierarchy is
 * rebuilt by the next tosp_setup_gmg. */
int tosp_set_freedofs(tosp_handle *h, const int64_t *freedofs, int64_t nfree);

/* Densities -> K(rho) and the whole multigrid hierarchy.  Replaces
 * GlobalStiffMatrix (I/GlobalStiffMatrix.m:1) + SetupGMG (I/SetupGMG.m:1), the
 * Galerkin refresh of I/StrSLP.m:345-365 and SetupGMGWOK
 * (I/WOK/SetupGMGWOK.m:1).  `xfil` are the filtered densities on the density
 * mesh (length nelem*mr_n^3, reference element order). */
int tosp_setup_gmg(tosp_handle *h, const double *xfil, int64_t ndens);

/* y = K(rho) x on the free dofs: KelemProd (I/WOK/KelemProd.m:1). */
int tosp_kelem_prod(tosp_handle *h, const double *x, double *y, int64_t nfree);

/* y = K(rho) x evaluated by the finest-level operator of the mixed V-cycle
 * (FP32 vectors, BF16 SIMP factors; sub-cell block products on the tensor
 * cores when n * nely is even, CUDA cores otherwise).  No counterpart in the
 * reference: it exposes the preconditioner's operator for inspection and
 * tests.  TOSP_PREC_MIXED handles only (TOSP_ERR_STATE otherwise); x and y are
 * FP64 on the free dofs. */
int tosp_kelem_prod_mixed(tosp_handle *h, const double *x, double *y, int64_t nfree);

/* y = K(rho) x by the product of the CG recurrence of mg.cg_product 1: the
 * tensor-core operator with FP32 SIMP factors and FP32 vectors.  No
 * counterpart in the reference (inspection and tests); handles created with
 * cg_product 1 only (TOSP_ERR_STATE otherwise); x and y are FP64 on the free
 * dofs. */
int tosp_kelem_prod_cg32(tosp_handle *h, const double *x, double *y, int64_t nfree);

/* One preconditioner application s = cycle(r) (VCycle/WCycle/FMVCycle,
 * I/VCycle.m:1, I/WCycle.m:1, I/FMVCycle.m:1) on free-dof vectors. */
int tosp_mg_cycle(tosp_handle *h, const double *r, double *s, int64_t nfree);

/* MG-preconditioned CG: SolveMG (I/SolveMG.m:1) / SolveMGWOK
 * (I/WOK/SolveMGWOK.m:1).  `x` is the warm start on entry and the solution on
 * exit; `f` the load on the free dofs; *it receives the reference's `it`.
 * Returns TOSP_NOT_CONVERGED (results still written) at the iteration cap. */
int tosp_solve_mg(tosp_handle *h, double *x, const double *f, int64_t nfree,
                  int32_t *it, double *relres);

/* Compliance sensitivities followed by the transposed filter: Grad
 * (I/Grad.m:1) / GradWOK (I/WOK/GradWOK.m:1).  `u` is the displacement on all
 * 3*nnodes dofs; `fgrad` has one entry per density element.  The densities
 * are those of the last tosp_setup_gmg.  `fgrad0` (may be NULL) receives the
 * unfiltered sensitivities. */
int tosp_grad(tosp_handle *h, const double *u, int64_t nfull, double *fgrad, double *fgrad0,
              int64_t ndens);

/* Filter: ApplyFilter (I/ApplyFilter.m:1) / ApplyFilterWOK
 * (I/WOK/ApplyFilterWOK.m:1); trans = 0: (W x)./w, trans = 1: W'(x./w). */
int tosp_apply_filter(tosp_handle *h, const double *x, double *y, int64_t ndens, int32_t trans);

/* Row sums w of the filter matrix (the `w` of I/ElemNeighborhood.m:181). */
int tosp_filter_weights(tosp_handle *h, double *w, int64_t ndens);

/* Compliance F = f' u on the free dofs (I/StrSLP.m:167,424), FP64. */
int tosp_compliance(tosp_handle *h, const double *f, const double *u, int64_t nfree, double *F);

/* Statistics of the last setup/solve on the handle. */
int tosp_last_stats(const tosp_handle *h, tosp_solve_stats *st);

/* Number of kernel launches this library has issued since it was loaded
 * (all handles).  Instrumentation for benchmarks. */
int64_t tosp_kernel_launches(void);

/* Time `reps` launches of the finest-level operator kernel on the handle's
 * stream with CUDA events bracketing each launch (inputs are the handle's
 * current vectors): `precision` TOSP_PREC_FP64 times the FP64 kernel of the
 * outer CG, TOSP_PREC_MIXED the FP32/BF16 kernel of the V-cycle (mixed
 * handles only), 2 the tensor-core kernel with FP32 factors of the CG's
 * product (cg_product 1 handles only).  Writes the mean device time per launch
 * in ms. */
int tosp_time_operator(tosp_handle *h, int32_t precision, int32_t reps, double *ms_per_launch);

/* Fault injection for tests of the bounded device waits (no counterpart in
 * the reference).  The next launches of the handle's persistent small-level
 * cycle (mg.small_cycle_max > 0) give up a grid-barrier wait after `polls`
 * polls (of 64 ns or more) instead of about 2^21, and when skip_block >= 0
 * that block skips its first barrier arrival, so the other blocks' waits run
 * out: the call then returns TOSP_ERR_TIMEOUT, the barrier state is reset and
 * the handle works normally again (the knob is cleared with it).  Nothing
 * faults, traps or waits without bound.  TOSP_ERR_STATE when the handle has
 * no persistent cycle. */
int tosp_inject_wait_fault(tosp_handle *h, int32_t polls, int32_t skip_block);

/* Blocks of the handle's persistent small-level cycle (0 when it has none). */
int tosp_small_cycle_blocks(const tosp_handle *h, int32_t *blocks);

/* KelemProd for callers that cannot allocate device memory at call time: a
 * host whose GPU memory belongs to its own pooling allocator (a MATLAB
 * gpuArray session), pipelines with work in flight on several streams, which
 * a cudaMalloc/cudaFree may synchronise, and services that fix their device
 * footprint at start-up.  No counterpart in the reference: it is
 * tosp_kelem_prod restricted to device pointers of the handle's GPU, with its
 * scratch (two full-length vectors) taken from a fixed 16 MiB array built
 * into the library instead of the handle.  The call runs at once on the
 * handle's stream and returns after y is written, so x must be complete
 * before the call.  Problems above 1,048,576 dofs (3*nnodes) are rejected
 * with TOSP_ERR_BAD_ARG; device ordinals from 64 up with
 * TOSP_ERR_UNSUPPORTED.  The first call on a device resolves the array's
 * address and should come before any stream capture.  All calls share the
 * array: calls whose GPU work overlaps race. */
int tosp_kelem_prod_noalloc(tosp_handle *h, const double *x, double *y, int64_t nfree);

/* ---- serving loop ------------------------------------------------------
 * A server runs many independent SetupGMG + SolveMG (zero start) + Grad
 * requests on the current device.  No counterpart in the reference (which
 * solves one problem per MATLAB process).  Requests are admitted in arrival
 * order while fewer than `max_slots` are in flight and the request's device
 * memory (the measured footprint of its shape once one handle of that shape
 * exists, an estimate before) fits `hbm_budget_bytes`; handles are cached per
 * problem shape and reused.  A worker sets an admitted request up (hierarchy,
 * initial residual, first CG iteration); then the request joins the batch of
 * in-flight requests of its shape (mesh, MR factor, grids, cycle, precision;
 * supports and loads may differ), and a runner advances every batch one CG
 * iteration per tick (each member's iteration is its handle's captured graph
 * on its own stream, one host synchronisation per tick for the batch).  For
 * requests with mg.small_cycle_max > 0 each visit to the levels with at most
 * that many nodes is one persistent launch for all members of the batch (the
 * member's graph is captured in segments around the visits).  A finished
 * request leaves its batch at once and a worker computes its Grad. */
typedef struct tosp_server tosp_server;

#define TOSP_REQ_QUEUED     0
#define TOSP_REQ_RUNNING    1
#define TOSP_REQ_DONE       2
#define TOSP_REQ_FAILED     3
#define TOSP_REQ_CANCELLED  4

typedef struct tosp_request_stats {
    int32_t it;            /* the reference's `it` of the solve                    */
    double  relres;        /* final relative residual                              */
    double  ms_latency;    /* submit -> results ready (host clock)                 */
    double  ms_queue;      /* time spent waiting for a slot / memory                */
    double  ms_run;        /* setup + solve + Grad                                 */
    int32_t precision;     /* precision that produced the result: a mixed-precision
                              request whose solve stalls or breaks down is re-run once
                              in FP64, warm-started from the mixed iterate            */
} tosp_request_stats;

int tosp_server_create(int32_t max_slots, int64_t hbm_budget_bytes, tosp_server **out);
/* Create `count` idle handles for the problem's shape ahead of its requests
 * (within the budget; TOSP_ERR_OOM otherwise), so that the first requests of
 * a shape do not wait for a handle's creation. */
int tosp_server_prepare(tosp_server *s, const tosp_problem *prob, const tosp_mg_params *mg, int32_t precision,
                        int32_t count);
/* Copies the problem arrays, densities `xfil` (density mesh) and load `f`
 * (free dofs); TOSP_ERR_OOM if the request can never fit the budget. */
int tosp_server_submit(tosp_server *s, const tosp_problem *prob, const tosp_mg_params *mg, int32_t precision,
                       const double *xfil, int64_t ndens, const double *f, int64_t nfree, int64_t *request_id);
int tosp_server_poll(tosp_server *s, int64_t request_id, int32_t *state);
/* Block until the request is done/failed/cancelled (TOSP_ERR_TIMEOUT otherwise). */
int tosp_server_wait(tosp_server *s, int64_t request_id, double timeout_s);
/* Copy results: u on the free dofs, the filtered sensitivities; returns the
 * solve status (TOSP_OK / TOSP_NOT_CONVERGED / an error). */
int tosp_server_result(tosp_server *s, int64_t request_id, double *u, int64_t nfree, double *fgrad, int64_t ndens,
                       tosp_request_stats *st);
/* Cancel a queued request (running requests complete). */
int tosp_server_cancel(tosp_server *s, int64_t request_id);
/* Forget a finished request and its results. */
int tosp_server_release(tosp_server *s, int64_t request_id);
int tosp_server_info(tosp_server *s, int32_t *active, int32_t *queued, int64_t *used_bytes, int64_t *cached_handles);
/* Runner counters: ticks, member iterations run inside batch graphs, and the
 * largest batch seen (instrumentation for tests and benchmarks). */
int tosp_server_counters(tosp_server *s, int64_t *ticks, int64_t *batched_iterations, int64_t *max_batch);
/* Cancels queued requests, waits for running ones, frees every handle. */
int tosp_server_destroy(tosp_server *s);

/* Host-only: the n^3 sub-element stiffness blocks kv (576 x n^3, column s is
 * k{s}(:), column-major) of I/ElemStiffMatrixGQMR.m:1 for hex8 elements. */
int tosp_elem_stiff_mr(double el, double eh, double ew, double nu, int32_t n, double *kv);

#ifdef __cplusplus
}
#endif

#endif /* TOSP_H */
