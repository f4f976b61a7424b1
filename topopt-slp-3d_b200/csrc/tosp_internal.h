// Internal declarations shared by the tosp CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "tosp.h"

namespace tosp {

// Count of kernel launches issued by this library (all handles, all threads).
void count_launch();
long long launch_count();

// ---------------------------------------------------------------------------
// Geometry of one structured hex8 grid (reference numbering: y fastest, then
// x, then z; dof = 3*node + component).
// ---------------------------------------------------------------------------
struct Grid {
    int nelx, nely, nelz;
    int nx, ny, nz;
    int64_t nnodes, ndof, nelem;
};

inline Grid make_grid(int nelx, int nely, int nelz) {
    Grid g;
    g.nelx = nelx; g.nely = nely; g.nelz = nelz;
    g.nx = nelx + 1; g.ny = nely + 1; g.nz = nelz + 1;
    g.nnodes = (int64_t)g.nx * g.ny * g.nz;
    g.ndof = 3 * g.nnodes;
    g.nelem = (int64_t)nelx * nely * nelz;
    return g;
}

// Element-brick tiling of the fine-level operator: a CTA owns BX x BY x BZ
// elements (y fastest) and the (BX+1)(BY+1)(BZ+1) nodes around them.
constexpr int BX = 4, BY = 8, BZ = 4;
constexpr int BRICK_ELEMS = BX * BY * BZ;            // 128 threads, one element each
constexpr int NBX = BX + 1, NBY = BY + 1, NBZ = BZ + 1;
constexpr int BRICK_NODES = NBX * NBY * NBZ;         // 225
constexpr int KE_PACK = 300;                          // upper triangle of a 24x24 block

// Order of the 300 upper-triangle entries (i <= j) in the fine operator's
// block layout: diagonal by diagonal (d = j - i = 0..23), and within a
// diagonal even i first, then odd i, so that consecutive entries never update
// the same output (the updates y_i += k u_j, y_j += k u_i are dependent
// through y otherwise).
__host__ __device__ constexpr int pair_d(int t) {
    int d = 0;
    while (t >= 24 - d) {
        t -= 24 - d;
        ++d;
    }
    return d;
}
__host__ __device__ constexpr int pair_i(int t) {
    const int d = pair_d(t);
    int r = t;
    for (int e = 0; e < d; ++e) r -= 24 - e;
    const int neven = (24 - d + 1) / 2;
    return r < neven ? 2 * r : 2 * (r - neven) + 1;
}
__host__ __device__ constexpr int pair_j(int t) { return pair_i(t) + pair_d(t); }
__host__ __device__ constexpr int pair_index_diag(int i) { return (i % 2 == 0) ? i / 2 : 12 + i / 2; }
// Row-major packed index of (i, j), i <= j (Galerkin build, Grad).
__host__ __device__ constexpr int pair_rowmajor(int i, int j) { return i * 24 - i * (i - 1) / 2 + (j - i); }

struct FineGeom {
    Grid g;
    int nelx_d, nely_d;        // density mesh (n x finer)
    int nbx, nby, nbz;         // bricks per direction
    int64_t nbricks;
    // per brick: 1 when one of its nodes has a fixed dof (the write-out then
    // reads the free-dof mask); null: every brick reads it
    const uint8_t *bfix;
};

// Coarse-level stencil: 27 neighbour blocks of 3x3 per node, stored
// offset-major / node-minor: st[(o*9 + ci*3 + cj) * nnodes + node].
constexpr int STENCIL_VALS = 27 * 9;

// ---------------------------------------------------------------------------
// Host helpers (ke.cpp)
// ---------------------------------------------------------------------------
// Sub-element stiffness blocks of I/ElemStiffMatrixGQMR.m (hex8): ks[s][i][j].
void elem_stiff_mr(double el, double eh, double ew, double nu, int n, std::vector<double> &ks);
// Pack the upper triangles (row-major i <= j) of ns 24x24 blocks.
void pack_upper(const std::vector<double> &ks, int ns, std::vector<double> &packed);
void coarse_fine_table(const std::vector<double> &ks, int n, std::vector<double> &S);

struct FilterTap { int dx, dy, dz; double w; };
// Neighbour offsets/weights of I/ElemNeighborhood.m:93-122 (all signs).
void filter_taps(double rmin, double el, double eh, double ew, int opfilter, std::vector<FilterTap> &taps);

// ---------------------------------------------------------------------------
// Kernel launchers.  All take the stream of the handle.
// ---------------------------------------------------------------------------
// SIMP factors w = emin + (E-emin) rho^p, in FP64 and (each optional) BF16,
// the BF16 values widened to FP64, and FP32.
void launch_simp(const double *rho, double *w64, __nv_bfloat16 *wbf, double *wq, float *w32, int64_t n, double p,
                 double emin, double E, cudaStream_t st);

// Fine MR operator y = K(w) x (y must be zeroed by the caller; fixed dofs of
// y stay zero).  kt: the n^3 blocks pair-major, see fine_nsp.
template <typename T, typename TW>
void launch_fine_apply(const T *x, T *y, const TW *w, const uint8_t *freemask, const T *kt, const FineGeom &fg,
                       int n, cudaStream_t st);
// y += diag(K(w)) (y zeroed by the caller); ke64: row-major packed blocks.
void launch_fine_diag(double *y, const double *w, const uint8_t *freemask, const double *ke64, const FineGeom &fg,
                      int n, cudaStream_t st);
// Stride of the pair-major block layout: entry t of block s at kt[t*nsp + s].
int fine_nsp(int n, int elem_bytes);
// The operator's block table from the row-major packed blocks (n = 2: the
// Walsh-Hadamard modes; otherwise pair-major with stride fine_nsp).
void fine_block_table(const std::vector<double> &packed_rowmajor, int n, int elem_bytes, std::vector<double> &kt);
void fine_mr2_const_table(const std::vector<double> &kt_padded, int elem_bytes, std::vector<double> &out);
void launch_fine_apply64_const(const double *x, double *y, const double *w, const uint8_t *freemask,
                               const double *ktab, const FineGeom &fg, cudaStream_t st);
// Tensor-core finest operator of the mixed V-cycle (MR factor n = 1, 2, 3):
// whether the kernel serves the mesh (its factor staging needs n * nely even),
// the B operand image (FP16 pieces of the scaled blocks, canonical
// shared-memory layout, then the block scale) and the launch.
bool fine_tc_supported(int n, int nely);
void fine_tc_image(const std::vector<double> &packed_rowmajor, int n, std::vector<uint16_t> &img);
void launch_fine_apply_tc(const float *x, float *y, const __nv_bfloat16 *w, const uint8_t *fm, const void *bimg,
                          const FineGeom &fg, int n, int *err, cudaStream_t st);
// The same product with FP32 SIMP factors and the blocks in three FP16 pieces
// (the CG's product of cg_product 1), with its own B image.
bool fine_tc_w32_supported(int n);
void fine_tc_image_w32(const std::vector<double> &packed_rowmajor, int n, std::vector<uint16_t> &img);
void launch_fine_apply_tc_w32(const float *x, float *y, const float *w, const uint8_t *fm, const void *bimg,
                              const FineGeom &fg, int n, int *err, cudaStream_t st);

// Sensitivities g0 (I/Grad.m:24-49), zero for elements not in freeDensG.
void launch_grad(const double *u, const double *rho, const uint8_t *free_elem, const double *kepack,
                 double *g0, const FineGeom &fg, int n, double p, double emin, double E, cudaStream_t st);

// Galerkin coarse element matrices (FP64, 576 per coarse element).
// Finest coarsening by the sub-cell table (coarse elements whose fine nodes
// are all free), then the masked triple products for the others.
void launch_coarse_from_fine_table(const double *w, const uint8_t *freemask_f, const double *kepack,
                                   const double *S, double *Ac, const FineGeom &fg, const Grid &gc, int n,
                                   cudaStream_t st);
void launch_coarse_from_coarse(const double *Af, const uint8_t *freemask_f, const Grid &gf,
                               double *Ac, const Grid &gc, cudaStream_t st);
// Node stencil from element matrices (masked), plus omega/diag.
template <typename T>
void launch_assemble_stencil(const double *Ae, const uint8_t *freemask, const Grid &g, T *stencil,
                             T *invdiag, double omega, bool node_major, cudaStream_t st);
// Stencil products: mode 0: y = A x; 1: y = b - A x; 2: y = x + invD (b - A x).
// node_major: layout [node][27 offsets][3x3], one warp per node; otherwise
// [27 offsets][3x3][node], one thread per node.
template <typename T>
void launch_stencil(const T *st_vals, const T *x, const T *b, const T *invdiag, T *y, const Grid &g,
                    int mode, bool node_major, cudaStream_t st);
// Fine-level helpers: y = b - t ; x = x + invD (b - t) ; x = invD b
template <typename T>
void launch_residual(const T *b, const T *t, T *r, int64_t n, cudaStream_t st);
template <typename T>
void launch_jacobi_update(T *x, const T *b, const T *t, const T *invdiag, int64_t n, int first,
                          cudaStream_t st);
// Last sweep of a cycle written in FP64: out = x + invD (b - t) (computed in T).
template <typename T>
void launch_jacobi_out(double *out, const T *x, const T *b, const T *t, const T *invdiag, int64_t n,
                       cudaStream_t st);
template <typename T>
void launch_invert_diag(const T *diag, const uint8_t *freemask, T *invdiag, double omega, int64_t n,
                        cudaStream_t st);
// Transfers (masked).  prolong: xf (+)= P xc ; restrict: bc = P^T rf.
// invd_c / xc (optional): also write the coarse level's first Jacobi sweep
// from zero, xc = invd_c bc.
template <typename T>
void launch_prolong(const T *xc, T *xf, const uint8_t *freemask_f, const Grid &gf, const Grid &gc,
                    bool accumulate, cudaStream_t st);
template <typename T>
void launch_restrict(const T *rf, T *bc, const uint8_t *freemask_c, const Grid &gf, const Grid &gc,
                     cudaStream_t st, const T *invd_c = nullptr, T *xc = nullptr);
// Restriction of the residual bf - tf (the level-0 residual fused in).
template <typename T>
void launch_restrict_res(const T *bf, const T *tf, T *bc, const uint8_t *freemask_c, const Grid &gf,
                         const Grid &gc, cudaStream_t st, const T *invd_c = nullptr, T *xc = nullptr);
void launch_coarse_freemask(const uint8_t *freemask_f, uint8_t *freemask_c, const Grid &gf,
                            const Grid &gc, cudaStream_t st);

// Coarsest direct solve: dense SPD matrix (padded to a multiple of 32, fixed
// dofs decoupled with a unit diagonal), explicit inverse in place by a blocked
// symmetric sweep (C: npad x 32 workspace, Pinv: 32 x 32), GEMV.
void launch_dense_assemble(const double *Ae, const uint8_t *freemask, const Grid &g, double *A,
                           int64_t npad, cudaStream_t st);
int dense_sweep_inverse(double *A, double *C, double *Pinv, int64_t npad, int *d_info, cudaStream_t st);
template <typename T>
void launch_dense_solve(const double *X, const T *b, T *x, int64_t n, int64_t npad, cudaStream_t st);

// Persistent small-level cycle (k_small.cu): the steps of a V/W cycle below a
// level, resolved to buffers on the host, run by one cooperative kernel with a
// grid barrier between steps.
enum SmallStepKind : int32_t {
    SS_STENCIL = 0,    // y = b - A x (mode 1) or x + invd (b - A x) (mode 2), warp per node
    SS_RESTRICT = 1,   // y = P^T x on the coarse grid gc (masked), optional xc = invdc y
    SS_PROLONG = 2,    // y += P x from the coarse grid gc (masked)
    SS_JACOBI0 = 3,    // y = invd b (first sweep from zero)
    SS_DENSE = 4,      // y = X b (coarsest direct solve)
    SS_COPY = 5,       // y = x (x null: y = 0)
};
template <typename T>
struct SmallStep {
    int32_t kind, mode;
    Grid g, gc;                  // the level's grid; a transfer's coarse grid
    const T *st, *x, *b, *invd;
    T *y;
    const uint8_t *fm;           // mask of the written level
    const T *invdc;              // restriction: the coarse level's first sweep
    T *xc;
    const double *X;             // dense solve: inverse, n x n used of npad x npad
    int64_t n, npad;
};
struct GridBarrier {
    unsigned count, gen;
    int err;
    unsigned limit;   // polls before a wait gives up (0: SMALL_WAIT_LIMIT)
    int skip;         // k > 0: block k - 1 skips its first arrival (fault injection for tests)
    int pad;
};
// Work buffers of the coarsest-grid PCG (mg.opchol = 1, k_coarse_pcg.cu):
// FP64 vectors of the coarsest level, 3 * max_blocks partial sums, the grid
// barrier and the iteration count of the last solve.
struct CoarsePcgWork {
    double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *part = nullptr;
    GridBarrier *bar = nullptr;
    int *iters = nullptr;
    int max_blocks = 0;
};
// y = pcg(A_c, b) on the coarsest grid: A_c as the FP64 node-major stencil,
// invd = 1 / diag(A_c) (0 on fixed dofs), stop at ||r|| <= tol ||b|| or maxit.
template <typename T>
void launch_coarse_pcg(const double *st, const double *invd, const T *b, T *x, const Grid &g, CoarsePcgWork &w,
                       double tol, int maxit, cudaStream_t stream);
int coarse_pcg_max_blocks();
// One member of a batched small-level cycle: its step list (SmallStep of the
// cycle precision), and the blocks of the launch that run it.
struct SmallBatchEntry {
    const void *steps;
    int32_t nsteps, block0, nblocks, pad;
};
template <typename T>
void launch_small_cycle_batch(const SmallBatchEntry *ent_dev, int nmem, int maxsteps, GridBarrier *bar, int blocks,
                              cudaStream_t st);
// Largest grid of 256-thread blocks that can be co-resident (cooperative launch).
int small_cycle_max_blocks(bool fp64);
int small_cycle_batch_max_blocks(bool fp64);
template <typename T>
void launch_small_cycle(const SmallStep<T> *steps_dev, int nsteps, GridBarrier *bar, int blocks, cudaStream_t st);

// Filter (I/ApplyFilter.m): trans 0: (W x)./w, 1: W (x./w); weights: w = W 1.
// radius: largest |offset| of the taps (the shared-memory tile's halo); -1
// selects the per-element kernel.
void launch_filter(const double *x, double *y, const double *wsum, const uint8_t *fixed,
                   const FilterTap *taps_dev, int ntaps, int nelx, int nely, int nelz, int trans,
                   int weights_only, int radius, cudaStream_t st);

// Vector kernels.
void launch_scatter_free(const double *v, const int64_t *idx, int64_t nfree, double *full, cudaStream_t st);
void launch_gather_free(const double *full, const int64_t *idx, int64_t nfree, double *v, cudaStream_t st);
template <typename TI, typename TO>
void launch_convert(const TI *a, TO *b, int64_t n, cudaStream_t st);
// Deterministic dot products: out[0] = sum a*b (fixed reduction tree).
constexpr int RED_BLOCKS = 592;
void launch_dot(const double *a, const double *b, int64_t n, double *partials, double *out, cudaStream_t st);
void launch_dot(const double *a, const float *b, int64_t n, double *partials, double *out, cudaStream_t st);
// a'b -> out0 and a'c -> out1 in one pass (partials: 2 * RED_BLOCKS).
void launch_dot2(const double *a, const double *b, const double *c, int64_t n, double *partials, double *out0,
                 double *out1, cudaStream_t st);
// PCG pieces (scalars in device memory, see solver.cpp for the slots).
void launch_pcg_direction(double *d, const double *s, double *sold, const double *scal, int64_t n, int mode,
                          double *x, cudaStream_t st, float *d32 = nullptr);
void launch_pcg_finish(double *x, const double *d, const double *scal, int64_t n, cudaStream_t st);
// launch_jacobi_out with the CG's dots r's (-> out0) and r's_old (-> out1,
// when so is given) of the new s in the same pass.
template <typename T>
void launch_jacobi_out_dot(double *out, const T *x, const T *b, const T *t, const T *invd, int64_t n, const double *r,
                           const double *so, double *partials, double *out0, double *out1, cudaStream_t st);
void launch_pcg_update(double *r, const double *q, double *scal, double *partials, int64_t n, cudaStream_t st,
                       float *b0 = nullptr, const float *invd0 = nullptr, float *x0 = nullptr);
void launch_pcg_update(double *r, const float *q, double *scal, double *partials, int64_t n, cudaStream_t st,
                       float *b0 = nullptr, const float *invd0 = nullptr, float *x0 = nullptr);
// r = f - t with r'r into scal[3] (residual replacement of cg_product 1), and
// the next mixed cycle's input as in launch_pcg_update.
void launch_replace_residual(const double *f, const double *t, double *r, double *scal, double *partials, int64_t n,
                             cudaStream_t st, float *b0 = nullptr, const float *invd0 = nullptr, float *x0 = nullptr);
void launch_set_scalar(double *dst, const double *src, cudaStream_t st);

// Loop state of an MG-preconditioned CG solve (I/SolveMG.m:26-53).
struct SolveState {
    int it = 0;             // the reference's `it` (iterations + 1)
    double nr = 0, nf = 0;  // relative residual, ||f||
    double best = 0;        // the stall test's best residual and its iteration
    int best_it = 0;
    int rc = 0;             // TOSP_OK, TOSP_NOT_CONVERGED or TOSP_ERR_BREAKDOWN
    bool done = false;      // the loop condition no longer holds
    double rmax = 0;        // cg_product 1: largest residual since the last replacement
    int replaced = 0;       // cg_product 1: residual replacements so far
};

// Serving-loop batches (solver.cpp): a solve's steps, and one CG iteration of
// several handles of one shape captured as a single graph.
int solve_start(tosp_handle *h, const double *x, const double *f);   // loads, r, norms, first iteration
int solve_step_account(tosp_handle *h);                               // after a batch iteration's sync
                                                                      // (and the residual replacement)
int solve_step(tosp_handle *h);                                       // one iteration on the handle's stream
const SolveState &solve_state(const tosp_handle *h);
int solve_stop(tosp_handle *h, double *x, int32_t *it, double *relres);  // final update, x to the host
// Batch key: handles with equal keys can share a batch graph (same grids,
// cycle and precision; supports and loads may differ).
std::string batch_key(const tosp_handle *h);
// A batch of handles of one shape (batch_key) stepping together: each
// member's iteration runs as its captured segments on its own stream, and
// every visit to the small levels between two segments is one persistent
// launch over all members (tables and barrier from batch_prepare).
struct BatchPlan {
    std::vector<tosp_handle *> mem;
    SmallBatchEntry *d_ent = nullptr;   // 3 variants x nmem entries (device)
    GridBarrier *d_bar = nullptr;
    int blocks = 0, maxsteps[3] = {0, 0, 0};
    bool fp64 = false;
};
int batch_prepare(BatchPlan &plan, cudaStream_t st, std::string &err);   // fills d_ent (allocated by the caller)
// Queue one CG iteration of every member (each at its own iteration number);
// ev_mem: one event per member; the caller synchronises the members' streams.
int batch_tick(const BatchPlan &plan, cudaStream_t main, cudaEvent_t *ev_mem, cudaEvent_t ev_small, std::string &err);

// Handle internals used by entry points that live outside solver.cpp.
int kelem_prod_with_scratch(tosp_handle *h, const double *x, double *y, int64_t nfree, double *xfull,
                            double *yfull);
int64_t handle_ndof(const tosp_handle *h);
int handle_device(const tosp_handle *h);
cudaStream_t handle_stream(const tosp_handle *h);
void set_handle_error(tosp_handle *h, const std::string &msg);

}  // namespace tosp
