// Handle, multigrid hierarchy, cycles and the MG-preconditioned CG, plus the
// extern "C" entry points of tosp.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <utility>
#include <string>
#include <vector>

#include "ptr_kind.h"
#include "tosp_internal.h"
#include "trace.h"

using namespace tosp;

#include <atomic>
static std::atomic<long long> g_launches{0};
void tosp::count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long tosp::launch_count() { return g_launches.load(std::memory_order_relaxed); }

namespace {

thread_local std::string g_create_error;

struct Level {
    Grid g;
    uint8_t *fm = nullptr;     // free flag per dof
    bool nm = false;           // stencil stored node-major, applied warp per node
    double *Ae = nullptr;      // Galerkin element matrices (levels >= 1), FP64
    void *st = nullptr;        // 27-point stencil (levels 1..L-2), cycle precision
    void *invd = nullptr;      // omega / diag(A), 0 on fixed dofs, cycle precision
    void *b = nullptr, *x = nullptr, *r = nullptr, *t = nullptr;   // cycle vectors
};

}  // namespace

struct tosp_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // problem
    int n = 1, ns = 1, precision = TOSP_PREC_FP64;
    double E = 1, nu = 0.3, p = 3, emin = 1e-9, el = 1, eh = 1, ew = 1, rmin = 1.5;
    int opfilter = 1;
    tosp_mg_params mg{};
    int ngrids = 2;
    bool mg_ok = true;         // false: no geometric hierarchy possible (operator/Grad/filter only)
    std::string mg_msg;
    FineGeom fg{};
    Grid dens{};               // density (= design) mesh as a grid of elements
    int64_t nfree = 0;
    int64_t *d_freeidx = nullptr;
    uint8_t *d_bfix = nullptr;      // per finest brick: touches a fixed dof
    // constants
    double *d_ke64 = nullptr;       // blocks packed per s (coarse build, Grad)
    double *d_cbS = nullptr;        // sub-cell Galerkin table of the finest coarsening
    double *d_kt64 = nullptr;       // pair-major layout of the fine operator
    float *d_kt32 = nullptr;
    std::vector<double> ktab_c;     // MR 2: FP64 Walsh-Hadamard coefficients passed with each launch
    uint16_t *d_tcimg = nullptr;    // mixed: tensor-core B operand image of the blocks (null: CUDA-core kernel)
    int *d_tcerr = nullptr;         // set by the tensor-core operator when an MMA wait times out
    uint16_t *d_tcimg32 = nullptr;  // cg_product 1: B image of the CG's product (three-piece blocks)
    // densities
    double *d_rho = nullptr, *d_w64 = nullptr;
    double *d_wq = nullptr;         // mixed: BF16-rounded factors in FP64 (V-cycle hierarchy)
    __nv_bfloat16 *d_wbf = nullptr;
    float *d_w32 = nullptr;         // cg_product 1: FP32 factors of the CG's tensor-core product
    uint8_t *d_free_elem = nullptr;
    // filter
    FilterTap *d_taps = nullptr;
    int filt_r = 0;                 // largest |offset| of the taps
    int ntaps = 0;
    uint8_t *d_fixed = nullptr;
    double *d_fw = nullptr;
    // hierarchy
    std::vector<Level> lev;
    double *d_diag64 = nullptr;     // diag of the finest operator
    double *d_Adense = nullptr, *d_sweepC = nullptr, *d_pinv = nullptr;   // coarsest: A, then A^{-1}
    int64_t ncoarse = 0, npad = 0;
    // coarsest grid by PCG (mg.opchol = 1 or the level rule's switch): FP64
    // node-major stencil, 1 / diag and the kernel's work buffers
    bool coarse_pcg = false;
    double *d_cst = nullptr, *d_cinvd = nullptr;
    CoarsePcgWork cpw;
    int *d_info = nullptr;
    bool setup_done = false;
    // persistent small-level cycle: first level it covers (-1: off), its grid
    // and three step lists (entered with the first sweep done, from zero, warm)
    // dots the CG wants from the preconditioner's last sweep (cg_iteration)
    struct {
        const double *r = nullptr, *so = nullptr;
        double *o0 = nullptr, *o1 = nullptr;
        bool want = false, done = false;
    } fdot;
    int small_l = -1;
    bool small_built = false;
    int small_blocks = 0;
    GridBarrier *d_bar = nullptr;
    unsigned char *d_steps = nullptr;
    int small_n[3] = {0, 0, 0};
    // one CG iteration (it >= 2) per parity of the iteration number (the
    // preconditioned residual alternates between cs and cso), captured once
    cudaGraphExec_t iter_graph[2] = {nullptr, nullptr};
    bool graph_failed = false;
    // CG (FP64, full-length vectors with zeros on fixed dofs)
    double *cx = nullptr, *cr = nullptr, *cd = nullptr, *cq = nullptr, *cs = nullptr, *cf = nullptr, *cso = nullptr;
    // cg_product 1: the direction in FP32 and its tensor-core product
    bool cg32 = false;
    float *cd32 = nullptr, *cq32 = nullptr;
    double *d_partials = nullptr, *d_scal = nullptr, *h_scal = nullptr;
    // staging
    double *d_stage_a = nullptr, *d_stage_b = nullptr;
    int64_t stage_len = 0;
    double *d_ufull = nullptr, *d_g0 = nullptr, *d_gf = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    tosp_solve_stats stats{};
    SolveState st{};                // loop state of the current solve
    // one CG iteration (it >= 2) per parity as graph segments split at the
    // visits to the persistent small-level cycle (serving-loop batches run
    // those visits batched across requests); seg_capture is set while the
    // segments are captured
    static constexpr int MAXSEG = 64;
    cudaGraphExec_t seg_graph[2][MAXSEG] = {};
    int nseg[2] = {0, 0};
    int seg_variant[MAXSEG] = {};   // small-cycle variant of visit i (the same for both parities)
    bool seg_failed = false, seg_capture = false;
    int seg_count = 0;
    std::vector<cudaGraph_t> seg_pending;
    int64_t bytes = 0;
    std::vector<void *> allocs;
};

namespace {

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            h->err = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call; \
            return (e_ == cudaErrorMemoryAllocation) ? TOSP_ERR_OOM : TOSP_ERR_CUDA;     \
        }                                                                                \
    } while (0)

#define CKL()                                                                   \
    do {                                                                        \
        cudaError_t e_ = cudaGetLastError();                                    \
        if (e_ != cudaSuccess) {                                                \
            h->err = std::string("CUDA launch error: ") + cudaGetErrorString(e_); \
            return TOSP_ERR_CUDA;                                               \
        }                                                                       \
    } while (0)

#define TRY(x)                   \
    do {                         \
        int rc_ = (x);           \
        if (rc_ != TOSP_OK) return rc_; \
    } while (0)

template <typename T>
int dalloc(tosp_handle *h, T **p, int64_t count) {
    *p = nullptr;
    if (count <= 0) count = 1;
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * (size_t)count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->err = "device allocation of " + std::to_string(sizeof(T) * count) + " bytes failed: " +
                 cudaGetErrorString(e);
        return TOSP_ERR_OOM;
    }
    h->allocs.push_back(q);
    h->bytes += (int64_t)sizeof(T) * count;
    *p = static_cast<T *>(q);
    return TOSP_OK;
}

// *on_dev: whether argument `what` is memory the handle's kernels can use
// directly (else it is host memory and gets staged).  Device memory of
// another GPU is refused: the kernels would fault on it without peer access.
int arg_location(tosp_handle *h, const void *p, const char *what, bool *on_dev) {
    *on_dev = false;
    if (!p) return TOSP_OK;
    cudaPointerAttributes a;
    const bool ok = cudaPointerGetAttributes(&a, p) == cudaSuccess;
    if (!ok) cudaGetLastError();
    const int k = classify_ptr(ok, ok ? (int)a.type : 0, ok ? a.device : -1, h->device);
    if (k == PTR_OTHER_DEVICE) {
        h->err = std::string(what) + " is device memory of GPU " + std::to_string(a.device) +
                 ", but the handle lives on GPU " + std::to_string(h->device);
        return TOSP_ERR_BAD_ARG;
    }
    *on_dev = k == PTR_DEVICE;
    return TOSP_OK;
}

// Copy `count` doubles from a host or device pointer into device memory.
int load_vec(tosp_handle *h, double *dst, const double *src, int64_t count) {
    CK(cudaMemcpyAsync(dst, src, sizeof(double) * count, cudaMemcpyDefault, h->stream));
    return TOSP_OK;
}
int store_vec(tosp_handle *h, double *dst, const double *src, int64_t count) {
    CK(cudaMemcpyAsync(dst, src, sizeof(double) * count, cudaMemcpyDefault, h->stream));
    return TOSP_OK;
}

int sync(tosp_handle *h) {
    CK(cudaStreamSynchronize(h->stream));
    CKL();
    return TOSP_OK;
}

// ----- level rules (I/StartStrSLP.m:107-133) --------------------------------
// Largest coarsest system of the direct solve: its explicit FP64 inverse
// (npad^2 doubles, 4.8 GB here) is applied as one GEMV per cycle.
constexpr int DENSE_MAX = 24576;

// The reference's level rule (I/StartStrSLP.m:122-132): with opchol = 0,
// grids are added while the coarsest system exceeds nmaxchol, and a mesh that
// cannot take another grid switches to PCG on the coarsest grid (pcg = true).
// The direct solve here is an explicit dense inverse of at most DENSE_MAX
// dofs, so a coarsest system between DENSE_MAX and nmaxchol, which the
// reference would factor with sparse Cholesky, gets one more grid when the
// mesh allows it and PCG otherwise.  opchol = 1 keeps ngrids and uses PCG.
int choose_levels(int nelx, int nely, int nelz, int ngrids, int nmaxchol, int opchol, bool &pcg, std::string &msg) {
    const int cap = nmaxchol < DENSE_MAX ? nmaxchol : DENSE_MAX;
    auto divisible = [&](int k) {
        const int m = 1 << (k - 1);
        return nelx % m == 0 && nely % m == 0 && nelz % m == 0;
    };
    pcg = opchol == 1;
    int ng = ngrids < 2 ? 2 : ngrids;
    while (ng >= 2 && !divisible(ng)) --ng;
    if (ng < 2) {
        msg = "geometric multigrid needs even element counts (the reference falls back to AMG, not provided)";
        return -1;
    }
    while (!pcg) {
        const double m = (double)(1 << (ng - 1));
        const double nc = (nelx / m + 1) * (nely / m + 1) * (nelz / m + 1) * 3;
        if (nc <= cap) break;
        if (divisible(ng + 1)) ++ng;
        else pcg = true;
    }
    return ng;
}

// ----- operators -------------------------------------------------------------
// The FP64 finest-level kernel (coefficients as a launch parameter for MR 2).
void launch_fine64(tosp_handle *h, const double *x, double *y) {
    if (h->n == 2 && !h->ktab_c.empty())
        launch_fine_apply64_const(x, y, h->d_w64, h->lev[0].fm, h->ktab_c.data(), h->fg, h->stream);
    else
        launch_fine_apply<double, double>(x, y, h->d_w64, h->lev[0].fm, h->d_kt64, h->fg, h->n, h->stream);
}

// y = K x at the finest level in the cycle precision (zeroes y first).
template <typename T>
int fine_apply(tosp_handle *h, const T *x, T *y) {
    CK(cudaMemsetAsync(y, 0, sizeof(T) * h->fg.g.ndof, h->stream));
    if constexpr (sizeof(T) == 8) {
        launch_fine64(h, x, y);
    } else if (h->d_tcimg) {
        launch_fine_apply_tc(x, y, h->d_wbf, h->lev[0].fm, h->d_tcimg, h->fg, h->n, h->d_tcerr, h->stream);
    } else {
        launch_fine_apply<float, __nv_bfloat16>(x, y, h->d_wbf, h->lev[0].fm, h->d_kt32, h->fg, h->n, h->stream);
    }
    CKL();
    return TOSP_OK;
}

int fine_apply64(tosp_handle *h, const double *x, double *y) { return fine_apply<double>(h, x, y); }

// cg_product 1: the CG's product y = K x on the tensor cores with FP32 factors.
int fine_apply_cg32(tosp_handle *h, const float *x, float *y) {
    CK(cudaMemsetAsync(y, 0, sizeof(float) * h->fg.g.ndof, h->stream));
    launch_fine_apply_tc_w32(x, y, h->d_w32, h->lev[0].fm, h->d_tcimg32, h->fg, h->n, h->d_tcerr, h->stream);
    CKL();
    return TOSP_OK;
}

// Damped Jacobi sweeps (I/Smooth.m:14-23).  first_done: the first sweep from
// a zero guess was already written into lev[l].x (fused into the CG update);
// out (finest level only): the last sweep is written to out in FP64 instead of
// lev[l].x (the preconditioned vector of the outer CG).
template <typename T>
int smooth(tosp_handle *h, int l, int niter, bool x_zero, bool first_done = false, double *out = nullptr) {
    Level &L = h->lev[l];
    const int64_t nd = L.g.ndof;
    T *b = (T *)L.b;
    if (niter == 0 && x_zero) CK(cudaMemsetAsync(L.x, 0, sizeof(T) * nd, h->stream));
    for (int it = 0; it < niter; ++it) {
        const bool first = x_zero && it == 0;
        if (first) {
            if (!first_done) launch_jacobi_update<T>((T *)L.x, b, nullptr, (const T *)L.invd, nd, 1, h->stream);
        } else if (l == 0) {
            TRY(fine_apply<T>(h, (const T *)L.x, (T *)L.t));
            if (out && it == niter - 1 && h->fdot.want) {
                launch_jacobi_out_dot<T>(out, (const T *)L.x, b, (const T *)L.t, (const T *)L.invd, nd, h->fdot.r,
                                         h->fdot.so, h->d_partials, h->fdot.o0, h->fdot.o1, h->stream);
                h->fdot.done = true;
            } else if (out && it == niter - 1)
                launch_jacobi_out<T>(out, (const T *)L.x, b, (const T *)L.t, (const T *)L.invd, nd, h->stream);
            else
                launch_jacobi_update<T>((T *)L.x, b, (const T *)L.t, (const T *)L.invd, nd, 0, h->stream);
        } else {
            launch_stencil<T>((const T *)L.st, (const T *)L.x, b, (const T *)L.invd, (T *)L.t, L.g, 2, L.nm,
                              h->stream);
            std::swap(L.x, L.t);
        }
        CKL();
    }
    return TOSP_OK;
}

template <typename T>
int residual(tosp_handle *h, int l) {
    Level &L = h->lev[l];
    if (l == 0) {
        TRY(fine_apply<T>(h, (const T *)L.x, (T *)L.t));
        launch_residual<T>((const T *)L.b, (const T *)L.t, (T *)L.r, L.g.ndof, h->stream);
    } else {
        launch_stencil<T>((const T *)L.st, (const T *)L.x, (const T *)L.b, nullptr, (T *)L.r, L.g, 1, L.nm,
                          h->stream);
    }
    CKL();
    return TOSP_OK;
}

template <typename T>
int coarse_solve(tosp_handle *h) {
    Level &C = h->lev[h->ngrids - 1];
    if (h->coarse_pcg) {
        launch_coarse_pcg<T>(h->d_cst, h->d_cinvd, (const T *)C.b, (T *)C.x, C.g, h->cpw, h->mg.tolPCG,
                             h->mg.maxiterPCG, h->stream);
        CKL();
        return TOSP_OK;
    }
    launch_dense_solve<T>(h->d_Adense, (const T *)C.b, (T *)C.x, C.g.ndof, h->npad, h->stream);
    CKL();
    return TOSP_OK;
}

// Persistent small-level cycle: step lists that replay cycle_vw / smooth from
// level small_l down with every buffer resolved (the x / t ping-pong of the
// stencil sweeps is followed on copies of the level pointers; a final copy
// returns level small_l's iterate to lev[small_l].x).
constexpr int SMALL_MAX_STEPS = 2048;

template <typename T>
struct SmallBuilder {
    tosp_handle *h;
    std::vector<SmallStep<T>> out;
    std::vector<T *> X, Tt;

    SmallStep<T> blank(int kind, const Grid &g) {
        SmallStep<T> s;
        memset(&s, 0, sizeof s);
        s.kind = kind;
        s.g = g;
        return s;
    }
    void smooth(int l, int niter, bool x_zero, bool first_done) {
        Level &L = h->lev[l];
        if (niter == 0 && x_zero) {
            SmallStep<T> s = blank(SS_COPY, L.g);
            s.y = X[l];
            out.push_back(s);
        }
        for (int it = 0; it < niter; ++it) {
            if (x_zero && it == 0) {
                if (!first_done) {
                    SmallStep<T> s = blank(SS_JACOBI0, L.g);
                    s.b = (const T *)L.b;
                    s.invd = (const T *)L.invd;
                    s.y = X[l];
                    out.push_back(s);
                }
            } else {
                SmallStep<T> s = blank(SS_STENCIL, L.g);
                s.mode = 2;
                s.st = (const T *)L.st;
                s.x = X[l];
                s.b = (const T *)L.b;
                s.invd = (const T *)L.invd;
                s.y = Tt[l];
                out.push_back(s);
                std::swap(X[l], Tt[l]);
            }
        }
    }
    void cycle(int l, bool x_zero, bool wcycle, bool first_done) {
        const int Lc = h->ngrids - 1;
        Level &L = h->lev[l];
        Level &C = h->lev[l + 1];
        smooth(l, h->mg.smoothiter1, x_zero, first_done);
        const bool fuse = l + 1 < Lc && h->mg.smoothiter1 >= 1;
        SmallStep<T> r = blank(SS_STENCIL, L.g);
        r.mode = 1;
        r.st = (const T *)L.st;
        r.x = X[l];
        r.b = (const T *)L.b;
        r.y = (T *)L.r;
        out.push_back(r);
        SmallStep<T> rs = blank(SS_RESTRICT, L.g);
        rs.gc = C.g;
        rs.x = (const T *)L.r;
        rs.y = (T *)C.b;
        rs.fm = C.fm;
        if (fuse) {
            rs.invdc = (const T *)C.invd;
            rs.xc = X[l + 1];
        }
        out.push_back(rs);
        if (l + 1 == Lc) {
            SmallStep<T> d = blank(SS_DENSE, C.g);
            d.b = (const T *)C.b;
            d.y = X[l + 1];
            d.X = h->d_Adense;
            d.n = C.g.ndof;
            d.npad = h->npad;
            out.push_back(d);
        } else {
            cycle(l + 1, true, wcycle, fuse);
            if (wcycle) cycle(l + 1, false, wcycle, false);
        }
        SmallStep<T> p = blank(SS_PROLONG, L.g);
        p.gc = C.g;
        p.x = X[l + 1];
        p.y = X[l];
        p.fm = L.fm;
        out.push_back(p);
        smooth(l, h->mg.smoothiter2, false, false);
    }
    void build(int ls, bool x_zero, bool first_done) {
        out.clear();
        X.assign(h->ngrids, nullptr);
        Tt.assign(h->ngrids, nullptr);
        for (int l = 0; l < h->ngrids; ++l) {
            X[l] = (T *)h->lev[l].x;
            Tt[l] = (T *)h->lev[l].t;
        }
        cycle(ls, x_zero, h->mg.cycle == 1, first_done);
        if (X[ls] != (T *)h->lev[ls].x) {
            SmallStep<T> c = blank(SS_COPY, h->lev[ls].g);
            c.x = X[ls];
            c.y = (T *)h->lev[ls].x;
            out.push_back(c);
        }
    }
};

// Chooses the first level of the persistent cycle and uploads its step lists
// (once per handle: the buffers never move).  Off unless small_cycle_max > 0,
// for FMV cycles, for hierarchies with thread-per-node stencils and when no
// stencil level is small.
template <typename T>
int build_small(tosp_handle *h) {
    h->small_built = true;
    h->small_l = -1;
    const int Lc = h->ngrids - 1;
    if (!h->mg_ok || h->mg.cycle == 2 || h->mg.small_cycle_max <= 0 || Lc < 2 || h->coarse_pcg) return TOSP_OK;
    const int64_t smax = h->mg.small_cycle_max;
    int ls = -1;
    for (int l = 1; l < Lc; ++l)
        if (h->lev[l].g.nnodes <= smax) {
            ls = l;
            break;
        }
    if (ls < 0) return TOSP_OK;
    for (int l = ls; l < Lc; ++l)
        if (!h->lev[l].nm) return TOSP_OK;
    const int maxb = small_cycle_max_blocks(sizeof(T) == 8);
    if (maxb < 1) return TOSP_OK;
    SmallBuilder<T> b{h, {}, {}, {}};
    std::vector<SmallStep<T>> all;
    int n[3];
    const bool variant[3][2] = {{true, true}, {true, false}, {false, false}};
    for (int v = 0; v < 3; ++v) {
        b.build(ls, variant[v][0], variant[v][1]);
        if ((int)b.out.size() > SMALL_MAX_STEPS) return TOSP_OK;
        n[v] = (int)b.out.size();
        b.out.resize(SMALL_MAX_STEPS);
        all.insert(all.end(), b.out.begin(), b.out.end());
    }
    TRY(dalloc(h, &h->d_steps, (int64_t)(sizeof(SmallStep<T>) * all.size())));
    CK(cudaMemcpy(h->d_steps, all.data(), sizeof(SmallStep<T>) * all.size(), cudaMemcpyHostToDevice));
    TRY(dalloc(h, &h->d_bar, 1));
    CK(cudaMemset(h->d_bar, 0, sizeof(GridBarrier)));
    // about two nodes per warp on the largest level, at most what is co-resident
    const int64_t want = (h->lev[ls].g.nnodes + 15) / 16;
    h->small_blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, maxb));
    for (int v = 0; v < 3; ++v) h->small_n[v] = n[v];
    h->small_l = ls;
    return TOSP_OK;
}

// While an iteration is captured as segments, a visit to the small levels
// closes the current segment (its graph is kept) and opens the next; the
// visit itself is left to the caller of the segments.
int segment_break(tosp_handle *h, int variant) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamEndCapture(h->stream, &g));
    h->seg_pending.push_back(g);
    if (h->seg_count < tosp_handle::MAXSEG) h->seg_variant[h->seg_count] = variant;
    h->seg_count++;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    return TOSP_OK;
}

template <typename T>
int small_cycle(tosp_handle *h, int variant) {
    if (h->seg_capture) return segment_break(h, variant);
    const SmallStep<T> *steps = reinterpret_cast<const SmallStep<T> *>(h->d_steps) + (size_t)variant * SMALL_MAX_STEPS;
    launch_small_cycle<T>(steps, h->small_n[variant], h->d_bar, h->small_blocks, h->stream);
    CKL();
    return TOSP_OK;
}

// VCycle / WCycle (I/VCycle.m:23-43, I/WCycle.m:23-44) on level l, right-hand
// side lev[l].b, iterate lev[l].x (zero when x_zero).
// first_done / out: see smooth (finest level of the outermost cycle only).
template <typename T>
int cycle_vw(tosp_handle *h, int l, bool x_zero, bool wcycle, bool first_done = false, double *out = nullptr) {
    const int Lc = h->ngrids - 1;
    Level &L = h->lev[l];
    Level &C = h->lev[l + 1];
    TRY(smooth<T>(h, l, h->mg.smoothiter1, x_zero, first_done));
    // the restriction also writes the coarse level's first sweep from zero
    const bool fuse = l + 1 < Lc && h->mg.smoothiter1 >= 1;
    const T *cinvd = fuse ? (const T *)C.invd : nullptr;
    T *cx = fuse ? (T *)C.x : nullptr;
    if (l == 0) {
        // finest residual b - A x restricted directly (no residual vector)
        TRY(fine_apply<T>(h, (const T *)L.x, (T *)L.t));
        launch_restrict_res<T>((const T *)L.b, (const T *)L.t, (T *)C.b, C.fm, L.g, C.g, h->stream, cinvd, cx);
    } else {
        TRY(residual<T>(h, l));
        launch_restrict<T>((const T *)L.r, (T *)C.b, C.fm, L.g, C.g, h->stream, cinvd, cx);
    }
    CKL();
    if (l + 1 == Lc) {
        TRY(coarse_solve<T>(h));
    } else if (l + 1 == h->small_l) {
        TRY(small_cycle<T>(h, fuse ? 0 : 1));
        if (wcycle) TRY(small_cycle<T>(h, 2));
    } else {
        TRY(cycle_vw<T>(h, l + 1, true, wcycle, fuse));
        if (wcycle) TRY(cycle_vw<T>(h, l + 1, false, wcycle));
    }
    launch_prolong<T>((const T *)C.x, (T *)L.x, L.fm, L.g, C.g, true, h->stream);
    CKL();
    TRY(smooth<T>(h, l, h->mg.smoothiter2, false, false, out));
    return TOSP_OK;
}

// FMVCycle (I/FMVCycle.m:22-39).
template <typename T>
int cycle_fmv(tosp_handle *h, int l, double *out = nullptr) {
    const int Lc = h->ngrids - 1;
    Level &L = h->lev[l];
    Level &C = h->lev[l + 1];
    launch_restrict<T>((const T *)L.b, (T *)C.b, C.fm, L.g, C.g, h->stream);
    CKL();
    if (l + 1 == Lc) TRY(coarse_solve<T>(h));
    else TRY(cycle_fmv<T>(h, l + 1));
    launch_prolong<T>((const T *)C.x, (T *)L.x, L.fm, L.g, C.g, false, h->stream);
    CKL();
    return cycle_vw<T>(h, l, false, false, false, out);
}

// The mixed CG update can prepare the next cycle's FP32 right-hand side and
// first Jacobi iterate (V/W cycles with a pre-smoothing sweep).
bool fused_first_sweep(const tosp_handle *h) { return h->mg.cycle != 2 && h->mg.smoothiter1 >= 1; }

// s = M^{-1} r on full-length FP64 vectors (r, s distinct from the level buffers).
// prepared (mixed only): lev[0].b = float(r) and, when fused_first_sweep,
// lev[0].x = invD b were written by the CG update.
int precondition(tosp_handle *h, const double *r, double *s, bool prepared = false) {
    Level &F = h->lev[0];
    const int64_t nd = F.g.ndof;
    double *out = h->mg.smoothiter2 >= 1 ? s : nullptr;
    if (h->precision == TOSP_PREC_FP64) {
        // the finest level reads r in place
        void *own_b = F.b;
        F.b = const_cast<double *>(r);
        int rc = h->mg.cycle == 2 ? cycle_fmv<double>(h, 0, out) : cycle_vw<double>(h, 0, true, h->mg.cycle == 1,
                                                                                     false, out);
        F.b = own_b;
        TRY(rc);
        if (!out) CK(cudaMemcpyAsync(s, F.x, sizeof(double) * nd, cudaMemcpyDeviceToDevice, h->stream));
    } else {
        if (!prepared) {
            launch_convert<double, float>(r, (float *)F.b, nd, h->stream);
            CKL();
        }
        const bool first_done = prepared && fused_first_sweep(h);
        if (h->mg.cycle == 2) TRY(cycle_fmv<float>(h, 0, out));
        else TRY(cycle_vw<float>(h, 0, true, h->mg.cycle == 1, first_done, out));
        if (!out) {
            launch_convert<float, double>((const float *)F.x, s, nd, h->stream);
            CKL();
        }
    }
    return TOSP_OK;
}

int ensure_stage(tosp_handle *h, int64_t len) {
    if (h->stage_len >= len) return TOSP_OK;
    TRY(dalloc(h, &h->d_stage_a, len));
    TRY(dalloc(h, &h->d_stage_b, len));
    h->stage_len = len;
    return TOSP_OK;
}

// Free-dof vector (host or device) -> full-length device vector.
int free_to_full(tosp_handle *h, const double *v, double *full, const char *what) {
    const double *src = v;
    bool dev = false;
    TRY(arg_location(h, v, what, &dev));
    if (!dev) {
        TRY(ensure_stage(h, h->nfree));
        TRY(load_vec(h, h->d_stage_a, v, h->nfree));
        src = h->d_stage_a;
    }
    CK(cudaMemsetAsync(full, 0, sizeof(double) * h->fg.g.ndof, h->stream));
    launch_scatter_free(src, h->d_freeidx, h->nfree, full, h->stream);
    CKL();
    return TOSP_OK;
}

int full_to_free(tosp_handle *h, const double *full, double *v, const char *what) {
    bool dev = false;
    TRY(arg_location(h, v, what, &dev));
    if (dev) {
        launch_gather_free(full, h->d_freeidx, h->nfree, v, h->stream);
        CKL();
        return TOSP_OK;
    }
    TRY(ensure_stage(h, h->nfree));
    launch_gather_free(full, h->d_freeidx, h->nfree, h->d_stage_b, h->stream);
    CKL();
    TRY(store_vec(h, v, h->d_stage_b, h->nfree));
    return TOSP_OK;
}

int build_masks(tosp_handle *h, const int64_t *freedofs, int64_t nfree) {
    const Grid &g0 = h->lev[0].g;
    std::vector<int64_t> idx(nfree);
    std::vector<uint8_t> fm(g0.ndof, 0);
    int64_t prev = -1;
    for (int64_t i = 0; i < nfree; ++i) {
        const int64_t d = freedofs[i] - 1;
        if (d < 0 || d >= g0.ndof) {
            h->err = "freedofs entry out of range at position " + std::to_string(i);
            return TOSP_ERR_BAD_ARG;
        }
        if (d <= prev) {
            h->err = "freedofs must be strictly ascending";
            return TOSP_ERR_BAD_ARG;
        }
        prev = d;
        idx[i] = d;
        fm[d] = 1;
    }
    if (h->d_freeidx == nullptr || h->nfree < nfree) TRY(dalloc(h, &h->d_freeidx, nfree));
    h->nfree = nfree;
    CK(cudaMemcpy(h->d_freeidx, idx.data(), sizeof(int64_t) * nfree, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->lev[0].fm, fm.data(), g0.ndof, cudaMemcpyHostToDevice));
    // bricks whose nodes carry a fixed dof: a node at x lies in brick x / BX
    // and, on a brick boundary, in brick x / BX - 1 (same in y and z)
    {
        const FineGeom &fg = h->fg;
        std::vector<uint8_t> bf((size_t)fg.nbricks, 0);
        for (int64_t d = 0; d < g0.ndof; ++d) {
            if (fm[d]) continue;
            const int64_t node = d / 3;
            const int ny = (int)(node % g0.ny), nx = (int)((node / g0.ny) % g0.nx), nz = (int)(node / ((int64_t)g0.ny * g0.nx));
            for (int bz = (nz - 1) / BZ; bz <= nz / BZ; ++bz)
                for (int bx = (nx - 1) / BX; bx <= nx / BX; ++bx)
                    for (int by = (ny - 1) / BY; by <= ny / BY; ++by)
                        if (bx >= 0 && by >= 0 && bz >= 0 && bx < fg.nbx && by < fg.nby && bz < fg.nbz)
                            bf[((size_t)bz * fg.nbx + bx) * fg.nby + by] = 1;
        }
        if (h->d_bfix == nullptr) TRY(dalloc(h, &h->d_bfix, fg.nbricks));
        CK(cudaMemcpy(h->d_bfix, bf.data(), bf.size(), cudaMemcpyHostToDevice));
        h->fg.bfix = h->d_bfix;
    }
    for (int l = 0; l + 1 < h->ngrids; ++l)
        launch_coarse_freemask(h->lev[l].fm, h->lev[l + 1].fm, h->lev[l].g, h->lev[l + 1].g, h->stream);
    CKL();
    h->setup_done = false;
    return sync(h);
}

int create_impl(tosp_handle *h, const tosp_problem *pb, const tosp_mg_params *mg, int precision) {
    if (!pb || !mg) {
        h->err = "null problem or mg parameters";
        return TOSP_ERR_BAD_ARG;
    }
    if (pb->nelx < 1 || pb->nely < 1 || pb->nelz < 1 || !(pb->el > 0) || !(pb->eh > 0) || !(pb->ew > 0)) {
        h->err = "invalid mesh dimensions or element sizes";
        return TOSP_ERR_BAD_ARG;
    }
    if (pb->mr_n < 1 || pb->mr_n > 3) {
        h->err = "mr_n must be 1, 2 or 3";
        return TOSP_ERR_UNSUPPORTED;
    }
    if (pb->opfilter < 0 || pb->opfilter > 2 || (pb->opfilter != 0 && !(pb->rmin > 0))) {
        h->err = "opfilter must be 0, 1 or 2 with rmin > 0";
        return TOSP_ERR_BAD_ARG;
    }
    if (mg->cycle < 0 || mg->cycle > 2 || mg->smoother != 0 || mg->smoothiter1 < 0 || mg->smoothiter2 < 0 ||
        !(mg->omega > 0) || mg->maxiterMG < 0) {
        h->err = "unsupported mg parameters (cycle 0/1/2, Jacobi smoother, omega > 0)";
        return TOSP_ERR_UNSUPPORTED;
    }
    if (precision != TOSP_PREC_FP64 && precision != TOSP_PREC_MIXED) {
        h->err = "precision must be TOSP_PREC_FP64 or TOSP_PREC_MIXED";
        return TOSP_ERR_BAD_ARG;
    }
    if (mg->cg_product < 0 || mg->cg_product > 1 || mg->replace_drop < 0.0 || mg->replace_drop >= 1.0) {
        h->err = "cg_product must be 0 or 1 and replace_drop in [0, 1)";
        return TOSP_ERR_BAD_ARG;
    }
    if (mg->cg_product == 1 && (precision != TOSP_PREC_MIXED || !fine_tc_supported(pb->mr_n, pb->nely) ||
                                !fine_tc_w32_supported(pb->mr_n))) {
        h->err = "cg_product 1 needs TOSP_PREC_MIXED and the tensor-core operator (n * nely even)";
        return TOSP_ERR_UNSUPPORTED;
    }
    if (!pb->freedofs || pb->nfree <= 0) {
        h->err = "freedofs missing";
        return TOSP_ERR_BAD_ARG;
    }
    CK(cudaGetDevice(&h->device));
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    h->n = pb->mr_n;
    h->ns = h->n * h->n * h->n;
    h->precision = precision;
    h->E = pb->E; h->nu = pb->nu; h->p = pb->p; h->emin = pb->emin;
    h->el = pb->el; h->eh = pb->eh; h->ew = pb->ew;
    h->opfilter = pb->opfilter; h->rmin = pb->rmin;
    h->mg = *mg;
    if (h->mg.replace_drop == 0.0) h->mg.replace_drop = 0.1;
    h->cg32 = mg->cg_product == 1;
    if (mg->opchol < 0 || mg->opchol > 1 || !(mg->tolPCG > 0) || mg->maxiterPCG < 1) {
        h->err = "opchol must be 0 or 1, tolPCG > 0 and maxiterPCG >= 1";
        return TOSP_ERR_BAD_ARG;
    }
    std::string msg;
    bool cpcg = false;
    int ng = choose_levels(pb->nelx, pb->nely, pb->nelz, mg->ngrids, mg->nmaxchol, mg->opchol, cpcg, msg);
    if (ng < 0) {
        // the operator, Grad and the filter still work; SolveMG/cycles report why not
        h->mg_ok = false;
        h->mg_msg = msg;
        ng = 1;
    }
    h->ngrids = ng;
    h->lev.resize(ng);
    for (int l = 0; l < ng; ++l)
        h->lev[l].g = make_grid(pb->nelx >> l, pb->nely >> l, pb->nelz >> l);
    const Grid &g0 = h->lev[0].g;
    FineGeom &fg = h->fg;
    fg.g = g0;
    fg.nelx_d = pb->nelx * h->n;
    fg.nely_d = pb->nely * h->n;
    fg.nbx = (g0.nelx + BX - 1) / BX;
    fg.nby = (g0.nely + BY - 1) / BY;
    fg.nbz = (g0.nelz + BZ - 1) / BZ;
    fg.nbricks = (int64_t)fg.nbx * fg.nby * fg.nbz;
    h->dens = make_grid(pb->nelx * h->n, pb->nely * h->n, pb->nelz * h->n);
    h->ncoarse = h->mg_ok ? h->lev[ng - 1].g.ndof : 0;
    h->coarse_pcg = h->mg_ok && cpcg;
    h->npad = h->coarse_pcg ? 0 : (h->ncoarse + 31) / 32 * 32;
    if (h->npad > DENSE_MAX) {
        h->err = "coarsest system too large for the dense direct solve: " + std::to_string(h->ncoarse) +
                 " dofs; use more grids";
        return TOSP_ERR_UNSUPPORTED;
    }

    // constant blocks
    std::vector<double> ks, packed;
    elem_stiff_mr(pb->el, pb->eh, pb->ew, pb->nu, h->n, ks);
    pack_upper(ks, h->ns, packed);
    TRY(dalloc(h, &h->d_ke64, (int64_t)packed.size()));
    CK(cudaMemcpy(h->d_ke64, packed.data(), sizeof(double) * packed.size(), cudaMemcpyHostToDevice));
    if (h->mg_ok) {
        std::vector<double> S;
        coarse_fine_table(ks, h->n, S);
        TRY(dalloc(h, &h->d_cbS, (int64_t)S.size()));
        CK(cudaMemcpy(h->d_cbS, S.data(), sizeof(double) * S.size(), cudaMemcpyHostToDevice));
    }
    {
        std::vector<double> kt64, kt32d;
        fine_block_table(packed, h->n, 8, kt64);
        if (h->n == 2) fine_mr2_const_table(kt64, 8, h->ktab_c);
        fine_block_table(packed, h->n, 4, kt32d);
        std::vector<float> kt32(kt32d.begin(), kt32d.end());
        TRY(dalloc(h, &h->d_kt64, (int64_t)kt64.size()));
        TRY(dalloc(h, &h->d_kt32, (int64_t)kt32.size()));
        CK(cudaMemcpy(h->d_kt64, kt64.data(), sizeof(double) * kt64.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_kt32, kt32.data(), sizeof(float) * kt32.size(), cudaMemcpyHostToDevice));
    }
    if (precision == TOSP_PREC_MIXED && fine_tc_supported(h->n, pb->nely)) {
        std::vector<uint16_t> img;
        fine_tc_image(packed, h->n, img);
        TRY(dalloc(h, &h->d_tcimg, (int64_t)img.size()));
        CK(cudaMemcpy(h->d_tcimg, img.data(), sizeof(uint16_t) * img.size(), cudaMemcpyHostToDevice));
        TRY(dalloc(h, &h->d_tcerr, 1));
        CK(cudaMemset(h->d_tcerr, 0, sizeof(int)));
        if (mg->cg_product == 1) {
            fine_tc_image_w32(packed, h->n, img);
            TRY(dalloc(h, &h->d_tcimg32, (int64_t)img.size()));
            CK(cudaMemcpy(h->d_tcimg32, img.data(), sizeof(uint16_t) * img.size(), cudaMemcpyHostToDevice));
        }
    }

    // levels
    const size_t tsz = precision == TOSP_PREC_FP64 ? 8 : 4;
    for (int l = 0; l < ng; ++l) {
        Level &L = h->lev[l];
        TRY(dalloc(h, &L.fm, L.g.ndof));
        uint8_t *vb;
        TRY(dalloc(h, &vb, (int64_t)tsz * L.g.ndof * 4));
        L.b = vb;
        L.x = vb + tsz * L.g.ndof;
        L.r = vb + 2 * tsz * L.g.ndof;
        L.t = vb + 3 * tsz * L.g.ndof;
        if (l >= 1) TRY(dalloc(h, &L.Ae, L.g.nelem * 576));
        if (l >= 1 && l < ng - 1) {
            uint8_t *sp;
            TRY(dalloc(h, &sp, (int64_t)tsz * L.g.nnodes * STENCIL_VALS));
            L.st = sp;
        }
        if (l < ng - 1 || !h->mg_ok) {
            uint8_t *ip;
            TRY(dalloc(h, &ip, (int64_t)tsz * L.g.ndof));
            L.invd = ip;
        }
    }
    TRY(dalloc(h, &h->d_diag64, g0.ndof));
    if (h->mg_ok && h->coarse_pcg) {
        const Grid &gc = h->lev[ng - 1].g;
        CoarsePcgWork &w = h->cpw;
        TRY(dalloc(h, &h->d_cst, gc.nnodes * STENCIL_VALS));
        TRY(dalloc(h, &h->d_cinvd, gc.ndof));
        TRY(dalloc(h, &w.x, gc.ndof));
        TRY(dalloc(h, &w.r, gc.ndof));
        TRY(dalloc(h, &w.p, gc.ndof));
        TRY(dalloc(h, &w.q, gc.ndof));
        w.max_blocks = coarse_pcg_max_blocks();
        TRY(dalloc(h, &w.part, 3 * (int64_t)w.max_blocks));
        TRY(dalloc(h, &w.bar, 1));
        CK(cudaMemset(w.bar, 0, sizeof(GridBarrier)));
        TRY(dalloc(h, &w.iters, 1));
    } else if (h->mg_ok) {
        TRY(dalloc(h, &h->d_Adense, h->npad * h->npad));
        TRY(dalloc(h, &h->d_sweepC, h->npad * 32));
        TRY(dalloc(h, &h->d_pinv, 32 * 32));
    }
    TRY(dalloc(h, &h->d_info, 1));
    // densities
    const int64_t nd = h->dens.nelem;
    TRY(dalloc(h, &h->d_rho, nd));
    TRY(dalloc(h, &h->d_w64, nd));
    if (precision == TOSP_PREC_MIXED) {
        TRY(dalloc(h, &h->d_wbf, nd));
        TRY(dalloc(h, &h->d_wq, nd));
    }
    if (h->cg32) TRY(dalloc(h, &h->d_w32, nd));
    TRY(dalloc(h, &h->d_free_elem, g0.nelem));
    {
        std::vector<uint8_t> fe(g0.nelem, pb->free_dens_g ? 0 : 1);
        if (pb->free_dens_g) {
            for (int64_t i = 0; i < pb->nfree_dens_g; ++i) {
                const int64_t e = pb->free_dens_g[i] - 1;
                if (e < 0 || e >= g0.nelem) {
                    h->err = "free_dens_g entry out of range";
                    return TOSP_ERR_BAD_ARG;
                }
                fe[e] = 1;
            }
        }
        CK(cudaMemcpy(h->d_free_elem, fe.data(), g0.nelem, cudaMemcpyHostToDevice));
    }
    // CG vectors
    TRY(dalloc(h, &h->cx, g0.ndof));
    TRY(dalloc(h, &h->cr, g0.ndof));
    TRY(dalloc(h, &h->cd, g0.ndof));
    TRY(dalloc(h, &h->cq, g0.ndof));
    TRY(dalloc(h, &h->cs, g0.ndof));
    TRY(dalloc(h, &h->cf, g0.ndof));
    if (mg->flexible) TRY(dalloc(h, &h->cso, g0.ndof));
    if (h->cg32) {
        TRY(dalloc(h, &h->cd32, g0.ndof));
        TRY(dalloc(h, &h->cq32, g0.ndof));
    }
    TRY(dalloc(h, &h->d_partials, 2 * RED_BLOCKS + 1));   // + the reductions' arrival counter
    CK(cudaMemset(h->d_partials, 0, sizeof(double) * (2 * RED_BLOCKS + 1)));
    TRY(dalloc(h, &h->d_scal, 16));
    CK(cudaMallocHost(&h->h_scal, sizeof(double) * 16));
    TRY(dalloc(h, &h->d_ufull, g0.ndof));
    TRY(dalloc(h, &h->d_g0, nd));
    TRY(dalloc(h, &h->d_gf, nd));
    // filter
    {
        std::vector<FilterTap> taps;
        if (pb->opfilter != 0) {
            const double eld = pb->el / h->n, ehd = pb->eh / h->n, ewd = pb->ew / h->n;
            filter_taps(pb->rmin, eld, ehd, ewd, pb->opfilter, taps);
        }
        h->ntaps = (int)taps.size();
        h->filt_r = 0;
        for (const FilterTap &t : taps)
            h->filt_r = std::max(h->filt_r, std::max(std::abs(t.dx), std::max(std::abs(t.dy), std::abs(t.dz))));
        if (h->ntaps) {
            TRY(dalloc(h, &h->d_taps, h->ntaps));
            CK(cudaMemcpy(h->d_taps, taps.data(), sizeof(FilterTap) * taps.size(), cudaMemcpyHostToDevice));
        }
        if (pb->fixed_dens && pb->nfixed_dens > 0) {
            std::vector<uint8_t> fx(nd, 0);
            for (int64_t i = 0; i < pb->nfixed_dens; ++i) {
                const int64_t e = pb->fixed_dens[i] - 1;
                if (e < 0 || e >= nd) {
                    h->err = "fixed_dens entry out of range";
                    return TOSP_ERR_BAD_ARG;
                }
                fx[e] = 1;
            }
            TRY(dalloc(h, &h->d_fixed, nd));
            CK(cudaMemcpy(h->d_fixed, fx.data(), nd, cudaMemcpyHostToDevice));
        }
        TRY(dalloc(h, &h->d_fw, nd));
        if (h->ntaps) {
            launch_filter(nullptr, h->d_fw, nullptr, h->d_fixed, h->d_taps, h->ntaps, h->dens.nelx, h->dens.nely,
                          h->dens.nelz, 0, 1, h->filt_r, h->stream);
            CKL();
        }
    }
    return build_masks(h, pb->freedofs, pb->nfree);
}

template <typename T>
int setup_levels(tosp_handle *h) {
    const int ng = h->ngrids;
    const int64_t nd0 = h->lev[0].g.ndof;
    // finest diagonal (FP64) -> omega/diag in the cycle precision
    CK(cudaMemsetAsync(h->d_diag64, 0, sizeof(double) * nd0, h->stream));
    // the V-cycle hierarchy is Galerkin-consistent with the V-cycle's finest
    // operator: FP64 factors for the FP64 path, the BF16-rounded ones for mixed
    const double *wh = h->d_wq ? h->d_wq : h->d_w64;
    launch_fine_diag(h->d_diag64, wh, h->lev[0].fm, h->d_ke64, h->fg, h->n, h->stream);
    CKL();
    if constexpr (sizeof(T) == 8) {
        launch_invert_diag<double>(h->d_diag64, h->lev[0].fm, (double *)h->lev[0].invd, h->mg.omega, nd0, h->stream);
    } else {
        launch_invert_diag<double>(h->d_diag64, h->lev[0].fm, h->cs, h->mg.omega, nd0, h->stream);
        launch_convert<double, float>(h->cs, (float *)h->lev[0].invd, nd0, h->stream);
    }
    CKL();
    launch_coarse_from_fine_table(wh, h->lev[0].fm, h->d_ke64, h->d_cbS, h->lev[1].Ae, h->fg, h->lev[1].g, h->n,
                                  h->stream);
    CKL();
    for (int l = 1; l < ng - 1; ++l) {
        Level &L = h->lev[l];
        const int64_t wmax = h->mg.warp_stencil_max == 0 ? 65536 : h->mg.warp_stencil_max;
        L.nm = L.g.nnodes <= wmax;
        launch_assemble_stencil<T>(L.Ae, L.fm, L.g, (T *)L.st, (T *)L.invd, h->mg.omega, L.nm, h->stream);
        launch_coarse_from_coarse(L.Ae, L.fm, L.g, h->lev[l + 1].Ae, h->lev[l + 1].g, h->stream);
        CKL();
    }
    Level &C = h->lev[ng - 1];
    if (h->coarse_pcg) {
        // the coarsest operator as an FP64 stencil and 1 / diag for the PCG
        CK(cudaMemsetAsync(h->d_info, 0, sizeof(int), h->stream));
        launch_assemble_stencil<double>(C.Ae, C.fm, C.g, h->d_cst, h->d_cinvd, 1.0, true, h->stream);
        CKL();
        if (!h->small_built) TRY(build_small<T>(h));
        return sync(h);
    }
    launch_dense_assemble(C.Ae, C.fm, C.g, h->d_Adense, h->npad, h->stream);
    CKL();
    dense_sweep_inverse(h->d_Adense, h->d_sweepC, h->d_pinv, h->npad, h->d_info, h->stream);
    CKL();
    int info = 0;
    CK(cudaMemcpyAsync(&info, h->d_info, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    TRY(sync(h));
    if (info != 0) {
        h->err = "coarsest-grid inversion failed: non-positive pivot at dof " + std::to_string(info - 1);
        return TOSP_ERR_BREAKDOWN;
    }
    if (!h->small_built) TRY(build_small<T>(h));
    return TOSP_OK;
}

int check_len(tosp_handle *h, int64_t got, int64_t want, const char *what) {
    if (got != want) {
        h->err = std::string(what) + ": length " + std::to_string(got) + " != expected " + std::to_string(want);
        return TOSP_ERR_BAD_ARG;
    }
    return TOSP_OK;
}

int need_mg(tosp_handle *h) {
    if (!h->mg_ok) {
        h->err = h->mg_msg;
        return TOSP_ERR_UNSUPPORTED;
    }
    return TOSP_OK;
}

// Reads (and clears) the tensor-core operator's timeout flag; call after a
// stream synchronisation.
int check_tc(tosp_handle *h) {
    if (h->cpw.bar) {
        GridBarrier b{};
        CK(cudaMemcpy(&b, h->cpw.bar, sizeof b, cudaMemcpyDeviceToHost));
        if (b.err) {
            CK(cudaMemset(h->cpw.bar, 0, sizeof b));
            h->err = "coarsest-grid PCG: grid barrier wait timed out";
            return TOSP_ERR_TIMEOUT;
        }
    }
    if (h->d_bar) {
        GridBarrier b{};
        CK(cudaMemcpy(&b, h->d_bar, sizeof b, cudaMemcpyDeviceToHost));
        if (b.err) {
            CK(cudaMemset(h->d_bar, 0, sizeof b));
            h->err = "persistent coarse cycle: grid barrier wait timed out";
            return TOSP_ERR_TIMEOUT;
        }
    }
    if (!h->d_tcerr) return TOSP_OK;
    int e = 0;
    CK(cudaMemcpy(&e, h->d_tcerr, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        CK(cudaMemset(h->d_tcerr, 0, sizeof(int)));
        h->err = e == 2 ? "tensor-core operator: dynamic shared memory not 16-byte aligned"
                        : "tensor-core operator: wait for MMA completion timed out";
        return TOSP_ERR_TIMEOUT;
    }
    return TOSP_OK;
}

int need_setup(tosp_handle *h) {
    if (!h->setup_done) {
        h->err = "tosp_setup_gmg must be called first (densities/hierarchy missing)";
        return TOSP_ERR_STATE;
    }
    return TOSP_OK;
}

int read_scalars(tosp_handle *h) {
    CK(cudaMemcpyAsync(h->h_scal, h->d_scal, sizeof(double) * 8, cudaMemcpyDeviceToHost, h->stream));
    return sync(h);
}

// One iteration of I/SolveMG.m:31-52 from the current r, ending with an
// asynchronous copy of the scalars to pinned host memory.  mode: 1 first
// iteration, 0 reference beta, 2 flexible beta.
int cg_iteration(tosp_handle *h, int mode, int k) {
    Level &F = h->lev[0];
    const int64_t nd = F.g.ndof;
    const bool mixed = h->precision == TOSP_PREC_MIXED;
    // flexible beta: s of iteration k alternates between cso (k odd) and cs
    // (k even), so the previous s is in the other buffer without a copy
    const bool alt = h->mg.flexible && (k & 1);
    double *s = alt ? h->cso : h->cs;
    double *s_old = alt ? h->cs : h->cso;
    // iterations after the first find the V-cycle's input prepared by the
    // previous update (mixed precision)
    // the dots of the new s ride on the preconditioner's last sweep when it
    // writes s (post-smoothing), else they take their own pass
    h->fdot.r = h->cr;
    h->fdot.so = mode == 2 ? s_old : nullptr;
    h->fdot.o0 = h->d_scal + 0;
    h->fdot.o1 = h->d_scal + 5;
    h->fdot.want = true;
    h->fdot.done = false;
    const int prc = precondition(h, h->cr, s, mixed && mode != 1);
    h->fdot.want = false;
    TRY(prc);
    if (!h->fdot.done) {
        if (mode == 2) launch_dot2(h->cr, s, s_old, nd, h->d_partials, h->d_scal + 0, h->d_scal + 5, h->stream);
        else launch_dot(h->cr, s, nd, h->d_partials, h->d_scal + 0, h->stream);
    }
    launch_pcg_direction(h->cd, s, nullptr, h->d_scal, nd, mode, h->cx, h->stream, h->cg32 ? h->cd32 : nullptr);
    CKL();
    const bool first = mixed && fused_first_sweep(h);
    float *b0 = mixed ? (float *)F.b : nullptr;
    const float *invd0 = first ? (const float *)F.invd : nullptr;
    float *x0 = first ? (float *)F.x : nullptr;
    if (h->cg32) {
        TRY(fine_apply_cg32(h, h->cd32, h->cq32));
        launch_dot(h->cd, (const float *)h->cq32, nd, h->d_partials, h->d_scal + 2, h->stream);
        launch_pcg_update(h->cr, (const float *)h->cq32, h->d_scal, h->d_partials, nd, h->stream, b0, invd0, x0);
    } else {
        TRY(fine_apply64(h, h->cd, h->cq));
        launch_dot(h->cd, h->cq, nd, h->d_partials, h->d_scal + 2, h->stream);
        launch_pcg_update(h->cr, h->cq, h->d_scal, h->d_partials, nd, h->stream, b0, invd0, x0);
    }
    CKL();
    CK(cudaMemcpyAsync(h->h_scal, h->d_scal, sizeof(double) * 8, cudaMemcpyDeviceToHost, h->stream));
    return TOSP_OK;
}

// Capture the generic iteration (it >= 2) of one parity into a CUDA graph: all
// buffers are fixed per handle, so the graph is reused by every later solve.
// On any capture failure the solver keeps launching the same kernels one by one.
void capture_iteration(tosp_handle *h, int parity) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        h->graph_failed = true;
        return;
    }
    const int rc = cg_iteration(h, h->mg.flexible ? 2 : 0, parity);
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc != TOSP_OK || e != cudaSuccess || !g ||
        cudaGraphInstantiate(&h->iter_graph[parity], g, 0) != cudaSuccess) {
        cudaGetLastError();
        h->iter_graph[parity] = nullptr;
        h->graph_failed = true;
    }
    if (g) cudaGraphDestroy(g);
}

// r = f - K x and the norms of I/SolveMG.m:27-29; from a zero start (K 0 = 0
// exactly) r = f without the product.  Starts the loop state.
int solve_init(tosp_handle *h) {
    const int64_t nd = h->lev[0].g.ndof;
    launch_dot(h->cx, h->cx, nd, h->d_partials, h->d_scal + 3, h->stream);
    CKL();
    TRY(read_scalars(h));
    if (h->h_scal[3] == 0.0) {
        CK(cudaMemcpyAsync(h->cr, h->cf, sizeof(double) * nd, cudaMemcpyDeviceToDevice, h->stream));
    } else {
        TRY(fine_apply64(h, h->cx, h->cq));
        launch_residual<double>(h->cf, h->cq, h->cr, nd, h->stream);
        CKL();
    }
    launch_dot(h->cf, h->cf, nd, h->d_partials, h->d_scal + 4, h->stream);
    launch_dot(h->cr, h->cr, nd, h->d_partials, h->d_scal + 3, h->stream);
    CKL();
    TRY(read_scalars(h));
    SolveState &S = h->st;
    S.nf = std::sqrt(h->h_scal[4]);
    S.nr = std::sqrt(h->h_scal[3]) / S.nf;
    S.it = 1;
    S.rc = TOSP_OK;
    S.best = S.nr;
    S.best_it = 1;
    S.rmax = S.nr;
    S.replaced = 0;
    S.done = !(S.nr > h->mg.tolMG && S.it <= h->mg.maxiterMG);
    return TOSP_OK;
}

// Queue iteration S.it of I/SolveMG.m:30-52 on the handle's stream (the
// first one launched kernel by kernel, the others as the captured graph of
// their parity).
int solve_launch_iteration(tosp_handle *h) {
    const int it = h->st.it;
    if (it == 1) return cg_iteration(h, 1, it);
    const int par = it & 1;
    if (!h->iter_graph[par] && !h->graph_failed) capture_iteration(h, par);
    if (h->iter_graph[par]) {
        CK(cudaGraphLaunch(h->iter_graph[par], h->stream));
        return TOSP_OK;
    }
    return cg_iteration(h, h->mg.flexible ? 2 : 0, it);
}

// Loop bookkeeping after an iteration whose scalars reached h_scal: the
// breakdown test, the relative residual, the iteration counter, the stall
// test and the loop condition of I/SolveMG.m:30.
void solve_account(tosp_handle *h) {
    SolveState &S = h->st;
    const double rho = h->h_scal[0], dq = h->h_scal[2], rr = h->h_scal[3];
    // r'M^{-1}r may turn negative when the smoother is not convergent for
    // the chosen omega (the V-cycle is then indefinite); the reference
    // PCG carries on in that case, so only d'Kd <= 0 and non-finite
    // values stop the iteration.
    if (!(dq > 0.0) || !std::isfinite(rho) || !std::isfinite(rr)) {
        h->err = "CG breakdown: r'M^{-1}r = " + std::to_string(rho) + ", d'q = " + std::to_string(dq) +
                 ", r'r = " + std::to_string(rr);
        S.rc = TOSP_ERR_BREAKDOWN;
        S.done = true;
        return;
    }
    S.nr = std::sqrt(rr) / S.nf;
    ++S.it;
    if (S.nr <= 0.5 * S.best) {
        S.best = S.nr;
        S.best_it = S.it;
    }
    if (h->mg.maxstall > 0 && S.nr > h->mg.tolMG && S.it - S.best_it >= h->mg.maxstall) {
        h->err = "CG stalled: relative residual not halved in " + std::to_string(h->mg.maxstall) + " iterations";
        S.rc = TOSP_NOT_CONVERGED;
        S.done = true;
        return;
    }
    S.done = !(S.nr > h->mg.tolMG && S.it <= h->mg.maxiterMG);
}

// The last iteration's x += alpha d (the others ride on the direction
// update), the final status and the statistics.
int solve_finish(tosp_handle *h, int32_t *it_out, double *relres_out) {
    SolveState &S = h->st;
    if (S.it > 1) {
        launch_pcg_finish(h->cx, h->cd, h->d_scal, h->lev[0].g.ndof, h->stream);
        CKL();
    }
    if (S.rc == TOSP_OK && S.nr > h->mg.tolMG && S.it > h->mg.maxiterMG) S.rc = TOSP_NOT_CONVERGED;
    if (it_out) *it_out = S.it;
    if (relres_out) *relres_out = S.nr;
    h->stats.it = S.it;
    h->stats.relres = S.nr;
    h->stats.replacements = S.replaced;
    TRY(check_tc(h));
    return S.rc;
}

// cg_product 1, after solve_account: once the recurrence residual has fallen
// by replace_drop below the largest one since the last replacement, claims
// convergence, or the loop ends otherwise, the iterate update of this
// iteration is applied and r is replaced by the FP64 residual f - K x (FP64
// operator).  The search direction is kept; the loop then continues from the
// true residual, so convergence is only accepted on it.
int replace_residual(tosp_handle *h) {
    SolveState &S = h->st;
    if (!h->cg32 || S.rc == TOSP_ERR_BREAKDOWN) return TOSP_OK;
    if (S.nr > S.rmax) S.rmax = S.nr;
    if (!S.done && !(S.nr < h->mg.replace_drop * S.rmax)) return TOSP_OK;
    Level &F = h->lev[0];
    const int64_t nd = F.g.ndof;
    launch_pcg_finish(h->cx, h->cd, h->d_scal, nd, h->stream);
    CKL();
    // the update is applied: the next direction update and the final one add nothing
    CK(cudaMemsetAsync(h->d_scal + 6, 0, sizeof(double), h->stream));
    TRY(fine_apply64(h, h->cx, h->cq));
    const bool first = fused_first_sweep(h);
    launch_replace_residual(h->cf, h->cq, h->cr, h->d_scal, h->d_partials, nd, h->stream, (float *)F.b,
                            first ? (const float *)F.invd : nullptr, first ? (float *)F.x : nullptr);
    CKL();
    TRY(read_scalars(h));
    S.nr = std::sqrt(h->h_scal[3]) / S.nf;
    S.rmax = S.nr;
    ++S.replaced;
    if (S.rc == TOSP_OK) S.done = !(S.nr > h->mg.tolMG && S.it <= h->mg.maxiterMG);
    return TOSP_OK;
}

int solve_impl(tosp_handle *h, int32_t *it_out, double *relres_out) {
    TRY(solve_init(h));
    while (!h->st.done) {
        TRY(solve_launch_iteration(h));
        TRY(sync(h));
        solve_account(h);
        TRY(replace_residual(h));
    }
    return solve_finish(h, it_out, relres_out);
}

}  // namespace

// KelemProd on device free-dof vectors with caller-provided full-length
// scratch (xfull, yfull: ndof doubles each); allocates nothing.
int tosp::kelem_prod_with_scratch(tosp_handle *h, const double *x, double *y, int64_t nfree, double *xfull,
                                  double *yfull) {
    bool xd = false, yd = false;
    TRY(arg_location(h, x, "x", &xd));
    TRY(arg_location(h, y, "y", &yd));
    if (!xd || !yd) {
        h->err = "x and y must be device pointers (this entry point stages nothing)";
        return TOSP_ERR_BAD_ARG;
    }
    TRY(check_len(h, nfree, h->nfree, "x"));
    TRY(need_setup(h));
    CK(cudaMemsetAsync(xfull, 0, sizeof(double) * h->fg.g.ndof, h->stream));
    launch_scatter_free(x, h->d_freeidx, h->nfree, xfull, h->stream);
    CKL();
    TRY(fine_apply64(h, xfull, yfull));
    launch_gather_free(yfull, h->d_freeidx, h->nfree, y, h->stream);
    CKL();
    return sync(h);
}

// ----- serving-loop batches ----------------------------------------------------
#define CK_E(call, err)                                                  \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) {                                         \
            err = std::string("CUDA error: ") + cudaGetErrorString(e_); \
            return TOSP_ERR_CUDA;                                        \
        }                                                                \
    } while (0)

int tosp::solve_start(tosp_handle *h, const double *x, const double *f) {
    TRY(need_mg(h));
    TRY(need_setup(h));
    TRY(free_to_full(h, x, h->cx, "x"));
    TRY(free_to_full(h, f, h->cf, "f"));
    TRY(solve_init(h));
    if (!h->st.done) {
        TRY(solve_launch_iteration(h));
        TRY(sync(h));
        solve_account(h);
    }
    return TOSP_OK;
}

int tosp::solve_step_account(tosp_handle *h) {
    solve_account(h);
    return replace_residual(h);
}

int tosp::solve_step(tosp_handle *h) {
    TRY(solve_launch_iteration(h));
    TRY(sync(h));
    solve_account(h);
    return replace_residual(h);
}

const SolveState &tosp::solve_state(const tosp_handle *h) { return h->st; }

int tosp::solve_stop(tosp_handle *h, double *x, int32_t *it, double *relres) {
    const int rc = solve_finish(h, it, relres);
    if (rc < 0) return rc;
    TRY(full_to_free(h, h->cx, x, "x"));
    TRY(sync(h));
    return rc;
}

std::string tosp::batch_key(const tosp_handle *h) {
    std::string k;
    auto add = [&](const void *p, size_t n) { k.append(static_cast<const char *>(p), n); };
    add(&h->fg.g.nelx, sizeof(int) * 3);
    add(&h->n, sizeof(int));
    add(&h->precision, sizeof(int));
    add(&h->ngrids, sizeof(int));
    add(&h->small_l, sizeof(int));
    add(&h->small_n[0], sizeof(int) * 3);
    add(&h->mg.cycle, sizeof(int32_t));
    add(&h->mg.smoothiter1, sizeof(int32_t) * 2);
    add(&h->mg.flexible, sizeof(int32_t));
    return k;
}

int tosp::batch_prepare(BatchPlan &plan, cudaStream_t st, std::string &err) {
    const int nmem = (int)plan.mem.size();
    if (nmem < 1) {
        err = "empty batch";
        return TOSP_ERR_BAD_ARG;
    }
    tosp_handle *h0 = plan.mem[0];
    plan.fp64 = h0->precision == TOSP_PREC_FP64;
    for (int v = 0; v < 3; ++v) plan.maxsteps[v] = h0->small_l >= 0 ? h0->small_n[v] : 0;
    if (h0->small_l < 0) {
        plan.blocks = 0;   // no small levels: members' launches only
        return TOSP_OK;
    }
    for (tosp_handle *h : plan.mem)
        if (batch_key(h) != batch_key(h0)) {
            err = "batch members of different shapes";
            return TOSP_ERR_BAD_ARG;
        }
    // at most one block per SM: the launch then leaves room for the other
    // batches' kernels (a cooperative launch waits until all its blocks fit)
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h0->device);
    const int maxb = std::min(small_cycle_batch_max_blocks(plan.fp64), std::max(sms, 1));
    if (maxb < nmem) {
        err = "too many batch members for one cooperative launch";
        return TOSP_ERR_UNSUPPORTED;
    }
    // each member keeps its own launch size, scaled down to what is co-resident
    std::vector<int> nb(nmem);
    int64_t total = 0;
    for (int m = 0; m < nmem; ++m) total += nb[m] = std::max(1, plan.mem[m]->small_blocks);
    if (total > maxb) {
        const int64_t want = total;
        total = 0;
        for (int m = 0; m < nmem; ++m) total += nb[m] = (int)std::max<int64_t>(1, (int64_t)nb[m] * maxb / want);
    }
    while (total > maxb) {
        for (int m = 0; m < nmem && total > maxb; ++m)
            if (nb[m] > 1) --nb[m], --total;
    }
    std::vector<SmallBatchEntry> ent((size_t)3 * nmem);
    const size_t step_bytes = plan.fp64 ? sizeof(SmallStep<double>) : sizeof(SmallStep<float>);
    for (int v = 0; v < 3; ++v) {
        int b0 = 0;
        for (int m = 0; m < nmem; ++m) {
            SmallBatchEntry &e = ent[(size_t)v * nmem + m];
            e.steps = static_cast<const unsigned char *>(plan.mem[m]->d_steps) + step_bytes * (size_t)v * SMALL_MAX_STEPS;
            e.nsteps = plan.mem[m]->small_n[v];
            e.block0 = b0;
            e.nblocks = nb[m];
            e.pad = 0;
            b0 += nb[m];
        }
    }
    plan.blocks = (int)total;
    cudaError_t e = cudaMemcpyAsync(plan.d_ent, ent.data(), sizeof(SmallBatchEntry) * ent.size(),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(plan.d_bar, 0, sizeof(GridBarrier), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        err = std::string("batch tables: ") + cudaGetErrorString(e);
        return TOSP_ERR_CUDA;
    }
    return TOSP_OK;
}

// Capture the generic iteration of one parity as segments (once per handle:
// the buffers never move).
int capture_segments(tosp_handle *h, int parity) {
    h->seg_pending.clear();
    h->seg_count = 0;
    h->seg_capture = true;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? cg_iteration(h, h->mg.flexible ? 2 : 0, parity) : TOSP_ERR_CUDA;
    cudaGraph_t last = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(h->stream, &last);
    h->seg_capture = false;
    if (last) h->seg_pending.push_back(last);
    bool ok = rc == TOSP_OK && e == cudaSuccess && e2 == cudaSuccess && last &&
              (int)h->seg_pending.size() <= tosp_handle::MAXSEG;
    for (size_t i = 0; i < h->seg_pending.size(); ++i) {
        if (ok && cudaGraphInstantiate(&h->seg_graph[parity][i], h->seg_pending[i], 0) != cudaSuccess) ok = false;
        if (h->seg_pending[i]) cudaGraphDestroy(h->seg_pending[i]);
    }
    const int nseg = (int)h->seg_pending.size();
    h->seg_pending.clear();
    if (!ok) {
        cudaGetLastError();
        for (auto &g : h->seg_graph[parity])
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        h->seg_failed = true;
        h->err = "iteration segments could not be captured";
        return TOSP_ERR_CUDA;
    }
    h->nseg[parity] = nseg;
    return TOSP_OK;
}

int tosp::batch_tick(const BatchPlan &plan, cudaStream_t main, cudaEvent_t *ev_mem, cudaEvent_t ev_small,
                     std::string &err) {
    const int nmem = (int)plan.mem.size();
    int nseg = -1;
    for (tosp_handle *h : plan.mem) {
        const int par = h->st.it & 1;
        if (!h->seg_graph[par][0] && !h->seg_failed) capture_segments(h, par);
        if (h->seg_failed) {
            err = h->err;
            return TOSP_ERR_CUDA;
        }
        if (nseg < 0) nseg = h->nseg[par];
        if (h->nseg[par] != nseg) {
            err = "batch members with different iteration structures";
            return TOSP_ERR_STATE;
        }
    }
    tosp_handle *h0 = plan.mem[0];
    for (int i = 0; i < nseg; ++i) {
        for (tosp_handle *h : plan.mem) CK_E(cudaGraphLaunch(h->seg_graph[h->st.it & 1][i], h->stream), err);
        if (i + 1 == nseg) break;
        // visit i of every member: one batched persistent launch
        for (int m = 0; m < nmem; ++m) {
            CK_E(cudaEventRecord(ev_mem[m], plan.mem[m]->stream), err);
            CK_E(cudaStreamWaitEvent(main, ev_mem[m], 0), err);
        }
        const int v = h0->seg_variant[i];
        if (plan.fp64)
            launch_small_cycle_batch<double>(plan.d_ent + (size_t)v * nmem, nmem, plan.maxsteps[v], plan.d_bar,
                                             plan.blocks, main);
        else
            launch_small_cycle_batch<float>(plan.d_ent + (size_t)v * nmem, nmem, plan.maxsteps[v], plan.d_bar,
                                            plan.blocks, main);
        CK_E(cudaGetLastError(), err);
        CK_E(cudaEventRecord(ev_small, main), err);
        for (tosp_handle *h : plan.mem) CK_E(cudaStreamWaitEvent(h->stream, ev_small, 0), err);
    }
    return TOSP_OK;
}

int64_t tosp::handle_ndof(const tosp_handle *h) { return h->fg.g.ndof; }
int tosp::handle_device(const tosp_handle *h) { return h->device; }
cudaStream_t tosp::handle_stream(const tosp_handle *h) { return h->stream; }
void tosp::set_handle_error(tosp_handle *h, const std::string &msg) { h->err = msg; }

// =============================================================================
// C ABI
// =============================================================================
extern "C" {

const char *tosp_version(void) { return "tosp 0.1 (sm_100a)"; }

void tosp_default_mg_params(tosp_mg_params *mg) {
    if (!mg) return;
    mg->ngrids = 3;
    mg->cycle = 1;
    mg->smoother = 0;
    mg->omega = 0.5;
    mg->smoothiter1 = 1;
    mg->smoothiter2 = 1;
    mg->tolMG = 1e-8;
    mg->maxiterMG = 5000;
    mg->nmaxchol = 60000;
    mg->flexible = 0;
    mg->maxstall = 0;
    mg->warp_stencil_max = 0;
    mg->small_cycle_max = 0;
    mg->cg_product = 0;
    mg->replace_drop = 0.1;
    mg->opchol = 0;
    mg->opcond = 1;
    mg->tolPCG = 1e-8;
    mg->maxiterPCG = 10000;
}

int tosp_create(const tosp_problem *prob, const tosp_mg_params *mg, int32_t precision, tosp_handle **out) {
    TraceRange trace_("tosp_create");
    if (!out) {
        g_create_error = "null output handle pointer";
        return TOSP_ERR_BAD_ARG;
    }
    *out = nullptr;
    tosp_handle *h = new (std::nothrow) tosp_handle();
    if (!h) {
        g_create_error = "host allocation failed";
        return TOSP_ERR_OOM;
    }
    const int rc = create_impl(h, prob, mg, precision);
    if (rc != TOSP_OK) {
        g_create_error = h->err;
        tosp_destroy(h);
        return rc;
    }
    *out = h;
    return TOSP_OK;
}

int tosp_destroy(tosp_handle *h) {
    if (!h) return TOSP_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (cudaGraphExec_t gx : h->iter_graph)
        if (gx) cudaGraphExecDestroy(gx);
    for (auto &row : h->seg_graph)
        for (cudaGraphExec_t gx : row)
            if (gx) cudaGraphExecDestroy(gx);
    for (void *p : h->allocs) cudaFree(p);
    if (h->h_scal) cudaFreeHost(h->h_scal);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return TOSP_OK;
}

const char *tosp_last_error(const tosp_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int tosp_info(const tosp_handle *h, int32_t *ngrids, int64_t *ncoarse, int64_t *device_bytes) {
    if (!h) return TOSP_ERR_BAD_ARG;
    if (ngrids) *ngrids = h->ngrids;
    if (ncoarse) *ncoarse = h->ncoarse;
    if (device_bytes) *device_bytes = h->bytes;
    return TOSP_OK;
}

int tosp_set_freedofs(tosp_handle *h, const int64_t *freedofs, int64_t nfree) {
    if (!h || !freedofs || nfree <= 0) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    return build_masks(h, freedofs, nfree);
}

int tosp_setup_gmg(tosp_handle *h, const double *xfil, int64_t ndens) {
    TraceRange trace_("SetupGMG");
    if (!h || !xfil) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(check_len(h, ndens, h->dens.nelem, "densities"));
    CK(cudaEventRecord(h->ev0, h->stream));
    TRY(load_vec(h, h->d_rho, xfil, ndens));
    launch_simp(h->d_rho, h->d_w64, h->d_wbf, h->d_wq, h->d_w32, ndens, h->p, h->emin, h->E, h->stream);
    CKL();
    h->setup_done = false;
    if (h->mg_ok) {
        const int rc = h->precision == TOSP_PREC_FP64 ? setup_levels<double>(h) : setup_levels<float>(h);
        if (rc != TOSP_OK) return rc;
    }
    CK(cudaEventRecord(h->ev1, h->stream));
    TRY(sync(h));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.ms_setup = ms;
    h->setup_done = true;
    return TOSP_OK;
}

int tosp_kelem_prod(tosp_handle *h, const double *x, double *y, int64_t nfree) {
    TraceRange trace_("KelemProd");
    if (!h || !x || !y) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(check_len(h, nfree, h->nfree, "x"));
    TRY(need_setup(h));
    TRY(free_to_full(h, x, h->cd, "x"));
    TRY(fine_apply64(h, h->cd, h->cq));
    TRY(full_to_free(h, h->cq, y, "y"));
    return sync(h);
}

int tosp_kelem_prod_mixed(tosp_handle *h, const double *x, double *y, int64_t nfree) {
    TraceRange trace_("KelemProdMixed");
    if (!h || !x || !y) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    if (h->precision != TOSP_PREC_MIXED) {
        h->err = "the FP32/BF16 operator exists only on TOSP_PREC_MIXED handles";
        return TOSP_ERR_STATE;
    }
    TRY(check_len(h, nfree, h->nfree, "x"));
    TRY(need_setup(h));
    Level &F = h->lev[0];
    const int64_t nd = F.g.ndof;
    TRY(free_to_full(h, x, h->cd, "x"));
    launch_convert<double, float>(h->cd, (float *)F.x, nd, h->stream);
    CKL();
    TRY(fine_apply<float>(h, (const float *)F.x, (float *)F.t));
    launch_convert<float, double>((const float *)F.t, h->cq, nd, h->stream);
    CKL();
    TRY(full_to_free(h, h->cq, y, "y"));
    TRY(sync(h));
    return check_tc(h);
}

int tosp_kelem_prod_cg32(tosp_handle *h, const double *x, double *y, int64_t nfree) {
    TraceRange trace_("KelemProdCG32");
    if (!h || !x || !y) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    if (!h->cg32) {
        h->err = "the CG's tensor-core product exists only on handles created with cg_product 1";
        return TOSP_ERR_STATE;
    }
    TRY(check_len(h, nfree, h->nfree, "x"));
    TRY(need_setup(h));
    const int64_t nd = h->lev[0].g.ndof;
    TRY(free_to_full(h, x, h->cd, "x"));
    launch_convert<double, float>(h->cd, h->cd32, nd, h->stream);
    CKL();
    TRY(fine_apply_cg32(h, h->cd32, h->cq32));
    launch_convert<float, double>(h->cq32, h->cq, nd, h->stream);
    CKL();
    TRY(full_to_free(h, h->cq, y, "y"));
    TRY(sync(h));
    return check_tc(h);
}

int tosp_mg_cycle(tosp_handle *h, const double *r, double *s, int64_t nfree) {
    TraceRange trace_("MGCycle");
    if (!h || !r || !s) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(check_len(h, nfree, h->nfree, "r"));
    TRY(need_mg(h));
    TRY(need_setup(h));
    TRY(free_to_full(h, r, h->cr, "r"));
    TRY(precondition(h, h->cr, h->cs));
    TRY(full_to_free(h, h->cs, s, "s"));
    TRY(sync(h));
    return check_tc(h);
}

int tosp_solve_mg(tosp_handle *h, double *x, const double *f, int64_t nfree, int32_t *it, double *relres) {
    TraceRange trace_("SolveMG");
    if (!h || !x || !f) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(check_len(h, nfree, h->nfree, "x/f"));
    TRY(need_mg(h));
    TRY(need_setup(h));
    CK(cudaEventRecord(h->ev0, h->stream));
    TRY(free_to_full(h, x, h->cx, "x"));
    TRY(free_to_full(h, f, h->cf, "f"));
    const int rc = solve_impl(h, it, relres);
    if (rc < 0) return rc;
    TRY(full_to_free(h, h->cx, x, "x"));
    CK(cudaEventRecord(h->ev1, h->stream));
    TRY(sync(h));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.ms_solve = ms;
    if (metrics_on()) {
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "{\"event\": \"solve\", \"ndof\": %lld, \"precision\": %d, \"it\": %d, \"relres\": %.6e, "
                      "\"ms\": %.3f, \"status\": %d}",
                      (long long)h->fg.g.ndof, h->precision, h->st.it, h->st.nr, ms, rc);
        metrics_line(buf);
    }
    return rc;
}

int tosp_apply_filter(tosp_handle *h, const double *x, double *y, int64_t ndens, int32_t trans) {
    TraceRange trace_("ApplyFilter");
    if (!h || !x || !y) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(check_len(h, ndens, h->dens.nelem, "x"));
    bool din = false, dout = false;
    TRY(arg_location(h, x, "x", &din));
    TRY(arg_location(h, y, "y", &dout));
    const double *src = x;
    if (!din) {
        TRY(load_vec(h, h->d_g0, x, ndens));
        src = h->d_g0;
    }
    double *dst = dout ? y : h->d_gf;
    if (h->opfilter == 0 || h->ntaps == 0) {
        CK(cudaMemcpyAsync(dst, src, sizeof(double) * ndens, cudaMemcpyDefault, h->stream));
    } else {
        launch_filter(src, dst, h->d_fw, h->d_fixed, h->d_taps, h->ntaps, h->dens.nelx, h->dens.nely, h->dens.nelz,
                      trans ? 1 : 0, 0, h->filt_r, h->stream);
        CKL();
    }
    if (!dout) TRY(store_vec(h, y, dst, ndens));
    return sync(h);
}

int tosp_filter_weights(tosp_handle *h, double *w, int64_t ndens) {
    if (!h || !w) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(check_len(h, ndens, h->dens.nelem, "w"));
    if (h->opfilter == 0) {
        h->err = "no filter (opfilter = 0)";
        return TOSP_ERR_STATE;
    }
    TRY(store_vec(h, w, h->d_fw, ndens));
    return sync(h);
}

int tosp_grad(tosp_handle *h, const double *u, int64_t nfull, double *fgrad, double *fgrad0, int64_t ndens) {
    TraceRange trace_("Grad");
    if (!h || !u || !fgrad) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(check_len(h, nfull, h->lev[0].g.ndof, "u"));
    TRY(check_len(h, ndens, h->dens.nelem, "fgrad"));
    TRY(need_setup(h));
    const double *du = u;
    bool udev = false, dout = false;
    TRY(arg_location(h, u, "u", &udev));
    TRY(arg_location(h, fgrad, "fgrad", &dout));
    if (!udev) {
        TRY(load_vec(h, h->d_ufull, u, nfull));
        du = h->d_ufull;
    }
    launch_grad(du, h->d_rho, h->d_free_elem, h->d_ke64, h->d_g0, h->fg, h->n, h->p, h->emin, h->E, h->stream);
    CKL();
    double *dst = dout ? fgrad : h->d_gf;
    if (h->opfilter == 0 || h->ntaps == 0) {
        CK(cudaMemcpyAsync(dst, h->d_g0, sizeof(double) * ndens, cudaMemcpyDeviceToDevice, h->stream));
    } else {
        launch_filter(h->d_g0, dst, h->d_fw, h->d_fixed, h->d_taps, h->ntaps, h->dens.nelx, h->dens.nely,
                      h->dens.nelz, 1, 0, h->filt_r, h->stream);
        CKL();
    }
    if (!dout) TRY(store_vec(h, fgrad, dst, ndens));
    if (fgrad0) TRY(store_vec(h, fgrad0, h->d_g0, ndens));
    return sync(h);
}

int tosp_compliance(tosp_handle *h, const double *f, const double *u, int64_t nfree, double *F) {
    if (!h || !f || !u || !F) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(check_len(h, nfree, h->nfree, "f/u"));
    TRY(ensure_stage(h, nfree));
    TRY(load_vec(h, h->d_stage_a, f, nfree));
    TRY(load_vec(h, h->d_stage_b, u, nfree));
    launch_dot(h->d_stage_a, h->d_stage_b, nfree, h->d_partials, h->d_scal + 8, h->stream);
    CKL();
    CK(cudaMemcpyAsync(h->h_scal + 8, h->d_scal + 8, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TRY(sync(h));
    *F = h->h_scal[8];
    return TOSP_OK;
}

int tosp_last_stats(const tosp_handle *h, tosp_solve_stats *st) {
    if (!h || !st) return TOSP_ERR_BAD_ARG;
    *st = h->stats;
    return TOSP_OK;
}

int64_t tosp_kernel_launches(void) { return (int64_t)launch_count(); }

int tosp_time_operator(tosp_handle *h, int32_t precision, int32_t reps, double *ms_per_launch) {
    if (!h || !ms_per_launch || reps < 1) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    TRY(need_setup(h));
    if (precision < 0 || precision > 2) return TOSP_ERR_BAD_ARG;
    if (precision == TOSP_PREC_MIXED && h->precision != TOSP_PREC_MIXED) {
        h->err = "the FP32/BF16 operator exists only on TOSP_PREC_MIXED handles";
        return TOSP_ERR_STATE;
    }
    if (precision == 2 && !h->cg32) {
        h->err = "the CG's tensor-core product exists only on handles created with cg_product 1";
        return TOSP_ERR_STATE;
    }
    const Grid &g0 = h->lev[0].g;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    double total = 0.0;
    for (int r = 0; r < reps; ++r) {
        if (precision == TOSP_PREC_FP64) {
            CK(cudaMemsetAsync(h->cq, 0, sizeof(double) * g0.ndof, h->stream));
            CK(cudaEventRecord(a, h->stream));
            launch_fine64(h, h->cd, h->cq);
        } else if (precision == 2) {
            CK(cudaMemsetAsync(h->cq32, 0, sizeof(float) * g0.ndof, h->stream));
            CK(cudaEventRecord(a, h->stream));
            launch_fine_apply_tc_w32(h->cd32, h->cq32, h->d_w32, h->lev[0].fm, h->d_tcimg32, h->fg, h->n, h->d_tcerr,
                                     h->stream);
        } else {
            Level &F = h->lev[0];
            CK(cudaMemsetAsync(F.t, 0, sizeof(float) * g0.ndof, h->stream));
            CK(cudaEventRecord(a, h->stream));
            if (h->d_tcimg)
                launch_fine_apply_tc((const float *)F.x, (float *)F.t, h->d_wbf, F.fm, h->d_tcimg, h->fg, h->n,
                                     h->d_tcerr, h->stream);
            else
                launch_fine_apply<float, __nv_bfloat16>((const float *)F.x, (float *)F.t, h->d_wbf, F.fm, h->d_kt32,
                                                        h->fg, h->n, h->stream);
        }
        CKL();
        CK(cudaEventRecord(b, h->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        total += ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms_per_launch = total / reps;
    return check_tc(h);
}

int tosp_inject_wait_fault(tosp_handle *h, int32_t polls, int32_t skip_block) {
    if (!h || polls < 1 || skip_block < -1) return TOSP_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    if (!h->d_bar || h->small_l < 0) {
        h->err = "no persistent small-level cycle on this handle (set small_cycle_max and run tosp_setup_gmg)";
        return TOSP_ERR_STATE;
    }
    if (skip_block >= h->small_blocks) {
        h->err = "skip_block beyond the cycle's " + std::to_string(h->small_blocks) + " blocks";
        return TOSP_ERR_BAD_ARG;
    }
    CK(cudaStreamSynchronize(h->stream));
    GridBarrier b{};
    CK(cudaMemcpy(&b, h->d_bar, sizeof b, cudaMemcpyDeviceToHost));
    b.limit = (unsigned)polls;
    b.skip = skip_block + 1;
    CK(cudaMemcpy(h->d_bar, &b, sizeof b, cudaMemcpyHostToDevice));
    return TOSP_OK;
}

int tosp_small_cycle_blocks(const tosp_handle *h, int32_t *blocks) {
    if (!h || !blocks) return TOSP_ERR_BAD_ARG;
    *blocks = h->small_l >= 0 ? h->small_blocks : 0;
    return TOSP_OK;
}

int tosp_elem_stiff_mr(double el, double eh, double ew, double nu, int32_t n, double *kv) {
    if (!kv || n < 1 || n > 4 || !(el > 0) || !(eh > 0) || !(ew > 0)) return TOSP_ERR_BAD_ARG;
    std::vector<double> ks;
    elem_stiff_mr(el, eh, ew, nu, n, ks);
    const int ns = n * n * n;
    for (int s = 0; s < ns; ++s)
        for (int j = 0; j < 24; ++j)
            for (int i = 0; i < 24; ++i) kv[(size_t)s * 576 + j * 24 + i] = ks[(size_t)s * 576 + i * 24 + j];
    return TOSP_OK;
}

}  // extern "C"
