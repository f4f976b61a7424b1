// Multigrid levels: Galerkin coarse operators, stencil products, Jacobi
// smoothing and the trilinear transfers.
//
// The reference forms A{l+1} = P{l}' A{l} P{l} with sparse products
// (I/SetupGMG.m:45-49, I/StrSLP.m:345-346), P restricted to the free rows and
// columns (I/Prolongation.m:53-55).  Here the same matrix is built element by
// element: a coarse element E is the union of 8 children c, and
//     Abar_E = sum_c  Pi_c' (M_c K_c M_c) Pi_c,
// where Pi_c = W_c (x) I3 interpolates E's 8 nodes to c's 8 nodes and M_c zeroes
// the child's fixed dofs.  Summing Abar_E over E and zeroing the coarse fixed
// dofs gives P'AP on the free dofs exactly.  For the apply, the element
// matrices are assembled into a 27-point node stencil of 3x3 blocks.
#include "tosp_internal.h"

namespace tosp {

static int num_sms_c() {
    static int n = 0;
    if (!n) {
        int dev;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    }
    return n;
}

static unsigned grid_for(int64_t n, int threads, int max_per_sm = 16) {
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)max_per_sm * num_sms_c();
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

// (x, y, z) of node I (y fastest); 32-bit division whenever the index fits.
__device__ __forceinline__ void node_xyz(int64_t I, int ny, int nx, int &x, int &y, int &z) {
    if (I <= 0x7fffffff) {
        const int i = (int)I, q = i / ny;
        y = i - q * ny;
        z = q / nx;
        x = q - z * nx;
    } else {
        const int64_t q = I / ny;
        y = (int)(I - q * ny);
        z = (int)(q / nx);
        x = (int)(q - (int64_t)z * nx);
    }
}

__device__ __forceinline__ double phi1(int f, int A) {
    const int d = f - 2 * A;
    return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0);
}

// Interpolation weight of coarse local node A at the local node a of child c.
__device__ __forceinline__ double wchild(int c, int a, int A) {
    const int cdx = (c >> 1) & 1, cdy = c & 1, cdz = (c >> 2) & 1;
    const int ax = (a >> 1) & 1, ay = a & 1, az = (a >> 2) & 1;
    const int Ax = (A >> 1) & 1, Ay = A & 1, Az = (A >> 2) & 1;
    return phi1(cdx + ax, Ax) * phi1(cdy + ay, Ay) * phi1(cdz + az, Az);
}

__device__ __forceinline__ int pidx(int i, int j) {   // packed upper index, i <= j
    return i * 24 - (i * (i - 1)) / 2 + (j - i);
}

constexpr int CB_THREADS = 192;   // 576 / 3 entries per thread

// One CTA per coarse element: accumulate the 8 children's triple products.
// FROM_FINE: children are fine elements, K_c = sum_s w_s KE_s;
// otherwise K_c is the stored element matrix of the finer level.
template <bool FROM_FINE, int N>
__global__ void __launch_bounds__(CB_THREADS)
k_coarse_build(const double *__restrict__ w, const double *__restrict__ kepack, const double *__restrict__ Af,
               const uint8_t *__restrict__ fmask, Grid gf, int nelx_d, int nely_d, double *__restrict__ Ac,
               Grid gc, int only_fixed) {
    constexpr int NS = N * N * N;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *ke = reinterpret_cast<double *>(smem_raw);          // NS*300 (FROM_FINE only)
    double *Kc = ke + (FROM_FINE ? NS * KE_PACK : 0);            // 576
    double *T = Kc + 576;                                        // 576
    double *Wc = T + 576;                                        // 64
    double *wsub = Wc + 64;                                      // NS
    uint8_t *fr = reinterpret_cast<uint8_t *>(wsub + NS);        // 24
    const int tid = threadIdx.x;
    if (FROM_FINE)
        for (int i = tid; i < NS * KE_PACK; i += CB_THREADS) ke[i] = kepack[i];

    for (int64_t E = blockIdx.x; E < gc.nelem; E += gridDim.x) {
        const int cy = (int)(E % gc.nely), cx = (int)((E / gc.nely) % gc.nelx),
                  cz = (int)(E / ((int64_t)gc.nely * gc.nelx));
        if (only_fixed) {
            // elements whose 27 fine nodes are all free were built from the table
            bool fixed = false;
            if (tid < 81) {
                const int nd = tid / 3, comp = tid % 3;
                const int64_t node = ((int64_t)(2 * cz + nd / 9) * gf.nx + (2 * cx + (nd / 3) % 3)) * gf.ny +
                                     (2 * cy + nd % 3);
                fixed = !fmask[3 * node + comp];
            }
            if (!__syncthreads_or(fixed)) continue;
        }
        double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
        for (int c = 0; c < 8; ++c) {
            const int fx = 2 * cx + ((c >> 1) & 1), fy = 2 * cy + (c & 1), fz = 2 * cz + ((c >> 2) & 1);
            __syncthreads();
            if (tid < 64) Wc[tid] = wchild(c, tid >> 3, tid & 7);
            if (tid < 24) {
                const int a = tid / 3, comp = tid % 3;
                const int64_t node = ((int64_t)(fz + ((a >> 2) & 1)) * gf.nx + (fx + ((a >> 1) & 1))) * gf.ny +
                                     (fy + (a & 1));
                fr[tid] = fmask[3 * node + comp];
            }
            if (FROM_FINE && tid < NS) {
                const int s = tid, sy = s % N, sx = (s / N) % N, sz = s / (N * N);
                wsub[s] = w[((int64_t)(fz * N + sz) * nelx_d + (fx * N + sx)) * nely_d + (fy * N + sy)];
            }
            __syncthreads();
            const int64_t child = ((int64_t)fz * gf.nelx + fx) * gf.nely + fy;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int e = tid + r * CB_THREADS;
                const int i = e / 24, j = e % 24;
                double v;
                if (FROM_FINE) {
                    const int pi = i <= j ? pidx(i, j) : pidx(j, i);
                    v = 0.0;
                    for (int s = 0; s < NS; ++s) v += wsub[s] * ke[s * KE_PACK + pi];
                } else {
                    v = Af[child * 576 + e];
                }
                Kc[e] = (fr[i] && fr[j]) ? v : 0.0;
            }
            __syncthreads();
            // T[i][B*3+cb] = sum_b Kc[i][b*3+cb] W[b][B]
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int e = tid + r * CB_THREADS;
                const int i = e / 24, j = e % 24, B = j / 3, cb = j % 3;
                double v = 0.0;
#pragma unroll
                for (int b = 0; b < 8; ++b) v += Kc[i * 24 + b * 3 + cb] * Wc[b * 8 + B];
                T[e] = v;
            }
            __syncthreads();
            // Abar[A*3+ca][j] += sum_a W[a][A] T[a*3+ca][j]
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int e = tid + r * CB_THREADS;
                const int i = e / 24, j = e % 24, A = i / 3, ca = i % 3;
                double v = 0.0;
#pragma unroll
                for (int a = 0; a < 8; ++a) v += Wc[a * 8 + A] * T[(a * 3 + ca) * 24 + j];
                acc[r] += v;
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) Ac[E * 576 + tid + r * CB_THREADS] = acc[r];
    }
}

template <bool FROM_FINE, int N>
static void launch_cb(const double *w, const double *kepack, const double *Af, const uint8_t *fm, const Grid &gf,
                      int nelx_d, int nely_d, double *Ac, const Grid &gc, cudaStream_t st, int only_fixed = 0) {
    constexpr int NS = N * N * N;
    const size_t smem = sizeof(double) * ((FROM_FINE ? NS * KE_PACK : 0) + 576 * 2 + 64 + NS) + 32;
    auto kern = k_coarse_build<FROM_FINE, N>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, CB_THREADS, smem);
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)per_sm * num_sms_c();
    if (grid > gc.nelem) grid = gc.nelem;
    kern<<<(unsigned)grid, CB_THREADS, smem, st>>>(w, kepack, Af, fm, gf, nelx_d, nely_d, Ac, gc, only_fixed);
    count_launch();
}

// Finest coarsening from the sub-cell table: Abar_E = sum_q w_q S_q over the
// 8 n^3 density cells q of coarse element E, valid when none of E's 27 fine
// nodes has a fixed dof (then M_c = I in every triple product).  A CTA of
// TB_THREADS threads takes TB_ELEMS coarse elements at a time; thread t owns
// packed entry t for all of them, reading S_q[t] once per cell.  Elements with
// a fixed fine dof are left for the masked kernel.
constexpr int TB_THREADS = 320;
constexpr int TB_ELEMS = 8;

template <int N>
__global__ void __launch_bounds__(TB_THREADS, 2)
k_coarse_table(const double *__restrict__ w, const uint8_t *__restrict__ fmask, const double *__restrict__ S,
               Grid gf, int nelx_d, int nely_d, double *__restrict__ Ac, Grid gc) {
    constexpr int Q = 8 * N * N * N;
    __shared__ double ws[TB_ELEMS * Q];
    __shared__ int fixed[TB_ELEMS];
    const int tid = threadIdx.x;
    int ti = 0, tj = 0;
    if (tid < KE_PACK) {   // packed upper index -> (i, j), row-major
        int t = tid;
        while (t >= 24 - ti) {
            t -= 24 - ti;
            ++ti;
        }
        tj = ti + t;
    }
    for (int64_t E0 = (int64_t)blockIdx.x * TB_ELEMS; E0 < gc.nelem; E0 += (int64_t)gridDim.x * TB_ELEMS) {
        __syncthreads();
        if (tid < TB_ELEMS) fixed[tid] = 0;
        __syncthreads();
        for (int k = tid; k < TB_ELEMS * Q; k += TB_THREADS) {
            const int e = k / Q, q = k - e * Q;
            const int64_t E = E0 + e;
            double v = 0.0;
            if (E < gc.nelem) {
                const int cy = (int)(E % gc.nely), cx = (int)((E / gc.nely) % gc.nelx),
                          cz = (int)(E / ((int64_t)gc.nely * gc.nelx));
                const int c = q / (N * N * N), sidx = q - c * N * N * N;
                const int fx = 2 * cx + ((c >> 1) & 1), fy = 2 * cy + (c & 1), fz = 2 * cz + ((c >> 2) & 1);
                const int sy = sidx % N, sx = (sidx / N) % N, sz = sidx / (N * N);
                v = w[((int64_t)(fz * N + sz) * nelx_d + (fx * N + sx)) * nely_d + (fy * N + sy)];
            }
            ws[k] = v;
        }
        for (int k = tid; k < TB_ELEMS * 81; k += TB_THREADS) {
            const int e = k / 81, r = k - e * 81, nd = r / 3, comp = r % 3;
            const int64_t E = E0 + e;
            if (E >= gc.nelem) continue;
            const int cy = (int)(E % gc.nely), cx = (int)((E / gc.nely) % gc.nelx),
                      cz = (int)(E / ((int64_t)gc.nely * gc.nelx));
            const int64_t node = ((int64_t)(2 * cz + nd / 9) * gf.nx + (2 * cx + (nd / 3) % 3)) * gf.ny +
                                 (2 * cy + nd % 3);
            if (!fmask[3 * node + comp]) fixed[e] = 1;
        }
        __syncthreads();
        if (tid < KE_PACK) {
            double acc[TB_ELEMS];
#pragma unroll
            for (int e = 0; e < TB_ELEMS; ++e) acc[e] = 0.0;
#pragma unroll 4
            for (int q = 0; q < Q; ++q) {
                const double sq = S[(size_t)q * KE_PACK + tid];
#pragma unroll
                for (int e = 0; e < TB_ELEMS; ++e) acc[e] += ws[e * Q + q] * sq;
            }
#pragma unroll
            for (int e = 0; e < TB_ELEMS; ++e) {
                const int64_t E = E0 + e;
                if (E >= gc.nelem || fixed[e]) continue;
                Ac[E * 576 + ti * 24 + tj] = acc[e];
                if (ti != tj) Ac[E * 576 + tj * 24 + ti] = acc[e];
            }
        }
    }
}

template <int N>
static void launch_table(const double *w, const uint8_t *fm, const double *S, const FineGeom &fg, double *Ac,
                         const Grid &gc, cudaStream_t st) {
    int64_t grid = (gc.nelem + TB_ELEMS - 1) / TB_ELEMS;
    const int64_t cap = (int64_t)4 * num_sms_c();
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    k_coarse_table<N><<<(unsigned)grid, TB_THREADS, 0, st>>>(w, fm, S, fg.g, fg.nelx_d, fg.nely_d, Ac, gc);
    count_launch();
}

void launch_coarse_from_fine_table(const double *w, const uint8_t *freemask_f, const double *kepack, const double *S,
                                   double *Ac, const FineGeom &fg, const Grid &gc, int n, cudaStream_t st) {
    if (n == 1) {
        launch_table<1>(w, freemask_f, S, fg, Ac, gc, st);
        launch_cb<true, 1>(w, kepack, nullptr, freemask_f, fg.g, fg.nelx_d, fg.nely_d, Ac, gc, st, 1);
    } else if (n == 2) {
        launch_table<2>(w, freemask_f, S, fg, Ac, gc, st);
        launch_cb<true, 2>(w, kepack, nullptr, freemask_f, fg.g, fg.nelx_d, fg.nely_d, Ac, gc, st, 1);
    } else {
        launch_table<3>(w, freemask_f, S, fg, Ac, gc, st);
        launch_cb<true, 3>(w, kepack, nullptr, freemask_f, fg.g, fg.nelx_d, fg.nely_d, Ac, gc, st, 1);
    }
}

void launch_coarse_from_coarse(const double *Af, const uint8_t *freemask_f, const Grid &gf, double *Ac,
                               const Grid &gc, cudaStream_t st) {
    launch_cb<false, 1>(nullptr, nullptr, Af, freemask_f, gf, 0, 0, Ac, gc, st);
}

// ---------------------------------------------------------------------------
// 27-point stencil assembly: block (I, I+o) = sum over the elements holding
// both nodes of the matching 3x3 block, with the level's fixed dofs zeroed.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_assemble_stencil(const double *__restrict__ Ae, const uint8_t *__restrict__ fmask, Grid g,
                                   T *__restrict__ stv, T *__restrict__ invdiag, double omega, int node_major) {
    for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < g.nnodes;
         I += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        node_xyz(I, g.ny, g.nx, x, y, z);
        uint8_t fi[3];
        for (int c = 0; c < 3; ++c) fi[c] = fmask[3 * I + c];
        for (int o = 0; o < 27; ++o) {
            const int oy = o % 3 - 1, ox = (o / 3) % 3 - 1, oz = o / 9 - 1;
            double blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            const int jx = x + ox, jy = y + oy, jz = z + oz;
            const bool jin = jx >= 0 && jx < g.nx && jy >= 0 && jy < g.ny && jz >= 0 && jz < g.nz;
            uint8_t fj[3] = {0, 0, 0};
            if (jin) {
                const int64_t J = ((int64_t)jz * g.nx + jx) * g.ny + jy;
                for (int c = 0; c < 3; ++c) fj[c] = fmask[3 * J + c];
                for (int d = 0; d < 8; ++d) {
                    const int dx = (d >> 1) & 1, dy = d & 1, dz = (d >> 2) & 1;
                    const int bx = dx + ox, by = dy + oy, bz = dz + oz;
                    if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
                    const int exx = x - dx, eyy = y - dy, ezz = z - dz;
                    if (exx < 0 || exx >= g.nelx || eyy < 0 || eyy >= g.nely || ezz < 0 || ezz >= g.nelz) continue;
                    const int64_t E = ((int64_t)ezz * g.nelx + exx) * g.nely + eyy;
                    const int aI = dz * 4 + dx * 2 + dy, aJ = bz * 4 + bx * 2 + by;
                    const double *m = Ae + E * 576;
                    for (int ci = 0; ci < 3; ++ci)
                        for (int cj = 0; cj < 3; ++cj) blk[ci * 3 + cj] += m[(aI * 3 + ci) * 24 + aJ * 3 + cj];
                }
            }
            for (int ci = 0; ci < 3; ++ci)
                for (int cj = 0; cj < 3; ++cj) {
                    const double v = (fi[ci] && fj[cj]) ? blk[ci * 3 + cj] : 0.0;
                    const int k = o * 9 + ci * 3 + cj;
                    if (node_major) stv[I * STENCIL_VALS + k] = (T)v;
                    else if (o >= 13) stv[(int64_t)(k - 13 * 9) * g.nnodes + I] = (T)v;
                    if (o == 13 && ci == cj) invdiag[3 * I + ci] = (T)((fi[ci] && v != 0.0) ? omega / v : 0.0);
                }
        }
    }
}

template <typename T>
void launch_assemble_stencil(const double *Ae, const uint8_t *freemask, const Grid &g, T *stencil, T *invdiag,
                             double omega, bool node_major, cudaStream_t st) {
    k_assemble_stencil<T><<<grid_for(g.nnodes, 128), 128, 0, st>>>(Ae, freemask, g, stencil, invdiag, omega,
                                                                    node_major ? 1 : 0);
    count_launch();
}
template void launch_assemble_stencil<double>(const double *, const uint8_t *, const Grid &, double *, double *,
                                              double, bool, cudaStream_t);
template void launch_assemble_stencil<float>(const double *, const uint8_t *, const Grid &, float *, float *,
                                             double, bool, cudaStream_t);

// ---------------------------------------------------------------------------
// Stencil products.  One thread per node, 3 dofs.  The offset-major layout
// keeps only the centre and the 13 "upper" offsets (o >= 13, 126 values per
// node): the block of a lower offset o is the transpose of the block stored
// at the neighbour J = I + off(o) for the opposite offset 26 - o, so the
// stencil's bytes are halved and the transposed reads hit nearby z-planes,
// which stay in L2.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128)
k_stencil(const T *__restrict__ stv, const T *__restrict__ x, const T *__restrict__ b, const T *__restrict__ invdiag,
          T *__restrict__ y, Grid g, int mode) {
    for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < g.nnodes;
         I += (int64_t)gridDim.x * blockDim.x) {
        int xx, yy, zz;
        node_xyz(I, g.ny, g.nx, xx, yy, zz);
        T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
        for (int o = 0; o < 27; ++o) {
            const int oy = o % 3 - 1, ox = (o / 3) % 3 - 1, oz = o / 9 - 1;
            const int jx = xx + ox, jy = yy + oy, jz = zz + oz;
            if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz) continue;
            const int64_t J = I + ((int64_t)oz * g.nx + ox) * g.ny + oy;
            const T x0 = x[3 * J], x1 = x[3 * J + 1], x2 = x[3 * J + 2];
            if (o >= 13) {
                const T *s = stv + (int64_t)((o - 13) * 9) * g.nnodes + I;
                a0 += s[0] * x0 + s[g.nnodes] * x1 + s[2 * g.nnodes] * x2;
                a1 += s[3 * g.nnodes] * x0 + s[4 * g.nnodes] * x1 + s[5 * g.nnodes] * x2;
                a2 += s[6 * g.nnodes] * x0 + s[7 * g.nnodes] * x1 + s[8 * g.nnodes] * x2;
            } else {
                const T *s = stv + (int64_t)((13 - o) * 9) * g.nnodes + J;   // block (J, 26 - o), transposed
                a0 += s[0] * x0 + s[3 * g.nnodes] * x1 + s[6 * g.nnodes] * x2;
                a1 += s[g.nnodes] * x0 + s[4 * g.nnodes] * x1 + s[7 * g.nnodes] * x2;
                a2 += s[2 * g.nnodes] * x0 + s[5 * g.nnodes] * x1 + s[8 * g.nnodes] * x2;
            }
        }
        if (mode == 0) {
            y[3 * I] = a0; y[3 * I + 1] = a1; y[3 * I + 2] = a2;
        } else if (mode == 1) {
            y[3 * I] = b[3 * I] - a0; y[3 * I + 1] = b[3 * I + 1] - a1; y[3 * I + 2] = b[3 * I + 2] - a2;
        } else {
            y[3 * I] = x[3 * I] + invdiag[3 * I] * (b[3 * I] - a0);
            y[3 * I + 1] = x[3 * I + 1] + invdiag[3 * I + 1] * (b[3 * I + 1] - a1);
            y[3 * I + 2] = x[3 * I + 2] + invdiag[3 * I + 2] * (b[3 * I + 2] - a2);
        }
    }
}

// Small levels: one warp per node over the node-major stencil.  Lane o < 27
// applies offset o's 3x3 block (nine contiguous values: the warp reads the
// node's 243 values as one contiguous run), then the warp sums the three
// partial rows.
template <typename T>
__global__ void __launch_bounds__(256)
k_stencil_warp(const T *__restrict__ stv, const T *__restrict__ x, const T *__restrict__ b,
               const T *__restrict__ invdiag, T *__restrict__ y, Grid g, int mode) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t I = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; I < g.nnodes; I += nw) {
        T a0 = 0, a1 = 0, a2 = 0;
        if (lane < 27) {
            int xx, yy, zz;
            node_xyz(I, g.ny, g.nx, xx, yy, zz);
            const int oy = lane % 3 - 1, ox = (lane / 3) % 3 - 1, oz = lane / 9 - 1;
            const int jx = xx + ox, jy = yy + oy, jz = zz + oz;
            if (jx >= 0 && jx < g.nx && jy >= 0 && jy < g.ny && jz >= 0 && jz < g.nz) {
                const int64_t J = I + ((int64_t)oz * g.nx + ox) * g.ny + oy;
                const T x0 = x[3 * J], x1 = x[3 * J + 1], x2 = x[3 * J + 2];
                const T *s = stv + I * STENCIL_VALS + lane * 9;
                a0 = s[0] * x0 + s[1] * x1 + s[2] * x2;
                a1 = s[3] * x0 + s[4] * x1 + s[5] * x2;
                a2 = s[6] * x0 + s[7] * x1 + s[8] * x2;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (lane < 3) {
            const T a = lane == 0 ? a0 : (lane == 1 ? a1 : a2);
            const int64_t d = 3 * I + lane;
            if (mode == 0) y[d] = a;
            else if (mode == 1) y[d] = b[d] - a;
            else y[d] = x[d] + invdiag[d] * (b[d] - a);
        }
    }
}

template <typename T>
void launch_stencil(const T *st_vals, const T *x, const T *b, const T *invdiag, T *y, const Grid &g, int mode,
                    bool node_major, cudaStream_t st) {
    if (node_major) {
        int64_t blocks = (g.nnodes + 7) / 8;   // 8 warps per block
        if (blocks > 65535) blocks = 65535;
        k_stencil_warp<T><<<(unsigned)blocks, 256, 0, st>>>(st_vals, x, b, invdiag, y, g, mode);
    } else {
        k_stencil<T><<<grid_for(g.nnodes, 128), 128, 0, st>>>(st_vals, x, b, invdiag, y, g, mode);
    }
    count_launch();
}
template void launch_stencil<double>(const double *, const double *, const double *, const double *, double *,
                                     const Grid &, int, bool, cudaStream_t);
template void launch_stencil<float>(const float *, const float *, const float *, const float *, float *,
                                    const Grid &, int, bool, cudaStream_t);

// ---------------------------------------------------------------------------
// Elementwise smoother pieces for the matrix-free finest level.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_residual(const T *b, const T *t, T *r, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - t[i];
}
template <typename T>
void launch_residual(const T *b, const T *t, T *r, int64_t n, cudaStream_t st) {
    k_residual<T><<<grid_for(n, 256), 256, 0, st>>>(b, t, r, n); count_launch();
}
template void launch_residual<double>(const double *, const double *, double *, int64_t, cudaStream_t);
template void launch_residual<float>(const float *, const float *, float *, int64_t, cudaStream_t);

// x = x + invD (b - t), or x = invD b for the first sweep from a zero guess
// (b - A*0 = b exactly, so the product is skipped).
template <typename T>
__global__ void k_jacobi(T *x, const T *b, const T *t, const T *invd, int64_t n, int first) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = first ? invd[i] * b[i] : x[i] + invd[i] * (b[i] - t[i]);
}
template <typename T>
void launch_jacobi_update(T *x, const T *b, const T *t, const T *invdiag, int64_t n, int first, cudaStream_t st) {
    k_jacobi<T><<<grid_for(n, 256), 256, 0, st>>>(x, b, t, invdiag, n, first); count_launch();
}
template void launch_jacobi_update<double>(double *, const double *, const double *, const double *, int64_t, int,
                                           cudaStream_t);
template void launch_jacobi_update<float>(float *, const float *, const float *, const float *, int64_t, int,
                                          cudaStream_t);

template <typename T>
__global__ void k_jacobi_out(double *out, const T *x, const T *b, const T *t, const T *invd, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)(x[i] + invd[i] * (b[i] - t[i]));
}
template <typename T>
void launch_jacobi_out(double *out, const T *x, const T *b, const T *t, const T *invdiag, int64_t n, cudaStream_t st) {
    k_jacobi_out<T><<<grid_for(n, 256), 256, 0, st>>>(out, x, b, t, invdiag, n); count_launch();
}
template void launch_jacobi_out<double>(double *, const double *, const double *, const double *, const double *,
                                        int64_t, cudaStream_t);
template void launch_jacobi_out<float>(double *, const float *, const float *, const float *, const float *, int64_t,
                                       cudaStream_t);

template <typename T>
__global__ void k_invert_diag(const T *diag, const uint8_t *fm, T *invd, double omega, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = (double)diag[i];
        invd[i] = (T)((fm[i] && d != 0.0) ? omega / d : 0.0);
    }
}
template <typename T>
void launch_invert_diag(const T *diag, const uint8_t *freemask, T *invdiag, double omega, int64_t n,
                        cudaStream_t st) {
    k_invert_diag<T><<<grid_for(n, 256), 256, 0, st>>>(diag, freemask, invdiag, omega, n); count_launch();
}
template void launch_invert_diag<double>(const double *, const uint8_t *, double *, double, int64_t, cudaStream_t);

// ---------------------------------------------------------------------------
// Trilinear transfers (I/Prolongation.m:24-52 weights 1, 1/2, 1/4, 1/8).
// ---------------------------------------------------------------------------
// All 8 candidate parents are read with clamped indices and the absent ones
// weighted by zero, so the loads issue together (a data-dependent trip count
// serialises them); the sum keeps the order of the parents, so the result is
// the same bit for bit.
template <typename T>
__global__ void k_prolong(const T *__restrict__ xc, T *__restrict__ xf, const uint8_t *__restrict__ fmf, Grid gf,
                          Grid gc, int accumulate) {
    for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < gf.nnodes;
         I += (int64_t)gridDim.x * blockDim.x) {
        int fx, fy, fz;
        node_xyz(I, gf.ny, gf.nx, fx, fy, fz);
        const int x0 = fx >> 1, y0 = fy >> 1, z0 = fz >> 1;
        const T wt = ((fx & 1) ? T(0.5) : T(1)) * ((fy & 1) ? T(0.5) : T(1)) * ((fz & 1) ? T(0.5) : T(1));
        T v0 = 0, v1 = 0, v2 = 0;
#pragma unroll
        for (int kz = 0; kz < 2; ++kz) {
            const bool okz = kz == 0 || (fz & 1);
            const int cz = min(z0 + kz, gc.nz - 1);
#pragma unroll
            for (int kx = 0; kx < 2; ++kx) {
                const bool okx = kx == 0 || (fx & 1);
                const int cx = min(x0 + kx, gc.nx - 1);
#pragma unroll
                for (int ky = 0; ky < 2; ++ky) {
                    const bool oky = ky == 0 || (fy & 1);
                    const int cy = min(y0 + ky, gc.ny - 1);
                    const T w = (okz && okx && oky) ? wt : T(0);
                    const int64_t J = ((int64_t)cz * gc.nx + cx) * gc.ny + cy;
                    v0 += w * xc[3 * J];
                    v1 += w * xc[3 * J + 1];
                    v2 += w * xc[3 * J + 2];
                }
            }
        }
        const T v[3] = {v0, v1, v2};
        for (int c = 0; c < 3; ++c) {
            const int64_t d = 3 * I + c;
            if (accumulate) {
                if (fmf[d]) xf[d] += v[c];
            } else {
                xf[d] = fmf[d] ? v[c] : T(0);
            }
        }
    }
}

template <typename T>
void launch_prolong(const T *xc, T *xf, const uint8_t *freemask_f, const Grid &gf, const Grid &gc, bool accumulate,
                    cudaStream_t st) {
    k_prolong<T><<<grid_for(gf.nnodes, 256), 256, 0, st>>>(xc, xf, freemask_f, gf, gc, accumulate ? 1 : 0); count_launch();
}
template void launch_prolong<double>(const double *, double *, const uint8_t *, const Grid &, const Grid &, bool,
                                     cudaStream_t);
template void launch_prolong<float>(const float *, float *, const uint8_t *, const Grid &, const Grid &, bool,
                                    cudaStream_t);

// RES: restrict rf - tf, the residual b - A x of the finest level.  The 27
// fine neighbours are read with clamped indices, those outside the mesh
// weighted by zero (loads issue together; same sum, same order).
template <typename T, bool RES>
__global__ void k_restrict(const T *__restrict__ rf, const T *__restrict__ tf, T *__restrict__ bc,
                           const uint8_t *__restrict__ fmc, Grid gf, Grid gc, const T *__restrict__ invdc,
                           T *__restrict__ xc) {
    for (int64_t J = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; J < gc.nnodes;
         J += (int64_t)gridDim.x * blockDim.x) {
        int cx, cy, cz;
        node_xyz(J, gc.ny, gc.nx, cx, cy, cz);
        T v0 = 0, v1 = 0, v2 = 0;
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz) {
            const int fz = 2 * cz + dz;
            const bool oz = fz >= 0 && fz < gf.nz;
            const int fzc = min(max(fz, 0), gf.nz - 1);
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const int fx = 2 * cx + dx;
                const bool ox = fx >= 0 && fx < gf.nx;
                const int fxc = min(max(fx, 0), gf.nx - 1);
#pragma unroll
                for (int dy = -1; dy <= 1; ++dy) {
                    const int fy = 2 * cy + dy;
                    const bool oy = fy >= 0 && fy < gf.ny;
                    const int fyc = min(max(fy, 0), gf.ny - 1);
                    const T wt = (oz && ox && oy)
                                     ? (dx ? T(0.5) : T(1)) * (dy ? T(0.5) : T(1)) * (dz ? T(0.5) : T(1))
                                     : T(0);
                    const int64_t I = ((int64_t)fzc * gf.nx + fxc) * gf.ny + fyc;
                    if constexpr (RES) {
                        v0 += wt * (rf[3 * I] - tf[3 * I]);
                        v1 += wt * (rf[3 * I + 1] - tf[3 * I + 1]);
                        v2 += wt * (rf[3 * I + 2] - tf[3 * I + 2]);
                    } else {
                        v0 += wt * rf[3 * I];
                        v1 += wt * rf[3 * I + 1];
                        v2 += wt * rf[3 * I + 2];
                    }
                }
            }
        }
        const T b[3] = {fmc[3 * J] ? v0 : T(0), fmc[3 * J + 1] ? v1 : T(0), fmc[3 * J + 2] ? v2 : T(0)};
        for (int c = 0; c < 3; ++c) {
            bc[3 * J + c] = b[c];
            if (xc) xc[3 * J + c] = invdc[3 * J + c] * b[c];
        }
    }
}

template <typename T>
void launch_restrict(const T *rf, T *bc, const uint8_t *freemask_c, const Grid &gf, const Grid &gc, cudaStream_t st,
                     const T *invd_c, T *xc) {
    k_restrict<T, false><<<grid_for(gc.nnodes, 256), 256, 0, st>>>(rf, nullptr, bc, freemask_c, gf, gc, invd_c, xc);
    count_launch();
}
template <typename T>
void launch_restrict_res(const T *bf, const T *tf, T *bc, const uint8_t *freemask_c, const Grid &gf, const Grid &gc,
                         cudaStream_t st, const T *invd_c, T *xc) {
    k_restrict<T, true><<<grid_for(gc.nnodes, 256), 256, 0, st>>>(bf, tf, bc, freemask_c, gf, gc, invd_c, xc);
    count_launch();
}
template void launch_restrict_res<double>(const double *, const double *, double *, const uint8_t *, const Grid &,
                                          const Grid &, cudaStream_t, const double *, double *);
template void launch_restrict_res<float>(const float *, const float *, float *, const uint8_t *, const Grid &,
                                         const Grid &, cudaStream_t, const float *, float *);
template void launch_restrict<double>(const double *, double *, const uint8_t *, const Grid &, const Grid &,
                                      cudaStream_t, const double *, double *);
template void launch_restrict<float>(const float *, float *, const uint8_t *, const Grid &, const Grid &,
                                     cudaStream_t, const float *, float *);

// Coarse dof is free when the fine dof at the same position is free
// (I/Prolongation.m:38-46,54).
__global__ void k_coarse_mask(const uint8_t *fmf, uint8_t *fmc, Grid gf, Grid gc) {
    for (int64_t J = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; J < gc.nnodes;
         J += (int64_t)gridDim.x * blockDim.x) {
        int cx, cy, cz;
        node_xyz(J, gc.ny, gc.nx, cx, cy, cz);
        const int64_t I = ((int64_t)(2 * cz) * gf.nx + 2 * cx) * gf.ny + 2 * cy;
        for (int c = 0; c < 3; ++c) fmc[3 * J + c] = fmf[3 * I + c];
    }
}

void launch_coarse_freemask(const uint8_t *freemask_f, uint8_t *freemask_c, const Grid &gf, const Grid &gc,
                            cudaStream_t st) {
    k_coarse_mask<<<grid_for(gc.nnodes, 256), 256, 0, st>>>(freemask_f, freemask_c, gf, gc); count_launch();
}

}  // namespace tosp
