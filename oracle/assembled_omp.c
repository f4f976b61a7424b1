/*
 * Oracle (TEST INFRASTRUCTURE ONLY): C/OpenMP restatement of the reference's
 * default, assembled solve path (genK = true), used as the timed CPU baseline
 * of the benchmark.  Nothing in the product links or calls this file.
 *
 *   stencil_assemble - I/GlobalStiffMatrix.m:16-65 (K = sum over elements of
 *                      sum_s kv_s (emin + (E-emin) rho_s^p), restricted to the
 *                      free dofs) and the coarse matrices P'AP of
 *                      I/SetupGMG.m:45-49 assembled from Galerkin element
 *                      matrices (kelem_omp.c).  The matrices are kept as node
 *                      stencils: for every node the 27 neighbour blocks of
 *                      3x3 entries (the non-zeros of MATLAB's sparse K), with
 *                      the rows and columns of fixed dofs zero.
 *   stencil_apply    - A*x (I/SolveMG.m:31,41; I/VCycle.m:25), b - A*x, and the
 *                      damped Jacobi sweep x + M\(b - A*x) with
 *                      M = diag(A)/omega (I/Smooth.m:14-17, I/SetupGMG.m:70).
 *   vec_*            - the PCG vector updates of I/SolveMG.m:36-49.
 *   filter_taps_apply - I/ApplyFilter.m:74-81 with the weights of
 *                      I/ElemNeighborhood.m:93-181 given as offset taps.
 *
 * Numbering follows the reference: node = (z*nx + x)*ny + y, dof = 3*node+c.
 * Stencil layout: st[node*243 + o*9 + ci*3 + cj] = A(3*node+ci, 3*nbr+cj)
 * with o = ((dz+1)*3 + (dx+1))*3 + (dy+1), nbr = node + (dz, dx, dy).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <omp.h>

static inline int64_t node_of(int x, int y, int z, int nx, int ny) { return ((int64_t)z * nx + x) * ny + y; }

static inline int64_t dens_index(int ex, int ey, int ez, int s, int n, int nelx_d, int nely_d) {
    const int sy = s % n, sx = (s / n) % n, sz = s / (n * n);
    return ((int64_t)(ez * n + sz) * nelx_d + (ex * n + sx)) * nely_d + (ey * n + sy);
}

/* Node stencils of sum_e K_e with masked rows/columns.  K_e is either
 * sum_s w_s ks_s (ks != NULL: finest level) or Ae[e] (coarse levels). */
void stencil_assemble(int nelx, int nely, int nelz, int n, const double *ks, const double *w, const double *Ae,
                      const unsigned char *fm, double *st, int nthreads) {
    const int nx = nelx + 1, ny = nely + 1, nz = nelz + 1, ns = n * n * n;
    const int nelx_d = nelx * n, nely_d = nely * n;
    const int64_t nnodes = (int64_t)nx * ny * nz;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nnodes * 243; ++i) st[i] = 0.0;
    /* 8 parity colours: elements of one colour share no node */
    for (int col = 0; col < 8; ++col) {
        const int cx = (col >> 1) & 1, cy = col & 1, cz = (col >> 2) & 1;
        const int mx = (nelx - cx + 1) / 2, my = (nely - cy + 1) / 2, mz = (nelz - cz + 1) / 2;
        const int64_t m = (int64_t)mx * my * mz;
#pragma omp parallel for schedule(static)
        for (int64_t t = 0; t < m; ++t) {
            const int ey = cy + 2 * (int)(t % my), ex = cx + 2 * (int)((t / my) % mx);
            const int ez = cz + 2 * (int)(t / ((int64_t)my * mx));
            double K[576];
            if (ks) {
                for (int i = 0; i < 576; ++i) K[i] = 0.0;
                for (int s = 0; s < ns; ++s) {
                    const double ws = w[dens_index(ex, ey, ez, s, n, nelx_d, nely_d)];
                    const double *k = ks + (int64_t)s * 576;
                    for (int i = 0; i < 576; ++i) K[i] += k[i] * ws;
                }
            } else {
                memcpy(K, Ae + (((int64_t)ez * nelx + ex) * nely + ey) * 576, sizeof(K));
            }
            for (int a = 0; a < 8; ++a) {
                const int ax = (a >> 1) & 1, ay = a & 1, az = (a >> 2) & 1;
                const int64_t na = node_of(ex + ax, ey + ay, ez + az, nx, ny);
                for (int b = 0; b < 8; ++b) {
                    const int bx = (b >> 1) & 1, by = b & 1, bz = (b >> 2) & 1;
                    const int64_t nb = node_of(ex + bx, ey + by, ez + bz, nx, ny);
                    const int o = ((bz - az + 1) * 3 + (bx - ax + 1)) * 3 + (by - ay + 1);
                    double *blk = st + na * 243 + o * 9;
                    for (int ci = 0; ci < 3; ++ci) {
                        if (!fm[3 * na + ci]) continue;
                        for (int cj = 0; cj < 3; ++cj)
                            if (fm[3 * nb + cj]) blk[ci * 3 + cj] += K[(3 * a + ci) * 24 + 3 * b + cj];
                    }
                }
            }
        }
    }
}

/* mode 0: y = A x; 1: y = b - A x; 2: y = x + minv .* (b - A x). */
void stencil_apply(int nelx, int nely, int nelz, const double *st, const double *x, const double *b,
                   const double *minv, double *y, int mode, int nthreads) {
    const int nx = nelx + 1, ny = nely + 1, nz = nelz + 1;
    const int64_t nnodes = (int64_t)nx * ny * nz;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t I = 0; I < nnodes; ++I) {
        const int iy = (int)(I % ny), ix = (int)((I / ny) % nx), iz = (int)(I / ((int64_t)ny * nx));
        const double *s = st + I * 243;
        double v0 = 0.0, v1 = 0.0, v2 = 0.0;
        for (int dz = -1; dz <= 1; ++dz) {
            const int jz = iz + dz;
            if (jz < 0 || jz >= nz) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int jx = ix + dx;
                if (jx < 0 || jx >= nx) continue;
                for (int dy = -1; dy <= 1; ++dy) {
                    const int jy = iy + dy;
                    if (jy < 0 || jy >= ny) continue;
                    const int o = ((dz + 1) * 3 + (dx + 1)) * 3 + (dy + 1);
                    const double *blk = s + o * 9;
                    const double *xj = x + 3 * node_of(jx, jy, jz, nx, ny);
                    v0 += blk[0] * xj[0] + blk[1] * xj[1] + blk[2] * xj[2];
                    v1 += blk[3] * xj[0] + blk[4] * xj[1] + blk[5] * xj[2];
                    v2 += blk[6] * xj[0] + blk[7] * xj[1] + blk[8] * xj[2];
                }
            }
        }
        const double v[3] = {v0, v1, v2};
        for (int c = 0; c < 3; ++c) {
            const int64_t d = 3 * I + c;
            if (mode == 0) y[d] = v[c];
            else if (mode == 1) y[d] = b[d] - v[c];
            else y[d] = x[d] + minv[d] * (b[d] - v[c]);
        }
    }
}

/* minv = omega / diag(A) on free dofs, 0 on fixed dofs. */
void stencil_minv(int nelx, int nely, int nelz, const double *st, const unsigned char *fm, double omega,
                  double *minv) {
    const int64_t nnodes = (int64_t)(nelx + 1) * (nely + 1) * (nelz + 1);
    for (int64_t I = 0; I < nnodes; ++I)
        for (int c = 0; c < 3; ++c) {
            const double dg = st[I * 243 + 13 * 9 + c * 3 + c];
            minv[3 * I + c] = (fm[3 * I + c] && dg != 0.0) ? omega / dg : 0.0;
        }
}

/* y = alpha x + beta y */
void vec_axpby(int64_t n, double alpha, const double *x, double beta, double *y, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) y[i] = alpha * x[i] + beta * y[i];
}

double vec_dot(int64_t n, const double *a, const double *b, int nthreads) {
    double s = 0.0;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* y = minv .* b (the first Jacobi sweep from x = 0). */
void vec_mul(int64_t n, const double *a, const double *b, double *y, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) y[i] = a[i] * b[i];
}

/* ApplyFilter with taps (dx, dy, dz, weight) on an nelx x nely x nelz
 * density mesh; fixed elements are decoupled with a unit diagonal.
 * x == NULL: y = W 1 (the row sums w).  trans 0: y = (W x)./w;
 * trans 1: y = W (x./w) (W is symmetric). */
void filter_taps_apply(int nelx, int nely, int nelz, int ntaps, const int *off, const double *tw,
                       const unsigned char *fixed, const double *wsum, const double *x, double *y, int trans,
                       int nthreads) {
    const int64_t ne = (int64_t)nelx * nely * nelz;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < ne; ++e) {
        const int ey = (int)(e % nely), ex = (int)((e / nely) % nelx), ez = (int)(e / ((int64_t)nely * nelx));
        if (fixed && fixed[e]) {
            y[e] = x ? x[e] / wsum[e] : 1.0;   /* unit row and column, w = 1 */
            continue;
        }
        double v = 0.0;
        for (int t = 0; t < ntaps; ++t) {
            const int jx = ex + off[3 * t], jy = ey + off[3 * t + 1], jz = ez + off[3 * t + 2];
            if (jx < 0 || jx >= nelx || jy < 0 || jy >= nely || jz < 0 || jz >= nelz) continue;
            const int64_t j = ((int64_t)jz * nelx + jx) * nely + jy;
            if (fixed && fixed[j]) continue;
            const double xj = x ? (trans ? x[j] / wsum[j] : x[j]) : 1.0;
            v += tw[t] * xj;
        }
        y[e] = (x && !trans) ? v / wsum[e] : v;
    }
}
