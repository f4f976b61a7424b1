/*
 * Oracle (TEST INFRASTRUCTURE ONLY): C/OpenMP restatement of the reference's
 * matrix-free solve path, used as the timed CPU baseline and as a second
 * oracle.  Nothing in the product links or calls this file.
 *
 *   kelem_prod_full  - I/WOK/KelemProd.m:57-100: per element
 *                      kel = kv * (emin + (E-emin) rho^p) (here: the SIMP
 *                      factors w are precomputed), y(dofs) += kel * x(dofs).
 *                      Elements are processed in 8 parity colours so that
 *                      threads never update the same node concurrently.
 *   prolong_full / restrict_full - I/Prolongation.m:15-55 trilinear stencil
 *                      applied on full-length vectors with free-dof masks.
 *   galerkin_*       - coarse element matrices whose sum is P'AP (the matrix
 *                      of I/SetupGMG.m:45-49 / I/WOK/GlobalStiffMatrixWOK.m).
 *   dense_assemble   - coarsest matrix with fixed dofs decoupled.
 *   grad_full        - I/Grad.m:24-49 quadratic forms.
 *
 * Numbering follows the reference: node = (z*nx + x)*ny + y, dof = 3*node+c,
 * element order y fastest, then x, then z; sub-elements likewise.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <omp.h>

static inline int64_t node_of(int x, int y, int z, int nx, int ny) { return ((int64_t)z * nx + x) * ny + y; }

static void elem_dofs(int ex, int ey, int ez, int nx, int ny, int64_t *d) {
    for (int a = 0; a < 8; ++a) {
        const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
        const int64_t nd = node_of(ex + dx, ey + dy, ez + dz, nx, ny);
        for (int c = 0; c < 3; ++c) d[3 * a + c] = 3 * nd + c;
    }
}

static inline int64_t dens_index(int ex, int ey, int ez, int s, int n, int nelx_d, int nely_d) {
    const int sy = s % n, sx = (s / n) % n, sz = s / (n * n);
    return ((int64_t)(ez * n + sz) * nelx_d + (ex * n + sx)) * nely_d + (ey * n + sy);
}

/* y += K(w) x over all elements; ks: ns blocks of 24x24 row-major. */
void kelem_prod_full(int nelx, int nely, int nelz, int n, const double *ks, const double *w, const double *x,
                     double *y, int nthreads) {
    const int nx = nelx + 1, ny = nely + 1, ns = n * n * n;
    const int nelx_d = nelx * n, nely_d = nely * n;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    for (int col = 0; col < 8; ++col) {
        const int cx = (col >> 1) & 1, cy = col & 1, cz = (col >> 2) & 1;
        const int mx = (nelx - cx + 1) / 2, my = (nely - cy + 1) / 2, mz = (nelz - cz + 1) / 2;
        const int64_t m = (int64_t)mx * my * mz;
#pragma omp parallel for schedule(static)
        for (int64_t t = 0; t < m; ++t) {
            const int ey = cy + 2 * (int)(t % my), ex = cx + 2 * (int)((t / my) % mx), ez = cz + 2 * (int)(t / ((int64_t)my * mx));
            int64_t d[24];
            elem_dofs(ex, ey, ez, nx, ny, d);
            double kel[576];
            for (int i = 0; i < 576; ++i) kel[i] = 0.0;
            for (int s = 0; s < ns; ++s) {
                const double ws = w[dens_index(ex, ey, ez, s, n, nelx_d, nely_d)];
                const double *k = ks + (int64_t)s * 576;
                for (int i = 0; i < 576; ++i) kel[i] += k[i] * ws;
            }
            double xe[24];
            for (int j = 0; j < 24; ++j) xe[j] = x[d[j]];
            for (int i = 0; i < 24; ++i) {
                double v = 0.0;
                for (int j = 0; j < 24; ++j) v += kel[i * 24 + j] * xe[j];
                y[d[i]] += v;
            }
        }
    }
}

void prolong_full(int nelxc, int nelyc, int nelzc, const double *xc, double *xf, const unsigned char *fmf,
                  int accumulate, int nthreads) {
    const int nxc = nelxc + 1, nyc = nelyc + 1;
    const int nxf = 2 * nelxc + 1, nyf = 2 * nelyc + 1, nzf = 2 * nelzc + 1;
    const int64_t nnf = (int64_t)nxf * nyf * nzf;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t I = 0; I < nnf; ++I) {
        const int fy = (int)(I % nyf), fx = (int)((I / nyf) % nxf), fz = (int)(I / ((int64_t)nyf * nxf));
        double v[3] = {0, 0, 0};
        const int x0 = fx >> 1, y0 = fy >> 1, z0 = fz >> 1;
        for (int kz = 0; kz < ((fz & 1) ? 2 : 1); ++kz)
            for (int kx = 0; kx < ((fx & 1) ? 2 : 1); ++kx)
                for (int ky = 0; ky < ((fy & 1) ? 2 : 1); ++ky) {
                    const double wt = ((fx & 1) ? 0.5 : 1.0) * ((fy & 1) ? 0.5 : 1.0) * ((fz & 1) ? 0.5 : 1.0);
                    const int64_t J = node_of(x0 + kx, y0 + ky, z0 + kz, nxc, nyc);
                    for (int c = 0; c < 3; ++c) v[c] += wt * xc[3 * J + c];
                }
        for (int c = 0; c < 3; ++c) {
            const int64_t d = 3 * I + c;
            if (accumulate) {
                if (fmf[d]) xf[d] += v[c];
            } else {
                xf[d] = fmf[d] ? v[c] : 0.0;
            }
        }
    }
}

void restrict_full(int nelxc, int nelyc, int nelzc, const double *rf, double *bc, const unsigned char *fmc,
                   int nthreads) {
    const int nxc = nelxc + 1, nyc = nelyc + 1, nzc = nelzc + 1;
    const int nxf = 2 * nelxc + 1, nyf = 2 * nelyc + 1, nzf = 2 * nelzc + 1;
    const int64_t nnc = (int64_t)nxc * nyc * nzc;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t J = 0; J < nnc; ++J) {
        const int cy = (int)(J % nyc), cx = (int)((J / nyc) % nxc), cz = (int)(J / ((int64_t)nyc * nxc));
        double v[3] = {0, 0, 0};
        for (int dz = -1; dz <= 1; ++dz) {
            const int fz = 2 * cz + dz;
            if (fz < 0 || fz >= nzf) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int fx = 2 * cx + dx;
                if (fx < 0 || fx >= nxf) continue;
                for (int dy = -1; dy <= 1; ++dy) {
                    const int fy = 2 * cy + dy;
                    if (fy < 0 || fy >= nyf) continue;
                    const double wt = (dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0);
                    const int64_t I = node_of(fx, fy, fz, nxf, nyf);
                    for (int c = 0; c < 3; ++c) v[c] += wt * rf[3 * I + c];
                }
            }
        }
        for (int c = 0; c < 3; ++c) bc[3 * J + c] = fmc[3 * J + c] ? v[c] : 0.0;
    }
}

static inline double phi1(int f, int A) {
    const int d = f - 2 * A;
    return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0);
}

/* Triple product Abar += (W'(x)I) K (W(x)I) for child c of a coarse element. */
static void add_child(const double *K, int c, double *Abar) {
    double W[8][8], T[576];
    const int cdx = (c >> 1) & 1, cdy = c & 1, cdz = (c >> 2) & 1;
    for (int a = 0; a < 8; ++a)
        for (int A = 0; A < 8; ++A)
            W[a][A] = phi1(cdx + ((a >> 1) & 1), (A >> 1) & 1) * phi1(cdy + (a & 1), A & 1) *
                      phi1(cdz + ((a >> 2) & 1), (A >> 2) & 1);
    for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) {
            const int B = j / 3, cb = j % 3;
            double v = 0;
            for (int b = 0; b < 8; ++b) v += K[i * 24 + b * 3 + cb] * W[b][B];
            T[i * 24 + j] = v;
        }
    for (int i = 0; i < 24; ++i) {
        const int A = i / 3, ca = i % 3;
        for (int j = 0; j < 24; ++j) {
            double v = 0;
            for (int a = 0; a < 8; ++a) v += W[a][A] * T[(a * 3 + ca) * 24 + j];
            Abar[i * 24 + j] += v;
        }
    }
}

static void gal(int nelxf, int nelyf, int nelzf, int n, const double *ks, const double *w, const double *Af,
                const unsigned char *fmf, double *Ac, int nthreads) {
    const int nelxc = nelxf / 2, nelyc = nelyf / 2, nelzc = nelzf / 2;
    const int nxf = nelxf + 1, nyf = nelyf + 1, ns = n * n * n;
    const int64_t nec = (int64_t)nelxc * nelyc * nelzc;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t E = 0; E < nec; ++E) {
        const int cy = (int)(E % nelyc), cx = (int)((E / nelyc) % nelxc), cz = (int)(E / ((int64_t)nelyc * nelxc));
        double *Ab = Ac + E * 576;
        memset(Ab, 0, sizeof(double) * 576);
        for (int c = 0; c < 8; ++c) {
            const int fx = 2 * cx + ((c >> 1) & 1), fy = 2 * cy + (c & 1), fz = 2 * cz + ((c >> 2) & 1);
            int64_t d[24];
            elem_dofs(fx, fy, fz, nxf, nyf, d);
            double K[576];
            if (ks) {
                memset(K, 0, sizeof(K));
                for (int s = 0; s < ns; ++s) {
                    const double ws = w[dens_index(fx, fy, fz, s, n, nelxf * n, nelyf * n)];
                    for (int i = 0; i < 576; ++i) K[i] += ks[(int64_t)s * 576 + i] * ws;
                }
            } else {
                memcpy(K, Af + (((int64_t)fz * nelxf + fx) * nelyf + fy) * 576, sizeof(K));
            }
            for (int i = 0; i < 24; ++i)
                for (int j = 0; j < 24; ++j)
                    if (!fmf[d[i]] || !fmf[d[j]]) K[i * 24 + j] = 0.0;
            add_child(K, c, Ab);
        }
    }
}

void galerkin_fine(int nelx, int nely, int nelz, int n, const double *ks, const double *w, const unsigned char *fmf,
                   double *Ac, int nthreads) {
    gal(nelx, nely, nelz, n, ks, w, 0, fmf, Ac, nthreads);
}

void galerkin_coarse(int nelxf, int nelyf, int nelzf, const double *Af, const unsigned char *fmf, double *Ac,
                     int nthreads) {
    gal(nelxf, nelyf, nelzf, 1, 0, 0, Af, fmf, Ac, nthreads);
}

/* Dense coarsest matrix (ndof x ndof, row-major) with fixed dofs decoupled. */
void dense_assemble(int nelx, int nely, int nelz, const double *Ae, const unsigned char *fm, double *A) {
    const int nx = nelx + 1, ny = nely + 1, nz = nelz + 1;
    const int64_t nd = 3LL * nx * ny * nz;
    memset(A, 0, sizeof(double) * nd * nd);
    for (int64_t E = 0; E < (int64_t)nelx * nely * nelz; ++E) {
        const int ey = (int)(E % nely), ex = (int)((E / nely) % nelx), ez = (int)(E / ((int64_t)nely * nelx));
        int64_t d[24];
        elem_dofs(ex, ey, ez, nx, ny, d);
        for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j)
                if (fm[d[i]] && fm[d[j]]) A[d[i] * nd + d[j]] += Ae[E * 576 + i * 24 + j];
    }
    for (int64_t i = 0; i < nd; ++i)
        if (!fm[i]) A[i * nd + i] = 1.0;
}

/* Unfiltered sensitivities of I/Grad.m:24-49 (free_elem may be NULL = all). */
void grad_full(int nelx, int nely, int nelz, int n, const double *ks, const double *u, const double *rho,
               const unsigned char *free_elem, double p, double emin, double E, double *g0, int nthreads) {
    const int nx = nelx + 1, ny = nely + 1, ns = n * n * n;
    const int64_t ne = (int64_t)nelx * nely * nelz;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < ne; ++e) {
        const int ey = (int)(e % nely), ex = (int)((e / nely) % nelx), ez = (int)(e / ((int64_t)nely * nelx));
        int64_t d[24];
        elem_dofs(ex, ey, ez, nx, ny, d);
        double ue[24];
        for (int j = 0; j < 24; ++j) ue[j] = u[d[j]];
        for (int s = 0; s < ns; ++s) {
            const int64_t di = dens_index(ex, ey, ez, s, n, nelx * n, nely * n);
            if (free_elem && !free_elem[e]) {
                g0[di] = 0.0;
                continue;
            }
            const double *k = ks + (int64_t)s * 576;
            double q = 0.0;
            for (int i = 0; i < 24; ++i) {
                double v = 0.0;
                for (int j = 0; j < 24; ++j) v += k[i * 24 + j] * ue[j];
                q += ue[i] * v;
            }
            g0[di] = -p * pow(rho[di], p - 1) * (E - emin) * q;
        }
    }
}
