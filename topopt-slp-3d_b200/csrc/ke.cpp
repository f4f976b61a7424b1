// Host-side constant tables: sub-element stiffness blocks and filter taps.
#include <cmath>

#include "tosp_internal.h"

namespace tosp {

// Stiffness integrand of each of the n^3 density sub-cubes of a hex8 element
// (I/ElemStiffMatrixGQMR.m:10-240 with elem.deg = 1): 2-point Gauss rule per
// sub-cube, B'DB accumulated, scaled by ct*a*b*c and symmetrised.  Sub-cube
// order y fastest, then x, then z; local node order (x0y0z0, x0y1z0, x1y0z0,
// x1y1z0, then z1); local dof = 3*node + component.
void elem_stiff_mr(double el, double eh, double ew, double nu, int n, std::vector<double> &ks) {
    const double a = el / 2, b = eh / 2, c = ew / 2;
    const double v = nu;
    const double d0 = 1.0 / ((1 + v) * (1 - 2 * v));
    double D[6][6] = {{0}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[i][j] = d0 * (i == j ? 1 - v : v);
    for (int i = 3; i < 6; ++i) D[i][i] = d0 * (1 - 2 * v) / 2;
    const int sx[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const int sy[8] = {-1, 1, -1, 1, -1, 1, -1, 1};
    const int sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    const double gp[2] = {-1.0 / std::sqrt(3.0), 1.0 / std::sqrt(3.0)};
    const int ns = n * n * n;
    ks.assign((size_t)ns * 576, 0.0);
    int ind = 0;
    for (int elz = 0; elz < n; ++elz)
        for (int elx = 0; elx < n; ++elx)
            for (int ely = 0; ely < n; ++ely) {
                double k2[24][24] = {{0}};
                const double cxm = -1.0 + (2.0 * elx + 1) / n, cym = -1.0 + (2.0 * ely + 1) / n,
                             czm = -1.0 + (2.0 * elz + 1) / n;
                const double minx = cxm - 1.0 / n, maxx = cxm + 1.0 / n;
                const double miny = cym - 1.0 / n, maxy = cym + 1.0 / n;
                const double minz = czm - 1.0 / n, maxz = czm + 1.0 / n;
                const double ct = ((maxx - minx) / 2) * ((maxy - miny) / 2) * ((maxz - minz) / 2);
                for (int g3 = 0; g3 < 2; ++g3)
                    for (int g1 = 0; g1 < 2; ++g1)
                        for (int g2 = 0; g2 < 2; ++g2) {
                            const double x1 = ((maxx - minx) / 2) * gp[g1] + (maxx + minx) / 2;
                            const double x2 = ((maxy - miny) / 2) * gp[g2] + (maxy + miny) / 2;
                            const double x3 = ((maxz - minz) / 2) * gp[g3] + (maxz + minz) / 2;
                            double dx[8], dy[8], dz[8];
                            for (int q = 0; q < 8; ++q) {
                                dx[q] = (1 / (8 * a)) * sx[q] * (1 + sy[q] * x2) * (1 + sz[q] * x3);
                                dy[q] = (1 / (8 * b)) * sy[q] * (1 + sx[q] * x1) * (1 + sz[q] * x3);
                                dz[q] = (1 / (8 * c)) * sz[q] * (1 + sx[q] * x1) * (1 + sy[q] * x2);
                            }
                            double B[6][24] = {{0}};
                            for (int q = 0; q < 8; ++q) {
                                B[0][3 * q] = dx[q];
                                B[1][3 * q + 1] = dy[q];
                                B[2][3 * q + 2] = dz[q];
                                B[3][3 * q] = dy[q];
                                B[3][3 * q + 1] = dx[q];
                                B[4][3 * q + 1] = dz[q];
                                B[4][3 * q + 2] = dy[q];
                                B[5][3 * q] = dz[q];
                                B[5][3 * q + 2] = dx[q];
                            }
                            double DB[6][24];
                            for (int i = 0; i < 6; ++i)
                                for (int j = 0; j < 24; ++j) {
                                    double s = 0;
                                    for (int k = 0; k < 6; ++k) s += D[i][k] * B[k][j];
                                    DB[i][j] = s;
                                }
                            for (int i = 0; i < 24; ++i)
                                for (int j = 0; j < 24; ++j) {
                                    double s = 0;
                                    for (int k = 0; k < 6; ++k) s += B[k][i] * DB[k][j];
                                    k2[i][j] += s;   // Gauss weights are 1
                                }
                        }
                double *out = &ks[(size_t)ind * 576];
                for (int i = 0; i < 24; ++i)
                    for (int j = 0; j < 24; ++j) {
                        const double kij = ct * (a * b * c) * k2[i][j];
                        const double kji = ct * (a * b * c) * k2[j][i];
                        out[i * 24 + j] = (kij + kji) / 2;
                    }
                ++ind;
            }
}

void pack_upper(const std::vector<double> &ks, int ns, std::vector<double> &packed) {
    packed.assign((size_t)ns * KE_PACK, 0.0);
    for (int s = 0; s < ns; ++s) {
        int t = 0;
        for (int i = 0; i < 24; ++i)
            for (int j = i; j < 24; ++j) packed[(size_t)s * KE_PACK + t++] = ks[(size_t)s * 576 + i * 24 + j];
    }
}

// Galerkin sub-cell table for the finest coarsening: for child c of a coarse
// element and sub-cube s of that child, S_(c,s) = Pi_c' KE_s Pi_c, where Pi_c
// interpolates the coarse element's 8 nodes to the child's 8 nodes with the
// trilinear weights of I/Prolongation.m:24-52.  Stored packed upper
// (row-major, i <= j), q = c * n^3 + s.
void coarse_fine_table(const std::vector<double> &ks, int n, std::vector<double> &S) {
    const int ns = n * n * n;
    auto phi1 = [](int f, int A) {
        const int d = f - 2 * A;
        return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0);
    };
    S.assign((size_t)8 * ns * KE_PACK, 0.0);
    for (int c = 0; c < 8; ++c) {
        double W[8][8];
        const int cdx = (c >> 1) & 1, cdy = c & 1, cdz = (c >> 2) & 1;
        for (int a = 0; a < 8; ++a)
            for (int A = 0; A < 8; ++A)
                W[a][A] = phi1(cdx + ((a >> 1) & 1), (A >> 1) & 1) * phi1(cdy + (a & 1), A & 1) *
                          phi1(cdz + ((a >> 2) & 1), (A >> 2) & 1);
        for (int s = 0; s < ns; ++s) {
            const double *K = &ks[(size_t)s * 576];
            double T[24][24];   // K Pi_c
            for (int i = 0; i < 24; ++i)
                for (int J = 0; J < 24; ++J) {
                    const int B = J / 3, cb = J % 3;
                    double v = 0.0;
                    for (int b = 0; b < 8; ++b) v += K[i * 24 + b * 3 + cb] * W[b][B];
                    T[i][J] = v;
                }
            double *out = &S[((size_t)c * ns + s) * KE_PACK];
            int t = 0;
            for (int I = 0; I < 24; ++I)
                for (int J = I; J < 24; ++J) {
                    const int A = I / 3, ca = I % 3;
                    double v = 0.0;
                    for (int a = 0; a < 8; ++a) v += W[a][A] * T[a * 3 + ca][J];
                    out[t++] = v;
                }
        }
    }
}

// Filter neighbourhood of I/ElemNeighborhood.m:93-122.  For each z-offset
// kz <= floor(rmin/ew): x-reach floor(sqrt(rmin^2-dz^2)/el); for each x-offset:
// y-reach floor(sqrt(rmin^2-dz^2-dx^2)/eh).  Gaussian (opfilter 1) or hat
// (opfilter 2) weight; the centre tap is beta (resp. 1) as at :143-147.
void filter_taps(double rmin, double el, double eh, double ew, int opfilter, std::vector<FilterTap> &taps) {
    taps.clear();
    const int frz = (int)std::floor(rmin / ew);
    const double rmin2 = rmin * rmin;
    double alpha = 0, beta = 1;
    if (opfilter == 1) {
        alpha = 1 / (2 * ((rmin / 3) * (rmin / 3)));
        beta = 1 / (2 * M_PI * (rmin / 3));
    }
    for (int kz = 0; kz <= frz; ++kz) {
        const double dz2 = (kz * ew) * (kz * ew);
        const int dxm = (int)std::floor(std::sqrt(rmin2 - dz2) / el);
        for (int ix = 0; ix <= dxm; ++ix) {
            const double dx2 = (ix * el) * (ix * el);
            const int dym = (int)std::floor(std::sqrt(rmin2 - dz2 - dx2) / eh);
            for (int jy = 0; jy <= dym; ++jy) {
                const double dy2 = (jy * eh) * (jy * eh);
                double wt;
                if (opfilter == 1) wt = std::exp(-(dz2 + dx2 + dy2) * alpha) * beta;
                else wt = (rmin - std::sqrt(dz2 + dx2 + dy2)) / rmin;
                if (kz == 0 && ix == 0 && jy == 0) wt = (opfilter == 1) ? beta : 1.0;
                for (int szs = 0; szs < (kz ? 2 : 1); ++szs)
                    for (int sxs = 0; sxs < (ix ? 2 : 1); ++sxs)
                        for (int sys = 0; sys < (jy ? 2 : 1); ++sys)
                            taps.push_back({sxs ? -ix : ix, sys ? -jy : jy, szs ? -kz : kz, wt});
            }
        }
    }
}

}  // namespace tosp
