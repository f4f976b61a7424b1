// Density filter (I/ApplyFilter.m:74-81 with W of I/ElemNeighborhood.m):
//   trans = 0:  y = (W x) ./ w        trans = 1:  y = W' (x ./ w) = W (x ./ w)
// W is symmetric with Gaussian/hat weights inside the radius; rows and
// columns of fixed elements are decoupled with a unit diagonal
// (I/ElemNeighborhood.m:173-179).  One thread per density element walks the
// tap list; neighbour values come through L1/L2.
#include "tosp_internal.h"

namespace tosp {

__global__ void k_filter(const double *__restrict__ x, double *__restrict__ y, const double *__restrict__ wsum,
                         const uint8_t *__restrict__ fixed, const FilterTap *__restrict__ taps, int ntaps, int nelx,
                         int nely, int nelz, int trans, int weights_only) {
    const int64_t n = (int64_t)nelx * nely * nelz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int ey = (int)(i % nely), ex = (int)((i / nely) % nelx), ez = (int)(i / ((int64_t)nely * nelx));
        if (fixed && fixed[i]) {
            y[i] = weights_only ? 1.0 : (trans ? x[i] / wsum[i] : x[i]);
            continue;
        }
        double acc = 0.0;
        for (int t = 0; t < ntaps; ++t) {
            const FilterTap tp = taps[t];
            const int jx = ex + tp.dx, jy = ey + tp.dy, jz = ez + tp.dz;
            if (jx < 0 || jx >= nelx || jy < 0 || jy >= nely || jz < 0 || jz >= nelz) continue;
            const int64_t j = ((int64_t)jz * nelx + jx) * nely + jy;
            if (fixed && fixed[j]) continue;
            if (weights_only) acc += tp.w;
            else if (trans) acc += tp.w * (x[j] / wsum[j]);
            else acc += tp.w * x[j];
        }
        y[i] = (weights_only || trans) ? acc : acc / wsum[i];
    }
}

void launch_filter(const double *x, double *y, const double *wsum, const uint8_t *fixed, const FilterTap *taps_dev,
                   int ntaps, int nelx, int nely, int nelz, int trans, int weights_only, cudaStream_t st) {
    const int64_t n = (int64_t)nelx * nely * nelz;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 16384) blocks = 16384;
    if (blocks < 1) blocks = 1;
    k_filter<<<(unsigned)blocks, 256, 0, st>>>(x, y, wsum, fixed, taps_dev, ntaps, nelx, nely, nelz, trans,
                                               weights_only); count_launch();
}

}  // namespace tosp
