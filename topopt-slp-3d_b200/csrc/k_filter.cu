// Density filter (I/ApplyFilter.m:74-81 with W of I/ElemNeighborhood.m):
//   trans = 0:  y = (W x) ./ w        trans = 1:  y = W' (x ./ w) = W (x ./ w)
// W is symmetric with Gaussian/hat weights inside the radius; rows and
// columns of fixed elements are decoupled with a unit diagonal
// (I/ElemNeighborhood.m:173-179).
//
// k_filter_tiled: a CTA loads a 32 x 8 x 4 brick of the filter's inputs with
// its halo (the taps' radius) into shared memory once (v_j = x_j, x_j / w_j
// or 1, and 0 for fixed or absent neighbours) and each thread walks the tap
// list (weights and tile offsets in shared memory) over the tile for four
// outputs along z at once: every input is read from global memory about once
// per tile instead of once per tap, no branch separates the taps' loads, and
// each tap's weight and offset serve four independent sums.  The taps are summed in the same order as the
// per-element kernel, absent ones adding zero, so the results are the same.
// k_filter (one thread per element walking the tap list through L1/L2)
// serves radii whose tile would not fit in shared memory.
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

constexpr int FT_Y = 32, FT_X = 8, FT_Z = 4;   // outputs per CTA (256 threads, four along z each)

__global__ void __launch_bounds__(256)
k_filter_tiled(const double *__restrict__ x, double *__restrict__ y, const double *__restrict__ wsum,
               const uint8_t *__restrict__ fixed, const FilterTap *__restrict__ taps, int ntaps, int nelx, int nely,
               int nelz, int trans, int weights_only, int R) {
    extern __shared__ __align__(16) unsigned char ft_smem[];
    double *sw = reinterpret_cast<double *>(ft_smem);                 // tap weights
    double *tile = sw + ntaps;
    int *soff = reinterpret_cast<int *>(tile + (FT_Y + 2 * R) * (FT_X + 2 * R) * (FT_Z + 2 * R));   // tap offsets in the tile
    const int TY = FT_Y + 2 * R, TX = FT_X + 2 * R, TZ = FT_Z + 2 * R, TXY = TX * TY;
    const int y0 = blockIdx.x * FT_Y, x0 = blockIdx.y * FT_X, z0 = blockIdx.z * FT_Z;
    const int tid = threadIdx.x;
    for (int t = tid; t < ntaps; t += blockDim.x) {
        const FilterTap tp = taps[t];
        sw[t] = tp.w;
        soff[t] = tp.dz * TXY + tp.dx * TY + tp.dy;
    }
    for (int idx = tid; idx < TY * TX * TZ; idx += blockDim.x) {
        const int ty = idx % TY, tx = (idx / TY) % TX, tz = idx / TXY;
        const int gy = y0 - R + ty, gx = x0 - R + tx, gz = z0 - R + tz;
        double v = 0.0;
        if (gy >= 0 && gy < nely && gx >= 0 && gx < nelx && gz >= 0 && gz < nelz) {
            const int64_t j = ((int64_t)gz * nelx + gx) * nely + gy;
            if (!(fixed && fixed[j])) v = weights_only ? 1.0 : (trans ? x[j] / wsum[j] : x[j]);
        }
        tile[idx] = v;
    }
    __syncthreads();
    const int ly = tid % FT_Y, lx = tid / FT_Y;
    const int gy = y0 + ly, gx = x0 + lx;
    if (gy >= nely || gx >= nelx) return;
    // the four outputs along z share every tap's weight and offset
    const double *c = tile + (R * TX + (lx + R)) * TY + (ly + R);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    for (int t = 0; t < ntaps; ++t) {
        const double w = sw[t];
        const double *ct = c + soff[t];
        a0 += w * ct[0];
        a1 += w * ct[TXY];
        a2 += w * ct[2 * TXY];
        a3 += w * ct[3 * TXY];
    }
    const double acc[FT_Z] = {a0, a1, a2, a3};
#pragma unroll
    for (int lz = 0; lz < FT_Z; ++lz) {
        const int gz = z0 + lz;
        if (gz >= nelz) break;
        const int64_t i = ((int64_t)gz * nelx + gx) * nely + gy;
        if (fixed && fixed[i]) y[i] = weights_only ? 1.0 : (trans ? x[i] / wsum[i] : x[i]);
        else y[i] = (weights_only || trans) ? acc[lz] : acc[lz] / wsum[i];
    }
}

size_t filter_tile_bytes(int ntaps, int R) {
    return sizeof(double) * ntaps + sizeof(double) * (FT_Y + 2 * R) * (FT_X + 2 * R) * (FT_Z + 2 * R) +
           sizeof(int) * ntaps;
}

void launch_filter(const double *x, double *y, const double *wsum, const uint8_t *fixed, const FilterTap *taps_dev,
                   int ntaps, int nelx, int nely, int nelz, int trans, int weights_only, int radius, cudaStream_t st) {
    const size_t smem = radius >= 0 ? filter_tile_bytes(ntaps, radius) : 0;
    if (radius >= 0 && smem <= 160 * 1024) {
        static int attr_dev = -1;   // opt-in above 48 KB, per device
        int dev = 0;
        cudaGetDevice(&dev);
        if (attr_dev != dev) {
            cudaFuncSetAttribute(k_filter_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
            attr_dev = dev;
        }
        const dim3 grid((unsigned)((nely + FT_Y - 1) / FT_Y), (unsigned)((nelx + FT_X - 1) / FT_X),
                        (unsigned)((nelz + FT_Z - 1) / FT_Z));
        k_filter_tiled<<<grid, 256, smem, st>>>(x, y, wsum, fixed, taps_dev, ntaps, nelx, nely, nelz, trans,
                                                weights_only, radius);
        count_launch();
        return;
    }
    const int64_t n = (int64_t)nelx * nely * nelz;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 16384) blocks = 16384;
    if (blocks < 1) blocks = 1;
    k_filter<<<(unsigned)blocks, 256, 0, st>>>(x, y, wsum, fixed, taps_dev, ntaps, nelx, nely, nelz, trans,
                                               weights_only); count_launch();
}

}  // namespace tosp
