// Persistent small-level multigrid cycle.
//
// Below the first coarse level with few nodes, a V- or W-cycle (I/VCycle.m:
// 23-43, I/WCycle.m:23-44 with Smooth, Prolongation and the coarsest direct
// solve) is a chain of tiny dependent steps: warp-per-node stencil sweeps and
// residuals, restrictions, prolongations and the dense solve, each a few
// microseconds of launch and drain latency for little work.  Here the whole
// chain is one cooperative kernel: the host resolves every step to its buffers
// once (SmallStep list, rebuilt after each hierarchy setup) and the kernel walks
// the list with a grid barrier between steps.  Each step's arithmetic is that of
// the standalone kernel it replaces (k_stencil_warp, k_restrict, k_prolong,
// k_jacobi, k_dense_gemv), so the results are the same.
//
// Vectors written by one step and read by a later one are loaded with
// ld.global.cg (L2, coherent across the grid after the barrier's acquire);
// stencils, diagonals, masks and the coarsest inverse are read-only for the
// whole kernel.  The barrier's wait is bounded: on time-out it sets bar->err
// and every block leaves the step loop.  The poll limit and one block that
// skips its first arrival can be set from the host (tosp_inject_wait_fault),
// so tests make the wait run out without faulting or hanging the GPU.
#include "grid_sync.cuh"
#include "tosp_internal.h"

namespace tosp {

namespace {

constexpr int SMALL_THREADS = 256;
constexpr uint32_t SMALL_WAIT_LIMIT = 1u << 21;   // polls of 64 ns or more: > 0.1 s

__device__ __forceinline__ void small_node_xyz(int64_t I, int ny, int nx, int &x, int &y, int &z) {
    const int i = (int)I, q = i / ny;   // small levels: node indices far below 2^31
    y = i - q * ny;
    z = q / nx;
    x = q - z * nx;
}

template <typename T>
__device__ __forceinline__ T ldc(const T *p) {
    return __ldcg(p);
}

// k_stencil_warp's arithmetic: lane o < 27 applies the node's block for
// offset o, the warp sums the partial rows.
template <typename T>
__device__ void step_stencil(const SmallStep<T> &s, int64_t warp, int64_t nwarps, int lane) {
    const Grid g = s.g;
    for (int64_t I = warp; I < g.nnodes; I += nwarps) {
        T a0 = 0, a1 = 0, a2 = 0;
        if (lane < 27) {
            int xx, yy, zz;
            small_node_xyz(I, g.ny, g.nx, xx, yy, zz);
            const int oy = lane % 3 - 1, ox = (lane / 3) % 3 - 1, oz = lane / 9 - 1;
            const int jx = xx + ox, jy = yy + oy, jz = zz + oz;
            if (jx >= 0 && jx < g.nx && jy >= 0 && jy < g.ny && jz >= 0 && jz < g.nz) {
                const int64_t J = I + ((int64_t)oz * g.nx + ox) * g.ny + oy;
                const T x0 = ldc(s.x + 3 * J), x1 = ldc(s.x + 3 * J + 1), x2 = ldc(s.x + 3 * J + 2);
                const T *sv = s.st + I * STENCIL_VALS + lane * 9;
                a0 = __ldg(sv + 0) * x0 + __ldg(sv + 1) * x1 + __ldg(sv + 2) * x2;
                a1 = __ldg(sv + 3) * x0 + __ldg(sv + 4) * x1 + __ldg(sv + 5) * x2;
                a2 = __ldg(sv + 6) * x0 + __ldg(sv + 7) * x1 + __ldg(sv + 8) * x2;
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
            if (s.mode == 1) s.y[d] = ldc(s.b + d) - a;
            else s.y[d] = ldc(s.x + d) + __ldg(s.invd + d) * (ldc(s.b + d) - a);
        }
    }
}

// k_restrict's arithmetic (27 fine neighbours, clamped, zero weights outside).
template <typename T>
__device__ void step_restrict(const SmallStep<T> &s, int64_t t0, int64_t nt) {
    const Grid gf = s.g, gc = s.gc;
    for (int64_t J = t0; J < gc.nnodes; J += nt) {
        int cx, cy, cz;
        small_node_xyz(J, gc.ny, gc.nx, cx, cy, cz);
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
                    v0 += wt * ldc(s.x + 3 * I);
                    v1 += wt * ldc(s.x + 3 * I + 1);
                    v2 += wt * ldc(s.x + 3 * I + 2);
                }
            }
        }
        const T b[3] = {s.fm[3 * J] ? v0 : T(0), s.fm[3 * J + 1] ? v1 : T(0), s.fm[3 * J + 2] ? v2 : T(0)};
        for (int c = 0; c < 3; ++c) {
            s.y[3 * J + c] = b[c];
            if (s.xc) s.xc[3 * J + c] = __ldg(s.invdc + 3 * J + c) * b[c];
        }
    }
}

// k_prolong's arithmetic, accumulating into the fine level.
template <typename T>
__device__ void step_prolong(const SmallStep<T> &s, int64_t t0, int64_t nt) {
    const Grid gf = s.g, gc = s.gc;
    for (int64_t I = t0; I < gf.nnodes; I += nt) {
        int fx, fy, fz;
        small_node_xyz(I, gf.ny, gf.nx, fx, fy, fz);
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
                    v0 += w * ldc(s.x + 3 * J);
                    v1 += w * ldc(s.x + 3 * J + 1);
                    v2 += w * ldc(s.x + 3 * J + 2);
                }
            }
        }
        const T v[3] = {v0, v1, v2};
        for (int c = 0; c < 3; ++c) {
            const int64_t d = 3 * I + c;
            if (s.fm[d]) s.y[d] = ldc(s.y + d) + v[c];
        }
    }
}

// k_dense_gemv's arithmetic: warp per row, four partial sums.
template <typename T>
__device__ void step_dense(const SmallStep<T> &s, int64_t warp, int64_t nwarps, int lane) {
    const int64_t n = s.n, npad = s.npad;
    for (int64_t row = warp; row < n; row += nwarps) {
        const double *xr = s.X + row * npad;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int64_t j = lane;
        for (; j + 96 < n; j += 128) {
            s0 += __ldg(xr + j) * (double)ldc(s.b + j);
            s1 += __ldg(xr + j + 32) * (double)ldc(s.b + j + 32);
            s2 += __ldg(xr + j + 64) * (double)ldc(s.b + j + 64);
            s3 += __ldg(xr + j + 96) * (double)ldc(s.b + j + 96);
        }
        for (; j < n; j += 32) s0 += __ldg(xr + j) * (double)ldc(s.b + j);
        double sum = (s0 + s1) + (s2 + s3);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) s.y[row] = (T)sum;
    }
}

// One step over threads tid of nt (a multiple of the warp size).
template <typename T>
__device__ __forceinline__ void run_step(const SmallStep<T> &s, int64_t tid, int64_t nt, int lane) {
    const int64_t warp = tid >> 5, nwarps = nt >> 5;
    switch (s.kind) {
    case SS_STENCIL:
        step_stencil(s, warp, nwarps, lane);
        break;
    case SS_RESTRICT:
        step_restrict(s, tid, nt);
        break;
    case SS_PROLONG:
        step_prolong(s, tid, nt);
        break;
    case SS_JACOBI0:
        for (int64_t i = tid; i < s.g.ndof; i += nt) s.y[i] = __ldg(s.invd + i) * ldc(s.b + i);
        break;
    case SS_DENSE:
        step_dense(s, warp, nwarps, lane);
        break;
    default:   // SS_COPY
        for (int64_t i = tid; i < s.g.ndof; i += nt) s.y[i] = s.x ? ldc(s.x + i) : T(0);
        break;
    }
}

// The small-level cycles of several solves of one shape (the serving loop's
// batch): member m owns blocks block0 .. block0 + nblocks - 1 and its own
// step list; step k of every member runs between the same two grid barriers,
// so one launch per visit serves the whole batch.
template <typename T>
__global__ void __launch_bounds__(SMALL_THREADS)
k_small_cycle_batch(const SmallBatchEntry *__restrict__ ent, int nmem, int maxsteps, GridBarrier *bar) {
    int m = 0;
    while (m + 1 < nmem && (int)blockIdx.x >= ent[m + 1].block0) ++m;
    const SmallBatchEntry me = ent[m];
    const SmallStep<T> *steps = reinterpret_cast<const SmallStep<T> *>(me.steps);
    const int64_t tid = (int64_t)(blockIdx.x - me.block0) * blockDim.x + threadIdx.x;
    const int64_t nt = (int64_t)me.nblocks * blockDim.x;
    const int lane = threadIdx.x & 31;
    const uint32_t limit = bar->limit ? bar->limit : SMALL_WAIT_LIMIT;
    for (int k = 0; k < maxsteps; ++k) {
        if (k < me.nsteps) run_step(steps[k], tid, nt, lane);
        if (k + 1 < maxsteps && !grid_barrier(bar, gridDim.x, limit, false)) return;
    }
}

template <typename T>
__global__ void __launch_bounds__(SMALL_THREADS)
k_small_cycle(const SmallStep<T> *__restrict__ steps, int nsteps, GridBarrier *bar) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nt = (int64_t)gridDim.x * blockDim.x;
    const int64_t warp = tid >> 5, nwarps = nt >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t limit = bar->limit ? bar->limit : SMALL_WAIT_LIMIT;
    const bool skip_first = bar->skip == (int)blockIdx.x + 1;
    for (int k = 0; k < nsteps; ++k) {
        const SmallStep<T> s = steps[k];
        switch (s.kind) {
        case SS_STENCIL:
            step_stencil(s, warp, nwarps, lane);
            break;
        case SS_RESTRICT:
            step_restrict(s, tid, nt);
            break;
        case SS_PROLONG:
            step_prolong(s, tid, nt);
            break;
        case SS_JACOBI0:
            for (int64_t i = tid; i < s.g.ndof; i += nt) s.y[i] = __ldg(s.invd + i) * ldc(s.b + i);
            break;
        case SS_DENSE:
            step_dense(s, warp, nwarps, lane);
            break;
        default:   // SS_COPY
            for (int64_t i = tid; i < s.g.ndof; i += nt) s.y[i] = s.x ? ldc(s.x + i) : T(0);
            break;
        }
        if (k + 1 < nsteps && !grid_barrier(bar, gridDim.x, limit, skip_first && k == 0)) return;
    }
}

}  // namespace

int small_cycle_max_blocks(bool fp64) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const cudaError_t e = fp64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_small_cycle<double>,
                                                                                SMALL_THREADS, 0)
                               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_small_cycle<float>,
                                                                                SMALL_THREADS, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return per_sm * sms;
}

int small_cycle_batch_max_blocks(bool fp64) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const cudaError_t e = fp64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_small_cycle_batch<double>,
                                                                                SMALL_THREADS, 0)
                               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_small_cycle_batch<float>,
                                                                                SMALL_THREADS, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return per_sm * sms;
}

template <typename T>
void launch_small_cycle(const SmallStep<T> *steps_dev, int nsteps, GridBarrier *bar, int blocks, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(SMALL_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_small_cycle<T>, steps_dev, nsteps, bar);
    count_launch();
}
template void launch_small_cycle<double>(const SmallStep<double> *, int, GridBarrier *, int, cudaStream_t);
template void launch_small_cycle<float>(const SmallStep<float> *, int, GridBarrier *, int, cudaStream_t);

template <typename T>
void launch_small_cycle_batch(const SmallBatchEntry *ent_dev, int nmem, int maxsteps, GridBarrier *bar, int blocks,
                              cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(SMALL_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_small_cycle_batch<T>, ent_dev, nmem, maxsteps, bar);
    count_launch();
}
template void launch_small_cycle_batch<double>(const SmallBatchEntry *, int, int, GridBarrier *, int, cudaStream_t);
template void launch_small_cycle_batch<float>(const SmallBatchEntry *, int, int, GridBarrier *, int, cudaStream_t);

}  // namespace tosp
