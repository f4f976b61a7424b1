// Coarsest-grid direct solve in FP64.
//
// The reference factors the coarsest Galerkin matrix once per setup with
// amd + sparse chol and applies eH = R\(R'\rH(perm)) in every cycle
// (I/SetupGMG.m:51-59, I/VCycle.m:40).  Here the coarsest matrix is assembled
// densely (fixed dofs decoupled with a unit diagonal, padded to a multiple of
// 32 with identity) and inverted once per setup in place by a blocked
// symmetric sweep, so that each cycle's coarse solve is a single FP64 GEMV
// that runs from L2.
#include "tosp_internal.h"

namespace tosp {

constexpr int TS = 32;

__global__ void k_dense_zero(double *A, int64_t nn) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x)
        A[i] = 0.0;
}

__global__ void k_dense_scatter(const double *__restrict__ Ae, const uint8_t *__restrict__ fm, Grid g, double *A,
                                int64_t npad) {
    const int64_t total = g.nelem * 576;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t E = t / 576;
        const int e = (int)(t % 576), i = e / 24, j = e % 24;
        const int ey = (int)(E % g.nely), ex = (int)((E / g.nely) % g.nelx), ez = (int)(E / ((int64_t)g.nely * g.nelx));
        const int a = i / 3, ca = i % 3, b = j / 3, cb = j % 3;
        const int64_t na = ((int64_t)(ez + ((a >> 2) & 1)) * g.nx + (ex + ((a >> 1) & 1))) * g.ny + (ey + (a & 1));
        const int64_t nb = ((int64_t)(ez + ((b >> 2) & 1)) * g.nx + (ex + ((b >> 1) & 1))) * g.ny + (ey + (b & 1));
        const int64_t di = 3 * na + ca, dj = 3 * nb + cb;
        if (fm[di] && fm[dj]) atomicAdd(&A[di * npad + dj], Ae[t]);
    }
}

__global__ void k_dense_unitdiag(double *A, const uint8_t *fm, int64_t n, int64_t npad) {
    for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < npad; d += (int64_t)gridDim.x * blockDim.x)
        if (d >= n || !fm[d]) A[d * npad + d] = 1.0;
}

void launch_dense_assemble(const double *Ae, const uint8_t *freemask, const Grid &g, double *A, int64_t npad,
                           cudaStream_t st) {
    k_dense_zero<<<1024, 256, 0, st>>>(A, npad * npad); count_launch();
    k_dense_scatter<<<1024, 256, 0, st>>>(Ae, freemask, g, A, npad); count_launch();
    k_dense_unitdiag<<<64, 256, 0, st>>>(A, freemask, g.ndof, npad); count_launch();
}

// --- blocked symmetric sweep (block Gauss-Jordan) ----------------------------
// Sweeping block k of a symmetric matrix:  P = A_kk,  C_i = A_ik P^{-1},
//   A_ij -= C_i A_kj (i, j != k),  A_ik = C_i,  A_kj = C_j',  A_kk = -P^{-1}.
// After all blocks the array holds -A^{-1}.  Every pivot block is a Schur
// complement of the SPD matrix (a leading-block Cholesky factor exists), so no
// pivoting is needed.  Each step is one small pivot inversion plus an
// embarrassingly parallel rank-32 update of the whole matrix.

// P^{-1} of the 32x32 pivot block by a scalar sweep in shared memory.
__global__ void k_sweep_pivot(const double *A, int64_t npad, int k, double *Pinv, int *info) {
    __shared__ double S[TS][TS + 1];
    __shared__ double rd;
    const int r = threadIdx.y, c = threadIdx.x;   // 32 x 32
    S[r][c] = A[(int64_t)(k * TS + r) * npad + k * TS + c];
    for (int p = 0; p < TS; ++p) {
        __syncthreads();
        if (r == 0 && c == 0) {   // one division per step, shared by all threads
            const double d = S[p][p];
            if (!(d > 0.0)) atomicExch(info, 1 + k * TS + p);
            rd = 1.0 / d;
        }
        __syncthreads();
        const double q = rd;
        double v;
        if (r == p && c == p) v = -q;
        else if (c == p) v = S[r][p] * q;
        else if (r == p) v = S[p][c] * q;
        else v = S[r][c] - S[r][p] * (S[p][c] * q);
        __syncthreads();
        S[r][c] = v;
    }
    __syncthreads();
    Pinv[r * TS + c] = -S[r][c];
}

// C_i = A_ik P^{-1} for every row block i != k.
__global__ void k_sweep_panel(const double *A, int64_t npad, int k, const double *Pinv, double *C) {
    __shared__ double At[TS][TS + 1];
    __shared__ double Pt[TS][TS + 1];
    const int i = blockIdx.x;
    if (i == k) return;
    const int r = threadIdx.y, c = threadIdx.x;
    At[r][c] = A[(int64_t)(i * TS + r) * npad + k * TS + c];
    Pt[r][c] = Pinv[r * TS + c];
    __syncthreads();
    double v = 0.0;
#pragma unroll 8
    for (int q = 0; q < TS; ++q) v += At[r][q] * Pt[q][c];
    C[(int64_t)(i * TS + r) * TS + c] = v;
}

// A_ij -= C_i A_kj for all entries outside row and column block k: a
// rank-32 update by 64 x 64 tiles, 256 threads, 4 x 4 outputs per thread
// (rows ty + 16 a, columns tx + 16 b) from shared copies of the tile's C rows
// and A_k columns.
constexpr int UT = 64;
__global__ void __launch_bounds__(256) k_sweep_update(double *A, int64_t npad, int k, const double *C, int ntile) {
    __shared__ double Cs[UT][TS + 1];
    __shared__ double Rs[TS][UT + 1];
    const int ti = blockIdx.x / ntile, tj = blockIdx.x % ntile;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int row0 = ti * UT, col0 = tj * UT;
    for (int e = threadIdx.x; e < UT * TS; e += 256) {
        const int rr = e / TS, q = e % TS;
        const int64_t gr = row0 + rr;
        Cs[rr][q] = gr < npad ? C[gr * TS + q] : 0.0;
        const int q2 = e / UT, cc = e % UT;
        const int64_t gc = col0 + cc;
        Rs[q2][cc] = gc < npad ? A[(int64_t)(k * TS + q2) * npad + gc] : 0.0;
    }
    __syncthreads();
    double acc[4][4] = {};
#pragma unroll 8
    for (int q = 0; q < TS; ++q) {
        double cv[4], rv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) cv[a] = Cs[ty + 16 * a][q];
#pragma unroll
        for (int b = 0; b < 4; ++b) rv[b] = Rs[q][tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = fma(cv[a], rv[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int64_t gr = row0 + ty + 16 * a;
        if (gr >= npad || gr / TS == k) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int64_t gc = col0 + tx + 16 * b;
            if (gc >= npad || gc / TS == k) continue;
            A[gr * npad + gc] -= acc[a][b];
        }
    }
}

// Column and row blocks of k: A_ik = C_i, A_ki = C_i', A_kk = -P^{-1}.
__global__ void k_sweep_setrc(double *A, int64_t npad, int k, const double *C, const double *Pinv) {
    const int i = blockIdx.x;
    const int r = threadIdx.y, c = threadIdx.x;
    if (i == k) {
        A[(int64_t)(k * TS + r) * npad + k * TS + c] = -Pinv[r * TS + c];
    } else {
        const double v = C[(int64_t)(i * TS + r) * TS + c];
        A[(int64_t)(i * TS + r) * npad + k * TS + c] = v;
        A[(int64_t)(k * TS + c) * npad + i * TS + r] = v;
    }
}

__global__ void k_negate(double *A, int64_t nn) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x)
        A[i] = -A[i];
}

int dense_sweep_inverse(double *A, double *C, double *Pinv, int64_t npad, int *d_info, cudaStream_t st) {
    const int nb = (int)(npad / TS);
    const int ntile = (int)((npad + UT - 1) / UT);
    const dim3 blk(TS, TS);
    cudaMemsetAsync(d_info, 0, sizeof(int), st);
    for (int k = 0; k < nb; ++k) {
        k_sweep_pivot<<<1, blk, 0, st>>>(A, npad, k, Pinv, d_info); count_launch();
        k_sweep_panel<<<nb, blk, 0, st>>>(A, npad, k, Pinv, C); count_launch();
        k_sweep_update<<<ntile * ntile, 256, 0, st>>>(A, npad, k, C, ntile); count_launch();
        k_sweep_setrc<<<nb, blk, 0, st>>>(A, npad, k, C, Pinv); count_launch();
    }
    k_negate<<<1024, 256, 0, st>>>(A, npad * npad); count_launch();
    return 0;
}

// x = X b (X symmetric, npad x npad; only the first n entries are used).
template <typename T>
__global__ void __launch_bounds__(256)
k_dense_gemv(const double *__restrict__ X, const T *__restrict__ b, T *__restrict__ x, int64_t n, int64_t npad) {
    // Four warps per row (two rows per block), four partial sums per lane:
    // the coarsest system has only a few thousand rows, and with one warp
    // per row the loads in flight were too few to cover the memory latency.
    __shared__ double part[8];
    const int lane = threadIdx.x & 127;   // lane within the row's four warps
    const int grp = threadIdx.x >> 7;     // row of the block (0, 1)
    const int w = threadIdx.x >> 5;       // warp of the block
    for (int64_t row0 = 2 * (int64_t)blockIdx.x; row0 < n; row0 += 2 * (int64_t)gridDim.x) {   // block-uniform
        const int64_t row = row0 + grp;
        double s = 0.0;
        if (row < n) {
            const double *xr = X + row * npad;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            int64_t j = lane;
            for (; j + 384 < n; j += 512) {
                s0 += xr[j] * (double)b[j];
                s1 += xr[j + 128] * (double)b[j + 128];
                s2 += xr[j + 256] * (double)b[j + 256];
                s3 += xr[j + 384] * (double)b[j + 384];
            }
            for (; j < n; j += 128) s0 += xr[j] * (double)b[j];
            s = (s0 + s1) + (s2 + s3);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) part[w] = s;
        __syncthreads();
        if (lane == 0 && row < n) x[row] = (T)((part[4 * grp] + part[4 * grp + 1]) + (part[4 * grp + 2] + part[4 * grp + 3]));
        __syncthreads();
    }
}

template <typename T>
void launch_dense_solve(const double *X, const T *b, T *x, int64_t n, int64_t npad, cudaStream_t st) {
    int64_t blocks = (n + 1) / 2;
    if (blocks > 2048) blocks = 2048;
    if (blocks < 1) blocks = 1;
    k_dense_gemv<T><<<(unsigned)blocks, 256, 0, st>>>(X, b, x, n, npad); count_launch();
}
template void launch_dense_solve<double>(const double *, const double *, double *, int64_t, int64_t, cudaStream_t);
template void launch_dense_solve<float>(const double *, const float *, float *, int64_t, int64_t, cudaStream_t);

}  // namespace tosp
