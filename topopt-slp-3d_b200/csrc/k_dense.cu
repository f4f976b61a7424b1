// Coarsest-grid direct solve in FP64.
//
// The reference factors the coarsest Galerkin matrix once per setup with
// amd + sparse chol and applies eH = R\(R'\rH(perm)) in every cycle
// (I/SetupGMG.m:51-59, I/VCycle.m:40).  Here the coarsest matrix is assembled
// densely (fixed dofs decoupled with a unit diagonal, padded to a multiple of
// 32 with identity), factored A = L L' by a blocked right-looking Cholesky,
// and inverted once (L Y = I, L' X = Y, both blocked over 32x32 tiles), so that
// each cycle's coarse solve is a single FP64 GEMV that runs from L2.
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

// --- blocked Cholesky ------------------------------------------------------
__global__ void k_potrf_tile(double *A, int64_t npad, int k, int *info) {
    __shared__ double s[TS][TS + 1];
    const int tx = threadIdx.x;   // 32 threads, one per row
    double *base = A + (int64_t)k * TS * npad + (int64_t)k * TS;
    for (int c = 0; c < TS; ++c) s[tx][c] = base[(int64_t)tx * npad + c];
    __syncthreads();
    for (int j = 0; j < TS; ++j) {
        if (tx == j) {
            const double d = s[j][j];
            if (!(d > 0.0)) {
                atomicExch(info, 1 + k * TS + j);
                s[j][j] = 1.0;
            } else {
                s[j][j] = sqrt(d);
            }
        }
        __syncthreads();
        if (tx > j) s[tx][j] /= s[j][j];
        __syncthreads();
        if (tx > j)
            for (int l = j + 1; l <= tx; ++l) s[tx][l] -= s[tx][j] * s[l][j];
        __syncthreads();
    }
    for (int c = 0; c < TS; ++c) base[(int64_t)tx * npad + c] = (c <= tx) ? s[tx][c] : 0.0;
}

// L_ik = A_ik L_kk^{-T} for tile rows i > k.
__global__ void k_trsm_panel(double *A, int64_t npad, int k) {
    __shared__ double L[TS][TS + 1];
    __shared__ double X[TS][TS + 1];
    const int tx = threadIdx.x;
    const int i = k + 1 + blockIdx.x;
    const double *lk = A + (int64_t)k * TS * npad + (int64_t)k * TS;
    double *ai = A + (int64_t)i * TS * npad + (int64_t)k * TS;
    for (int c = 0; c < TS; ++c) {
        L[tx][c] = lk[(int64_t)tx * npad + c];
        X[tx][c] = ai[(int64_t)tx * npad + c];
    }
    __syncthreads();
    for (int j = 0; j < TS; ++j) {
        double v = X[tx][j];
        for (int p = 0; p < j; ++p) v -= X[tx][p] * L[j][p];
        X[tx][j] = v / L[j][j];
    }
    for (int c = 0; c < TS; ++c) ai[(int64_t)tx * npad + c] = X[tx][c];
}

// A_ij -= L_ik L_jk' for the lower tiles k < j <= i.
__global__ void k_syrk(double *A, int64_t npad, int k) {
    __shared__ double Li[TS][TS + 1];
    __shared__ double Lj[TS][TS + 1];
    const int t = blockIdx.x;
    int row = (int)((sqrt(8.0 * t + 1.0) - 1.0) / 2.0);
    while ((row + 1) * (row + 2) / 2 <= t) ++row;
    while (row * (row + 1) / 2 > t) --row;
    const int col = t - row * (row + 1) / 2;
    const int i = k + 1 + row, j = k + 1 + col;
    const int tid = threadIdx.x;   // 256 threads
    const double *li = A + (int64_t)i * TS * npad + (int64_t)k * TS;
    const double *lj = A + (int64_t)j * TS * npad + (int64_t)k * TS;
    for (int e = tid; e < TS * TS; e += blockDim.x) {
        const int r = e / TS, c = e % TS;
        Li[r][c] = li[(int64_t)r * npad + c];
        Lj[r][c] = lj[(int64_t)r * npad + c];
    }
    __syncthreads();
    double *aij = A + (int64_t)i * TS * npad + (int64_t)j * TS;
    for (int e = tid; e < TS * TS; e += blockDim.x) {
        const int r = e / TS, c = e % TS;
        double v = 0.0;
#pragma unroll 8
        for (int p = 0; p < TS; ++p) v += Li[r][p] * Lj[c][p];
        aij[(int64_t)r * npad + c] -= v;
    }
}

// --- inverse from the factor -------------------------------------------------
// Forward: Y_kc = L_kk^{-1} (I_kc - sum_{c<=j<k} L_kj Y_jc), c <= k.
__global__ void k_fwd(const double *A, double *Y, int64_t npad, int k) {
    __shared__ double Lt[TS][TS + 1];
    __shared__ double Bt[TS][TS + 1];
    __shared__ double acc[TS][TS + 1];
    const int c = blockIdx.x;   // column tile
    const int r = threadIdx.y, q = threadIdx.x;   // 32 x 32
    double v = (c == k && r == q) ? 1.0 : 0.0;
    for (int j = c; j < k; ++j) {
        Lt[r][q] = A[(int64_t)(k * TS + r) * npad + j * TS + q];
        Bt[r][q] = Y[(int64_t)(j * TS + r) * npad + c * TS + q];
        __syncthreads();
#pragma unroll 8
        for (int p = 0; p < TS; ++p) v -= Lt[r][p] * Bt[p][q];
        __syncthreads();
    }
    acc[r][q] = v;
    Lt[r][q] = A[(int64_t)(k * TS + r) * npad + k * TS + q];
    __syncthreads();
    if (r == 0) {   // one thread per column solves down the tile
        for (int rr = 0; rr < TS; ++rr) {
            double z = acc[rr][q];
            for (int p = 0; p < rr; ++p) z -= Lt[rr][p] * acc[p][q];
            acc[rr][q] = z / Lt[rr][rr];
        }
    }
    __syncthreads();
    Y[(int64_t)(k * TS + r) * npad + c * TS + q] = acc[r][q];
}

// Backward (in place over Y): X_kc = L_kk^{-T} (Y_kc - sum_{j>k} L_jk' X_jc).
__global__ void k_bwd(const double *A, double *X, int64_t npad, int k, int nb) {
    __shared__ double Lt[TS][TS + 1];
    __shared__ double Bt[TS][TS + 1];
    __shared__ double acc[TS][TS + 1];
    const int c = blockIdx.x;
    const int r = threadIdx.y, q = threadIdx.x;
    double v = X[(int64_t)(k * TS + r) * npad + c * TS + q];
    for (int j = k + 1; j < nb; ++j) {
        Lt[r][q] = A[(int64_t)(j * TS + r) * npad + k * TS + q];   // L_jk[r][q]
        Bt[r][q] = X[(int64_t)(j * TS + r) * npad + c * TS + q];
        __syncthreads();
#pragma unroll 8
        for (int p = 0; p < TS; ++p) v -= Lt[p][r] * Bt[p][q];
        __syncthreads();
    }
    acc[r][q] = v;
    Lt[r][q] = A[(int64_t)(k * TS + r) * npad + k * TS + q];
    __syncthreads();
    if (r == 0) {
        for (int rr = TS - 1; rr >= 0; --rr) {
            double z = acc[rr][q];
            for (int p = rr + 1; p < TS; ++p) z -= Lt[p][rr] * acc[p][q];
            acc[rr][q] = z / Lt[rr][rr];
        }
    }
    __syncthreads();
    X[(int64_t)(k * TS + r) * npad + c * TS + q] = acc[r][q];
}

int dense_cholesky_inverse(double *A, double *X, int64_t npad, int *d_info, cudaStream_t st) {
    const int nb = (int)(npad / TS);
    cudaMemsetAsync(d_info, 0, sizeof(int), st);
    for (int k = 0; k < nb; ++k) {
        k_potrf_tile<<<1, TS, 0, st>>>(A, npad, k, d_info); count_launch();
        const int m = nb - k - 1;
        if (m > 0) {
            k_trsm_panel<<<m, TS, 0, st>>>(A, npad, k); count_launch();
            k_syrk<<<m * (m + 1) / 2, 256, 0, st>>>(A, npad, k); count_launch();
        }
    }
    const dim3 blk(TS, TS);
    // tiles above the block diagonal of L^{-1} are zero and are read by the
    // backward sweep
    cudaMemsetAsync(X, 0, sizeof(double) * npad * npad, st);
    for (int k = 0; k < nb; ++k) k_fwd<<<k + 1, blk, 0, st>>>(A, X, npad, k); count_launch();
    for (int k = nb - 1; k >= 0; --k) k_bwd<<<nb, blk, 0, st>>>(A, X, npad, k, nb); count_launch();
    return 0;
}

// x = X b (X symmetric, npad x npad; only the first n entries are used).
template <typename T>
__global__ void k_dense_gemv(const double *__restrict__ X, const T *__restrict__ b, T *__restrict__ x, int64_t n,
                             int64_t npad) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t row = warp; row < n; row += nwarps) {
        const double *xr = X + row * npad;
        double s = 0.0;
        for (int64_t j = lane; j < n; j += 32) s += xr[j] * (double)b[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) x[row] = (T)s;
    }
}

template <typename T>
void launch_dense_solve(const double *X, const T *b, T *x, int64_t n, int64_t npad, cudaStream_t st) {
    int64_t blocks = (n * 32 + 255) / 256;
    if (blocks > 2048) blocks = 2048;
    if (blocks < 1) blocks = 1;
    k_dense_gemv<T><<<(unsigned)blocks, 256, 0, st>>>(X, b, x, n, npad); count_launch();
}
template void launch_dense_solve<double>(const double *, const double *, double *, int64_t, int64_t, cudaStream_t);
template void launch_dense_solve<float>(const double *, const float *, float *, int64_t, int64_t, cudaStream_t);

}  // namespace tosp
