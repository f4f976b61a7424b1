// Vector kernels of the FP64 outer CG (I/SolveMG.m:26-53) and the free-dof
// boundary conversions.  Dot products use a fixed two-stage reduction tree
// (RED_BLOCKS partial sums, then one block), so results are bitwise
// reproducible run to run.
#include "tosp_internal.h"

namespace tosp {

static unsigned gridv(int64_t n) {
    int64_t b = (n + 255) / 256;
    if (b > 8192) b = 8192;
    if (b < 1) b = 1;
    return (unsigned)b;
}

__global__ void k_scatter(const double *v, const int64_t *idx, int64_t nfree, double *full) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nfree; i += (int64_t)gridDim.x * blockDim.x)
        full[idx[i]] = v[i];
}
void launch_scatter_free(const double *v, const int64_t *idx, int64_t nfree, double *full, cudaStream_t st) {
    k_scatter<<<gridv(nfree), 256, 0, st>>>(v, idx, nfree, full); count_launch();
}

__global__ void k_gather(const double *full, const int64_t *idx, int64_t nfree, double *v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nfree; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = full[idx[i]];
}
void launch_gather_free(const double *full, const int64_t *idx, int64_t nfree, double *v, cudaStream_t st) {
    k_gather<<<gridv(nfree), 256, 0, st>>>(full, idx, nfree, v); count_launch();
}

template <typename TI, typename TO>
__global__ void k_convert(const TI *a, TO *b, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (TO)a[i];
}
template <typename TI, typename TO>
void launch_convert(const TI *a, TO *b, int64_t n, cudaStream_t st) {
    k_convert<TI, TO><<<gridv(n), 256, 0, st>>>(a, b, n); count_launch();
}
template void launch_convert<double, float>(const double *, float *, int64_t, cudaStream_t);
template void launch_convert<float, double>(const float *, double *, int64_t, cudaStream_t);

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
    __syncthreads();
    return s;   // valid in thread 0
}

// Reductions finish in the last block to arrive (a self-resetting counter
// after the 2 * RED_BLOCKS partials), which sums the partials in the fixed
// order of a single-block reduction: one launch per dot, deterministic.
__device__ __forceinline__ unsigned *red_counter(double *partials) {
    return reinterpret_cast<unsigned *>(partials + 2 * RED_BLOCKS);
}

// Grid-stride loop of the reduction kernels over [0, n), taken B strides at a
// time (VB = 4 by default): load(k, i) reads element i into slot k for the B
// elements of a batch, then use(k, i) consumes them in index order.  The
// reduction grid is a few blocks per SM, so a thread walks dozens of
// elements; with one element's loads in flight the loop waits one DRAM
// latency per element, with B it waits one per batch.  A thread visits its elements in the same order as the
// plain grid-stride loop, so its running sums are bitwise the same.  The
// plain dot (two loads per element) takes batches of eight.
constexpr int VB = 4;
template <int B = VB, class Load, class Use>
__device__ __forceinline__ void grid_batched(int64_t n, Load load, Use use) {
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; i + (B - 1) * T < n; i += B * T) {
#pragma unroll
        for (int k = 0; k < B; ++k) load(k, i + k * T);
#pragma unroll
        for (int k = 0; k < B; ++k) use(k, i + k * T);
    }
    for (; i < n; i += T) {
        load(0, i);
        use(0, i);
    }
}

// Call after thread 0 wrote this block's partial(s); true in every thread of
// the last block, which then sees all partials.
__device__ __forceinline__ bool last_block(unsigned *counter) {
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicInc(counter, gridDim.x - 1) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

__device__ __forceinline__ double sum_partials(const double *partials, int np, double *sh) {
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += __ldcg(partials + i);
    return block_sum(s, sh);
}

template <typename TB>
__global__ void __launch_bounds__(256, 4) k_dot_partial(const double *a, const TB *b, int64_t n, double *partials, double *out) {
    __shared__ double sh[32];
    double s = 0.0;
    constexpr int VB8 = 2 * VB;
    double av[VB8];
    TB bv[VB8];
    grid_batched<VB8>(
        n, [&](int k, int64_t i) { av[k] = a[i]; bv[k] = b[i]; },
        [&](int k, int64_t) { s += av[k] * (double)bv[k]; });
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
    if (last_block(red_counter(partials))) {
        const double t = sum_partials(partials, gridDim.x, sh);
        if (threadIdx.x == 0) out[0] = t;
    }
}

void launch_dot(const double *a, const double *b, int64_t n, double *partials, double *out, cudaStream_t st) {
    k_dot_partial<double><<<RED_BLOCKS, 256, 0, st>>>(a, b, n, partials, out); count_launch();
}
void launch_dot(const double *a, const float *b, int64_t n, double *partials, double *out, cudaStream_t st) {
    k_dot_partial<float><<<RED_BLOCKS, 256, 0, st>>>(a, b, n, partials, out); count_launch();
}

// a'b and a'c in one pass over a (partials: 2 * RED_BLOCKS).
__global__ void __launch_bounds__(256, 4) k_dot2_partial(const double *a, const double *b, const double *c, int64_t n, double *partials,
                               double *out0, double *out1) {
    __shared__ double sh[32];
    double s = 0.0, t = 0.0;
    double av[VB], bv[VB], cv[VB];
    grid_batched(
        n, [&](int k, int64_t i) { av[k] = a[i]; bv[k] = b[i]; cv[k] = c[i]; },
        [&](int k, int64_t) {
            s += av[k] * bv[k];
            t += av[k] * cv[k];
        });
    s = block_sum(s, sh);
    t = block_sum(t, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = s;
        partials[RED_BLOCKS + blockIdx.x] = t;
    }
    if (last_block(red_counter(partials))) {
        const double s0 = sum_partials(partials, gridDim.x, sh);
        const double s1 = sum_partials(partials + RED_BLOCKS, gridDim.x, sh);
        if (threadIdx.x == 0) {
            out0[0] = s0;
            out1[0] = s1;
        }
    }
}

void launch_dot2(const double *a, const double *b, const double *c, int64_t n, double *partials, double *out0,
                 double *out1, cudaStream_t st) {
    k_dot2_partial<<<RED_BLOCKS, 256, 0, st>>>(a, b, c, n, partials, out0, out1); count_launch();
}

// The finest post-sweep of the preconditioner written as the FP64 CG vector,
// s = x + invd (b - t) (k_jacobi_out), with the CG's dots of the new s in the
// same pass: r's -> out0 and, when so is given, r's_old -> out1.  Same grid,
// loop order and reduction tree as k_dot2_partial / k_dot_partial, so the
// dots are bitwise those of the separate kernels.
template <typename T>
__global__ void __launch_bounds__(256, 4) k_jacobi_out_dot(double *out, const T *x, const T *b, const T *t, const T *invd, int64_t n,
                                 const double *r, const double *so, double *partials, double *out0, double *out1) {
    __shared__ double sh[32];
    double s0 = 0.0, s1 = 0.0;
    T xv[VB], bv[VB], tv[VB], dv[VB];
    double rv[VB], ov[VB];
    grid_batched(
        n,
        [&](int k, int64_t i) {
            xv[k] = x[i];
            bv[k] = b[i];
            tv[k] = t[i];
            dv[k] = invd[i];
            rv[k] = r[i];
            if (so) ov[k] = so[i];
        },
        [&](int k, int64_t i) {
            const double si = (double)(xv[k] + dv[k] * (bv[k] - tv[k]));
            out[i] = si;
            s0 += rv[k] * si;
            if (so) s1 += rv[k] * ov[k];
        });
    s0 = block_sum(s0, sh);
    if (so) s1 = block_sum(s1, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = s0;
        partials[RED_BLOCKS + blockIdx.x] = s1;
    }
    if (last_block(red_counter(partials))) {
        const double t0 = sum_partials(partials, gridDim.x, sh);
        const double t1 = so ? sum_partials(partials + RED_BLOCKS, gridDim.x, sh) : 0.0;
        if (threadIdx.x == 0) {
            out0[0] = t0;
            if (so) out1[0] = t1;
        }
    }
}

template <typename T>
void launch_jacobi_out_dot(double *out, const T *x, const T *b, const T *t, const T *invd, int64_t n, const double *r,
                           const double *so, double *partials, double *out0, double *out1, cudaStream_t st) {
    k_jacobi_out_dot<T><<<RED_BLOCKS, 256, 0, st>>>(out, x, b, t, invd, n, r, so, partials, out0, out1);
    count_launch();
}
template void launch_jacobi_out_dot<float>(double *, const float *, const float *, const float *, const float *,
                                           int64_t, const double *, const double *, double *, double *, double *,
                                           cudaStream_t);
template void launch_jacobi_out_dot<double>(double *, const double *, const double *, const double *, const double *,
                                            int64_t, const double *, const double *, double *, double *, double *,
                                            cudaStream_t);

// Scalar slots (see solver.cpp): 0 rho, 1 gamma2 (previous rho), 2 d'q, 3 r'r,
// 5 r's_old, 6 the previous iteration's alpha.  mode 1: first iteration
// (d = s); 0: beta = rho/gamma2 (I/SolveMG.m:43-46); 2: flexible beta =
// (rho - r's_old)/gamma2.  When sold is given it receives s (the next
// iteration's s_old).  The iterate update of the previous iteration,
// x += alpha d (I/SolveMG.m:40), is done here, while d is read anyway, before
// d is replaced (modes 0 and 2); launch_pcg_finish applies the last one.
// d32 (optional) receives the new d in FP32, the input of the tensor-core
// product.
__global__ void k_pcg_direction(double *d, const double *s, double *sold, const double *scal, int64_t n, int mode,
                                double *x, float *d32) {
    const double beta = mode == 1 ? 0.0 : (mode == 2 ? (scal[0] - scal[5]) / scal[1] : scal[0] / scal[1]);
    const double alpha = scal[6];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double si = s[i];
        double dn = si;
        if (mode != 1) {
            const double di = d[i];
            x[i] += alpha * di;
            dn = beta * di + si;
        }
        d[i] = dn;
        if (d32) d32[i] = (float)dn;
        if (sold) sold[i] = si;
    }
}
void launch_pcg_direction(double *d, const double *s, double *sold, const double *scal, int64_t n, int mode,
                          double *x, cudaStream_t st, float *d32) {
    k_pcg_direction<<<gridv(n), 256, 0, st>>>(d, s, sold, scal, n, mode, x, d32); count_launch();
}

// x += alpha d with the last iteration's alpha (slot 6).
__global__ void k_pcg_finish(double *x, const double *d, const double *scal, int64_t n) {
    const double alpha = scal[6];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += alpha * d[i];
}
void launch_pcg_finish(double *x, const double *d, const double *scal, int64_t n, cudaStream_t st) {
    k_pcg_finish<<<gridv(n), 256, 0, st>>>(x, d, scal, n); count_launch();
}

// r -= alpha q (alpha = rho / d'q, kept in slot 6 for the iterate update),
// r'r into slot 3 and gamma2 = rho (last block).  For the mixed V-cycle (b0
// given) it also writes the next cycle's FP32 right-hand side b0 = r and, when
// x0 is given, its first Jacobi iterate x0 = invd0 b0 (the sweep from a zero
// guess).
template <typename TQ>
__global__ void __launch_bounds__(256, 4) k_pcg_update(double *r, const TQ *q, double *scal, int64_t n, double *partials, float *b0,
                             const float *invd0, float *x0) {
    __shared__ double sh[32];
    const double alpha = scal[0] / scal[2];
    double s = 0.0;
    double rv[VB];
    TQ qv[VB];
    float dv[VB];
    grid_batched(
        n,
        [&](int k, int64_t i) {
            rv[k] = r[i];
            qv[k] = q[i];
            if (b0 && x0) dv[k] = invd0[i];
        },
        [&](int k, int64_t i) {
            const double ri = rv[k] - alpha * (double)qv[k];
            r[i] = ri;
            s += ri * ri;
            if (b0) {
                const float bi = (float)ri;
                b0[i] = bi;
                if (x0) x0[i] = dv[k] * bi;
            }
        });
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
    if (last_block(red_counter(partials))) {
        const double t = sum_partials(partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            scal[3] = t;
            scal[1] = scal[0];
            scal[6] = alpha;
        }
    }
}

void launch_pcg_update(double *r, const double *q, double *scal, double *partials, int64_t n, cudaStream_t st,
                       float *b0, const float *invd0, float *x0) {
    k_pcg_update<double><<<RED_BLOCKS, 256, 0, st>>>(r, q, scal, n, partials, b0, invd0, x0); count_launch();
}
void launch_pcg_update(double *r, const float *q, double *scal, double *partials, int64_t n, cudaStream_t st,
                       float *b0, const float *invd0, float *x0) {
    k_pcg_update<float><<<RED_BLOCKS, 256, 0, st>>>(r, q, scal, n, partials, b0, invd0, x0); count_launch();
}

// Residual replacement: r = f - t (t = K x by the FP64 operator), r'r into
// slot 3 (last block) and, for the mixed V-cycle (b0 given), the next cycle's
// FP32 right-hand side and first Jacobi iterate as in k_pcg_update.
__global__ void __launch_bounds__(256, 4) k_replace_residual(const double *f, const double *t, double *r, double *scal, int64_t n,
                                   double *partials, float *b0, const float *invd0, float *x0) {
    __shared__ double sh[32];
    double s = 0.0;
    double fv[VB], tv[VB];
    float dv[VB];
    grid_batched(
        n,
        [&](int k, int64_t i) {
            fv[k] = f[i];
            tv[k] = t[i];
            if (b0 && x0) dv[k] = invd0[i];
        },
        [&](int k, int64_t i) {
            const double ri = fv[k] - tv[k];
            r[i] = ri;
            s += ri * ri;
            if (b0) {
                const float bi = (float)ri;
                b0[i] = bi;
                if (x0) x0[i] = dv[k] * bi;
            }
        });
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
    if (last_block(red_counter(partials))) {
        const double t2 = sum_partials(partials, gridDim.x, sh);
        if (threadIdx.x == 0) scal[3] = t2;
    }
}
void launch_replace_residual(const double *f, const double *t, double *r, double *scal, double *partials, int64_t n,
                             cudaStream_t st, float *b0, const float *invd0, float *x0) {
    k_replace_residual<<<RED_BLOCKS, 256, 0, st>>>(f, t, r, scal, n, partials, b0, invd0, x0); count_launch();
}

__global__ void k_set_scalar(double *dst, const double *src) { *dst = *src; }
void launch_set_scalar(double *dst, const double *src, cudaStream_t st) { k_set_scalar<<<1, 1, 0, st>>>(dst, src); count_launch(); }

}  // namespace tosp
