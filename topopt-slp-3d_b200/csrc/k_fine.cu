// Fine-level multiresolution hex8 operator, its diagonal, the SIMP factors
// and the compliance sensitivities.
//
// Operator (I/WOK/KelemProd.m:57-100): y_e = sum_s w_s KE_s u_e for every
// displacement element e, scatter-added over the nodes.  The n^3 blocks KE_s
// are the same for every element; they live in shared memory as packed upper
// triangles (each stored entry feeds two FMAs).  A persistent CTA walks
// element bricks of BX x BY x BZ: it stages the brick's nodal values in
// shared memory, each thread forms one element's 24 outputs, the outputs are
// summed into a shared node brick in 8 parity colours (elements of one colour
// share no node), and the brick is written back with plain stores for nodes
// only this brick touches and atomics on the brick faces.
#include <cuda_bf16.h>

#include "tosp_internal.h"

namespace tosp {

template <typename T> __device__ __forceinline__ T to_t(double v) { return (T)v; }
__device__ __forceinline__ float wval(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ double wval(double v) { return v; }
__device__ __forceinline__ float wval(float v) { return v; }

__device__ __forceinline__ void atomic_add(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(float *p, float v) { atomicAdd(p, v); }

template <typename T, typename TW, int N, bool DIAG>
__global__ void __launch_bounds__(BRICK_ELEMS)
k_fine_apply(const T *__restrict__ x, T *__restrict__ y, const TW *__restrict__ w,
             const uint8_t *__restrict__ freemask, const T *__restrict__ kepack, FineGeom fg) {
    constexpr int NS = N * N * N;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *ke = reinterpret_cast<T *>(smem_raw);             // NS * 300
    T *xs = ke + NS * KE_PACK;                             // BRICK_NODES * 3
    T *ys = xs + BRICK_NODES * 3;                          // BRICK_NODES * 3
    const int tid = threadIdx.x;
    for (int i = tid; i < NS * KE_PACK; i += BRICK_ELEMS) ke[i] = kepack[i];

    const Grid &g = fg.g;
    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    const int color = (lx & 1) | ((ly & 1) << 1) | ((lz & 1) << 2);

    for (int64_t brick = blockIdx.x; brick < fg.nbricks; brick += gridDim.x) {
        const int bby = (int)(brick % fg.nby);
        const int bbx = (int)((brick / fg.nby) % fg.nbx);
        const int bbz = (int)(brick / ((int64_t)fg.nby * fg.nbx));
        const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
        __syncthreads();   // previous brick done with xs/ys (and ke loaded)
        for (int i = tid; i < BRICK_NODES * 3; i += BRICK_ELEMS) {
            const int ln = i / 3, c = i - 3 * ln;
            const int ny_ = ln % NBY, nx_ = (ln / NBY) % NBX, nz_ = ln / (NBY * NBX);
            const int gx = ex0 + nx_, gy = ey0 + ny_, gz = ez0 + nz_;
            T v = T(0);
            if (!DIAG && gx < g.nx && gy < g.ny && gz < g.nz)
                v = x[3 * (((int64_t)gz * g.nx + gx) * g.ny + gy) + c];
            xs[i] = v;
            ys[i] = T(0);
        }
        __syncthreads();

        const int ex = ex0 + lx, ey = ey0 + ly, ez = ez0 + lz;
        const bool valid = ex < g.nelx && ey < g.nely && ez < g.nelz;
        T acc[24];
#pragma unroll
        for (int i = 0; i < 24; ++i) acc[i] = T(0);
        if (valid) {
            T u[24];
            if (!DIAG) {
#pragma unroll
                for (int a = 0; a < 8; ++a) {
                    const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
                    const int ln = ((lz + dz) * NBX + (lx + dx)) * NBY + (ly + dy);
#pragma unroll
                    for (int c = 0; c < 3; ++c) u[3 * a + c] = xs[3 * ln + c];
                }
            }
#pragma unroll 1
            for (int s = 0; s < NS; ++s) {
                const int sy = s % N, sx = (s / N) % N, sz = s / (N * N);
                const int64_t di = ((int64_t)(ez * N + sz) * fg.nelx_d + (ex * N + sx)) * fg.nely_d + (ey * N + sy);
                const T ws = (T)wval(w[di]);
                const T *k = ke + s * KE_PACK;
                if (DIAG) {
                    int t = 0;
#pragma unroll
                    for (int i = 0; i < 24; ++i) {
                        acc[i] += ws * k[t];
                        t += 24 - i;
                    }
                } else {
                    T wu[24];
#pragma unroll
                    for (int i = 0; i < 24; ++i) wu[i] = ws * u[i];
                    int t = 0;
#pragma unroll
                    for (int i = 0; i < 24; ++i) {
                        acc[i] += k[t] * wu[i];
                        ++t;
#pragma unroll
                        for (int j = i + 1; j < 24; ++j) {
                            const T kij = k[t++];
                            acc[i] += kij * wu[j];
                            acc[j] += kij * wu[i];
                        }
                    }
                }
            }
        }
        // colour-ordered accumulation into the node brick
#pragma unroll 1
        for (int col = 0; col < 8; ++col) {
            if (valid && col == color) {
#pragma unroll
                for (int a = 0; a < 8; ++a) {
                    const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
                    const int ln = ((lz + dz) * NBX + (lx + dx)) * NBY + (ly + dy);
#pragma unroll
                    for (int c = 0; c < 3; ++c) ys[3 * ln + c] += acc[3 * a + c];
                }
            }
            __syncthreads();
        }
        for (int i = tid; i < BRICK_NODES * 3; i += BRICK_ELEMS) {
            const int ln = i / 3, c = i - 3 * ln;
            const int ny_ = ln % NBY, nx_ = (ln / NBY) % NBX, nz_ = ln / (NBY * NBX);
            const int gx = ex0 + nx_, gy = ey0 + ny_, gz = ez0 + nz_;
            if (gx < g.nx && gy < g.ny && gz < g.nz) {
                const int64_t dof = 3 * (((int64_t)gz * g.nx + gx) * g.ny + gy) + c;
                if (freemask[dof]) {
                    const bool inner = nx_ > 0 && nx_ < BX && ny_ > 0 && ny_ < BY && nz_ > 0 && nz_ < BZ;
                    if (inner) y[dof] = ys[i];
                    else atomic_add(&y[dof], ys[i]);
                }
            }
        }
    }
}

static int g_num_sms = 0;
static int num_sms() {
    if (!g_num_sms) {
        int dev;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return g_num_sms;
}

template <typename T, typename TW, int N, bool DIAG>
static void launch_fine_t(const T *x, T *y, const TW *w, const uint8_t *fm, const T *kp, const FineGeom &fg,
                          cudaStream_t st) {
    constexpr int NS = N * N * N;
    const size_t smem = sizeof(T) * (NS * KE_PACK + 2 * BRICK_NODES * 3);
    auto kern = k_fine_apply<T, TW, N, DIAG>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = true;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BRICK_ELEMS, smem);
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)per_sm * num_sms();
    if (grid > fg.nbricks) grid = fg.nbricks;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, BRICK_ELEMS, smem, st>>>(x, y, w, fm, kp, fg); count_launch();
}

template <typename T, typename TW>
void launch_fine_apply(const T *x, T *y, const TW *w, const uint8_t *freemask, const T *kepack,
                       const FineGeom &fg, int n, bool diag_only, cudaStream_t st) {
    if (n == 1) {
        if (diag_only) launch_fine_t<T, TW, 1, true>(x, y, w, freemask, kepack, fg, st);
        else launch_fine_t<T, TW, 1, false>(x, y, w, freemask, kepack, fg, st);
    } else if (n == 2) {
        if (diag_only) launch_fine_t<T, TW, 2, true>(x, y, w, freemask, kepack, fg, st);
        else launch_fine_t<T, TW, 2, false>(x, y, w, freemask, kepack, fg, st);
    } else {
        if (diag_only) launch_fine_t<T, TW, 3, true>(x, y, w, freemask, kepack, fg, st);
        else launch_fine_t<T, TW, 3, false>(x, y, w, freemask, kepack, fg, st);
    }
}

template void launch_fine_apply<double, double>(const double *, double *, const double *, const uint8_t *,
                                                const double *, const FineGeom &, int, bool, cudaStream_t);
template void launch_fine_apply<float, __nv_bfloat16>(const float *, float *, const __nv_bfloat16 *,
                                                      const uint8_t *, const float *, const FineGeom &, int,
                                                      bool, cudaStream_t);

// ---------------------------------------------------------------------------
// SIMP factors emin + (E - emin) rho^p (I/GlobalStiffMatrix.m:49,
// I/WOK/KelemProd.m:74).  Integer p uses repeated products.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double powp(double x, double p) {
    if (p == 1.0) return x;
    if (p == 2.0) return x * x;
    if (p == 3.0) return x * x * x;
    return pow(x, p);
}

__global__ void k_simp(const double *rho, double *w64, __nv_bfloat16 *wbf, int64_t n, double p, double emin,
                       double E) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double w = emin + (E - emin) * powp(rho[i], p);
        w64[i] = w;
        if (wbf) wbf[i] = __double2bfloat16(w);
    }
}

void launch_simp(const double *rho, double *w64, __nv_bfloat16 *wbf, int64_t n, double p, double emin, double E,
                 cudaStream_t st) {
    int64_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_simp<<<(unsigned)blocks, 256, 0, st>>>(rho, w64, wbf, n, p, emin, E); count_launch();
}

// ---------------------------------------------------------------------------
// Sensitivities (I/Grad.m:24-49, mr.interp = false):
//   g0(v_s) = -p rho_s^(p-1) (E-emin) u_e' KE_s u_e  for e in freeDensG.
// One thread per displacement element; KE_s packed in shared memory.
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(128)
k_grad(const double *__restrict__ u, const double *__restrict__ rho, const uint8_t *__restrict__ free_elem,
       const double *__restrict__ kepack, double *__restrict__ g0, FineGeom fg, double p, double emin, double E) {
    constexpr int NS = N * N * N;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *ke = reinterpret_cast<double *>(smem_raw);
    for (int i = threadIdx.x; i < NS * KE_PACK; i += blockDim.x) ke[i] = kepack[i];
    __syncthreads();
    const Grid &g = fg.g;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < g.nelem;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int ey = (int)(e % g.nely), ex = (int)((e / g.nely) % g.nelx), ez = (int)(e / ((int64_t)g.nely * g.nelx));
        const bool fr = free_elem[e] != 0;
        double ue[24];
        if (fr) {
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
                const int64_t node = ((int64_t)(ez + dz) * g.nx + (ex + dx)) * g.ny + (ey + dy);
#pragma unroll
                for (int c = 0; c < 3; ++c) ue[3 * a + c] = u[3 * node + c];
            }
        }
#pragma unroll 1
        for (int s = 0; s < NS; ++s) {
            const int sy = s % N, sx = (s / N) % N, sz = s / (N * N);
            const int64_t di = ((int64_t)(ez * N + sz) * fg.nelx_d + (ex * N + sx)) * fg.nely_d + (ey * N + sy);
            double out = 0.0;
            if (fr) {
                const double *k = ke + s * KE_PACK;
                double q = 0.0;
                int t = 0;
#pragma unroll
                for (int i = 0; i < 24; ++i) {
                    double row = 0.5 * k[t++] * ue[i];
#pragma unroll
                    for (int j = i + 1; j < 24; ++j) row += k[t++] * ue[j];
                    q += row * ue[i];
                }
                q *= 2.0;
                const double xs = rho[di];
                out = -p * powp(xs, p - 1.0) * (E - emin) * q;
            }
            g0[di] = out;
        }
    }
}

void launch_grad(const double *u, const double *rho, const uint8_t *free_elem, const double *kepack, double *g0,
                 const FineGeom &fg, int n, double p, double emin, double E, cudaStream_t st) {
    const int ns = n * n * n;
    const size_t smem = sizeof(double) * ns * KE_PACK;
    int64_t blocks = (fg.g.nelem + 127) / 128;
    if (blocks > 8 * num_sms()) blocks = 8 * num_sms();
    if (blocks < 1) blocks = 1;
    if (n == 1) {
        k_grad<1><<<(unsigned)blocks, 128, smem, st>>>(u, rho, free_elem, kepack, g0, fg, p, emin, E); count_launch();
    } else if (n == 2) {
        k_grad<2><<<(unsigned)blocks, 128, smem, st>>>(u, rho, free_elem, kepack, g0, fg, p, emin, E); count_launch();
    } else {
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_grad<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            attr = true;
        }
        k_grad<3><<<(unsigned)blocks, 128, smem, st>>>(u, rho, free_elem, kepack, g0, fg, p, emin, E); count_launch();
    }
}

}  // namespace tosp
