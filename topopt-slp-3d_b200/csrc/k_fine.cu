// Fine-level multiresolution hex8 operator, its diagonal, the SIMP factors
// and the compliance sensitivities.
//
// Operator (I/WOK/KelemProd.m:57-100): y_e = K_e u_e with
// K_e = sum_s w_s KE_s for every displacement element e, scatter-added over
// the nodes.  The n^3 blocks KE_s are the same for every element; they live in
// shared memory pair-major (for each upper-triangle entry (i,j) the n^3 block
// values are contiguous), so each thread forms one entry of its K_e with
// vector loads and n^3 FMAs and uses it twice (y_i += k u_j, y_j += k u_i):
// 300 (n^3 + 2) FMAs per element instead of 600 n^3 for block-by-block
// products.  A persistent CTA walks
// element bricks of BX x BY x BZ: it stages the brick's nodal values in
// shared memory, each thread forms one element's 24 outputs, the outputs are
// summed into the brick's nodes corner by corner (brick.cuh), and the result
// is written with plain stores for nodes only this brick touches and atomics
// on the brick faces.
#include <cuda_bf16.h>

#include <cstring>
#include <type_traits>
#include <utility>

#include "brick.cuh"
#include "mr2_pattern.h"
#include "tosp_internal.h"

namespace tosp {

__device__ __forceinline__ float wval(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ double wval(double v) { return v; }
__device__ __forceinline__ float wval(float v) { return v; }

template <typename T> struct Vec;
template <> struct Vec<float> { using type = float4; static constexpr int W = 4; };
template <> struct Vec<double> { using type = double2; static constexpr int W = 2; };

__device__ __forceinline__ float dot_vec(const float4 v, const float *w) { return w[0] * v.x + w[1] * v.y + w[2] * v.z + w[3] * v.w; }
__device__ __forceinline__ double dot_vec(const double2 v, const double *w) { return w[0] * v.x + w[1] * v.y; }

// One packed entry t of the element matrix: k = sum_s w_s KE_s[i][j], then
// y_i += k u_j and (for i != j) y_j += k u_i.  Entries are visited diagonal
// by diagonal (pair_i/pair_j) so consecutive updates hit different
// accumulators.
template <typename T, int NSP, int t>
__device__ __forceinline__ void pair_step(const T *__restrict__ kt, const T (&w)[NSP], const T (&u)[24],
                                          T (&acc)[24]) {
    constexpr int i = pair_i(t), j = pair_j(t);
    T k;
    if constexpr (NSP == 1) {
        k = w[0] * kt[t];
    } else {
        // two independent partial sums halve the dependent FMA chain
        constexpr int W = Vec<T>::W, NV = NSP / W;
        const typename Vec<T>::type *kv = reinterpret_cast<const typename Vec<T>::type *>(kt + t * NSP);
        T k0 = dot_vec(kv[0], w);
        if constexpr (NV > 1) {
            T k1 = dot_vec(kv[1], w + W);
#pragma unroll
            for (int q = 2; q < NV; ++q) {
                if (q % 2 == 0) k0 += dot_vec(kv[q], w + q * W);
                else k1 += dot_vec(kv[q], w + q * W);
            }
            k = k0 + k1;
        } else {
            k = k0;
        }
    }
    if constexpr (i == j) {
        acc[i] += k * u[i];
    } else {
        acc[i] += k * u[j];
        acc[j] += k * u[i];
    }
}

template <typename T, int NSP, int... Ts>
__device__ __forceinline__ void all_pairs(const T *__restrict__ kt, const T (&w)[NSP], const T (&u)[24], T (&acc)[24],
                                          std::integer_sequence<int, Ts...>) {
    (pair_step<T, NSP, Ts>(kt, w, u, acc), ...);
}

// --- MR factor 2: Walsh-Hadamard form -------------------------------------
// K_e = sum_b what_b Khat_b with what = H w (8-point Walsh-Hadamard transform
// of the sub-cube factors) and Khat = H KE / 8; mr2_mask marks the non-zero
// modes of each entry (mr2_mask; structural zeros skipped at compile time: 1548 instead
// of 2400 FMAs).  Entry t's non-zero values are contiguous in shared memory,
// padded to the vector width.
__host__ __device__ constexpr int mr2_nz(int t) {
    int c = 0;
    for (int m = 0; m < 8; ++m) c += (mr2_mask(t) >> m) & 1;
    return c;
}
__host__ __device__ constexpr int mr2_off(int t, int w) {
    int o = 0;
    for (int q = 0; q < t; ++q) o += (mr2_nz(q) + w - 1) / w * w;
    return o;
}

template <typename T, int t>
__device__ __forceinline__ void pair_step_mr2(const T *__restrict__ kt, const T (&wh)[8], const T (&u)[24],
                                              T (&acc)[24]) {
    constexpr int i = pair_i(t), j = pair_j(t);
    constexpr int W = Vec<T>::W, NZ = mr2_nz(t), NV = (NZ + W - 1) / W;
    constexpr unsigned MASK = mr2_mask(t);
    const typename Vec<T>::type *kv = reinterpret_cast<const typename Vec<T>::type *>(kt + mr2_off(t, W));
    T vals[NV * W];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        const typename Vec<T>::type v = kv[q];
        if constexpr (W == 4) {
            vals[4 * q] = v.x; vals[4 * q + 1] = v.y; vals[4 * q + 2] = v.z; vals[4 * q + 3] = v.w;
        } else {
            vals[2 * q] = v.x; vals[2 * q + 1] = v.y;
        }
    }
    // two partial sums over the set modes (shorter dependent chains)
    T k0 = T(0), k1 = T(0);
    int idx = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        if ((MASK >> m) & 1) {
            if (idx & 1) k1 += wh[m] * vals[idx];
            else k0 += wh[m] * vals[idx];
            ++idx;
        }
    }
    const T k = k0 + k1;
    if constexpr (i == j) {
        acc[i] += k * u[i];
    } else {
        acc[i] += k * u[j];
        acc[j] += k * u[i];
    }
}

template <typename T, int... Ts>
__device__ __forceinline__ void all_pairs_mr2(const T *__restrict__ kt, const T (&wh)[8], const T (&u)[24],
                                              T (&acc)[24], std::integer_sequence<int, Ts...>) {
    (pair_step_mr2<T, Ts>(kt, wh, u, acc), ...);
}

// MR-2 Walsh-Hadamard coefficients as a kernel parameter (12 384 bytes, in
// the constant bank): every coefficient index is a compile-time constant, so
// the FMAs take them as constant-bank operands and no shared-memory load is
// issued for them.  Entry t's non-zero modes start at mr2_off(t, 1).
struct Mr2Table {
    double v[kMr2Nonzeros];
};

template <int t>
__device__ __forceinline__ void pair_step_mr2c(const Mr2Table &kt, const double (&wh)[8], const double (&u)[24],
                                               double (&acc)[24]) {
    constexpr int i = pair_i(t), j = pair_j(t);
    constexpr unsigned MASK = mr2_mask(t);
    constexpr int OFF = mr2_off(t, 1);
    double k0 = 0.0, k1 = 0.0;
    int idx = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        if ((MASK >> m) & 1) {
            if (idx & 1) k1 = fma(wh[m], kt.v[OFF + idx], k1);
            else k0 = fma(wh[m], kt.v[OFF + idx], k0);
            ++idx;
        }
    }
    const double k = k0 + k1;
    if constexpr (i == j) {
        acc[i] = fma(k, u[i], acc[i]);
    } else {
        acc[i] = fma(k, u[j], acc[i]);
        acc[j] = fma(k, u[i], acc[j]);
    }
}

template <int... Ts>
__device__ __forceinline__ void all_pairs_mr2c(const Mr2Table &kt, const double (&wh)[8], const double (&u)[24],
                                               double (&acc)[24], std::integer_sequence<int, Ts...>) {
    (pair_step_mr2c<Ts>(kt, wh, u, acc), ...);
}

template <typename T, int N> struct FineShape {
    static constexpr int NS = N * N * N;
    static constexpr int NSP = (N == 1) ? 1 : (NS + Vec<T>::W - 1) / Vec<T>::W * Vec<T>::W;
    // shared-memory length of the block table
    static constexpr int KT_LEN = (N == 2) ? mr2_off(KE_PACK, Vec<T>::W) : KE_PACK * NSP;
};

// Operator: persistent CTAs over element bricks; see the file header.  Used
// for the FP32/BF16 V-cycle operator (MR 1 and 3) and FP64 with MR 3.
template <typename T, typename TW, int N>
__global__ void __launch_bounds__(BRICK_ELEMS)
k_fine_apply(const T *__restrict__ x, T *__restrict__ y, const TW *__restrict__ w,
             const uint8_t *__restrict__ freemask, const T *__restrict__ ktg, FineGeom fg) {
    constexpr int NS = FineShape<T, N>::NS, NSP = FineShape<T, N>::NSP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *kt = reinterpret_cast<T *>(smem_raw);               // KE_PACK * NSP (pair-major)
    T *xs = kt + FineShape<T, N>::KT_LEN;                   // BRICK_NODES * 3
    T *ys = xs + BRICK_NODES * 3;                           // BRICK_NODES * 3 node sums
    const int tid = threadIdx.x;
    for (int i = tid; i < FineShape<T, N>::KT_LEN; i += BRICK_ELEMS) kt[i] = ktg[i];

    const Grid &g = fg.g;
    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);

    for (int64_t brick = blockIdx.x; brick < fg.nbricks; brick += gridDim.x) {
        int bbx, bby, bbz;
        brick_xyz(brick, fg, bbx, bby, bbz);
        const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
        __syncthreads();   // previous brick done with xs/ys (and kt loaded)
        for (int i = tid; i < BRICK_NODES * 3; i += BRICK_ELEMS) {
            const int ln = i / 3, c = i - 3 * ln;
            const int ny_ = ln % NBY, nx_ = (ln / NBY) % NBX, nz_ = ln / (NBY * NBX);
            const int gx = ex0 + nx_, gy = ey0 + ny_, gz = ez0 + nz_;
            T v = T(0);
            if (gx < g.nx && gy < g.ny && gz < g.nz) v = x[3 * (((int64_t)gz * g.nx + gx) * g.ny + gy) + c];
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
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
                const int ln = ((lz + dz) * NBX + (lx + dx)) * NBY + (ly + dy);
#pragma unroll
                for (int c = 0; c < 3; ++c) u[3 * a + c] = xs[3 * ln + c];
            }
            T wv[NSP];
#pragma unroll
            for (int s = 0; s < NSP; ++s) {
                if (s < NS) {
                    const int sy = s % N, sx = (s / N) % N, sz = s / (N * N);
                    wv[s] = (T)wval(w[((int64_t)(ez * N + sz) * fg.nelx_d + (ex * N + sx)) * fg.nely_d + (ey * N + sy)]);
                } else {
                    wv[s] = T(0);
                }
            }
            if constexpr (N == 2) {
                // 8-point Walsh-Hadamard transform of the sub-cube factors
                T wh[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) wh[q] = wv[q];
#pragma unroll
                for (int bit = 1; bit < 8; bit <<= 1) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (!(q & bit)) {
                            const T a = wh[q], b = wh[q | bit];
                            wh[q] = a + b;
                            wh[q | bit] = a - b;
                        }
                    }
                }
                all_pairs_mr2<T>(kt, wh, u, acc, std::make_integer_sequence<int, KE_PACK>{});
            } else {
                all_pairs<T, NSP>(kt, wv, u, acc, std::make_integer_sequence<int, KE_PACK>{});
            }
        }
        brick_accumulate(ys, acc, valid, brick_base_node(tid));
        brick_writeout(ys, y, freemask, g, ex0, ey0, ez0, tid);
    }
}

// FP64 operator for MR factor 1 and 2 with staged inputs: the next brick's
// nodal values and SIMP factors are copied into the second half of double
// buffers with cp.async while the current brick computes, so the global-load
// latency is hidden behind the element-matrix arithmetic (three CTAs per SM
// leave too few warps to hide it otherwise).  Factors are stored s-major
// (ws[s * BRICK_ELEMS + element]) so that both the copies and the reads are
// conflict-free.  Node offsets come from the per-CTA slot table.
__device__ __forceinline__ void cp_async8(void *dst, const void *src, int nbytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(nbytes)
                 : "memory");
}

template <int N>
struct StagedLayout {
    static constexpr int NS = N * N * N;
    static constexpr int KT = (FineShape<double, N>::KT_LEN + 1) / 2 * 2;   // doubles, 16-byte multiple
    static constexpr int XS = BRICK_NODES * 4;                               // nodes padded to 4 values
    static constexpr int SLOTS = (BRICK_SLOTS + 1) / 2 * 2;                  // slot table length
    static constexpr size_t OFF_XS = sizeof(double) * KT;
    static constexpr size_t OFF_YS = OFF_XS + sizeof(double) * 2 * XS;
    static constexpr size_t OFF_WS = OFF_YS + sizeof(double) * XS;
    static constexpr size_t OFF_REL = OFF_WS + sizeof(double) * 2 * NS * BRICK_ELEMS;
    static constexpr size_t OFF_PK = OFF_REL + sizeof(int32_t) * SLOTS;
    static constexpr size_t BYTES = OFF_PK + sizeof(uint16_t) * SLOTS;
};

template <int N>
__device__ __forceinline__ void stage_brick64(int64_t brick, int buf, const double *__restrict__ x,
                                              const double *__restrict__ w, const FineGeom &fg, unsigned char *smem,
                                              const int32_t *rel, const uint16_t *pk, int tid) {
    using L = StagedLayout<N>;
    const Grid &g = fg.g;
    int bbx, bby, bbz;
    brick_xyz(brick, fg, bbx, bby, bbz);
    const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
    double *xs = reinterpret_cast<double *>(smem + L::OFF_XS) + buf * L::XS;
    const double *xb = x + brick_base_dof(ex0, ey0, ez0, g);
    // node by node: three values into a node's 4-value slot
    if (brick_interior(ex0, ey0, ez0, g)) {
        for (int ln = tid; ln < BRICK_NODES; ln += BRICK_ELEMS) {
            const double *src = xb + rel[3 * ln];
            double *dst = xs + 4 * ln;
            cp_async8(dst, src, 8);
            cp_async8(dst + 1, src + 1, 8);
            cp_async8(dst + 2, src + 2, 8);
        }
    } else {
        for (int ln = tid; ln < BRICK_NODES; ln += BRICK_ELEMS) {
            const bool in = brick_slot_in(pk[3 * ln], ex0, ey0, ez0, g);
            const double *src = in ? xb + rel[3 * ln] : x;
            double *dst = xs + 4 * ln;
            cp_async8(dst, src, in ? 8 : 0);
            cp_async8(dst + 1, in ? src + 1 : x, in ? 8 : 0);
            cp_async8(dst + 2, in ? src + 2 : x, in ? 8 : 0);
        }
    }
    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    const int ex = ex0 + lx, ey = ey0 + ly, ez = ez0 + lz;
    const bool valid = ex < g.nelx && ey < g.nely && ez < g.nelz;
    double *ws = reinterpret_cast<double *>(smem + L::OFF_WS) + buf * L::NS * BRICK_ELEMS;
#pragma unroll
    for (int s = 0; s < L::NS; ++s) {
        const int sy = s % N, sx = (s / N) % N, sz = s / (N * N);
        const double *src =
            valid ? w + ((int64_t)(ez * N + sz) * fg.nelx_d + (ex * N + sx)) * fg.nely_d + (ey * N + sy) : w;
        cp_async8(ws + s * BRICK_ELEMS + tid, src, valid ? 8 : 0);
    }
}

struct NoTable {};

template <int N, typename KP>
__global__ void __launch_bounds__(BRICK_ELEMS, N == 2 ? 3 : 1)
k_fine_apply64(const double *__restrict__ x, double *__restrict__ y, const double *__restrict__ w,
               const uint8_t *__restrict__ freemask, const double *__restrict__ ktg, FineGeom fg,
               const __grid_constant__ KP ktc) {
    constexpr bool CONST_KE = std::is_same<KP, Mr2Table>::value;
    using L = StagedLayout<N>;
    constexpr int NS = L::NS, NSP = FineShape<double, N>::NSP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *kt = reinterpret_cast<double *>(smem_raw);
    double *ys = reinterpret_cast<double *>(smem_raw + L::OFF_YS);
    int32_t *rel = reinterpret_cast<int32_t *>(smem_raw + L::OFF_REL);
    uint16_t *pk = reinterpret_cast<uint16_t *>(smem_raw + L::OFF_PK);
    const int tid = threadIdx.x;
    const Grid &g = fg.g;
    if constexpr (!CONST_KE)
        for (int i = tid; i < FineShape<double, N>::KT_LEN; i += BRICK_ELEMS) kt[i] = ktg[i];
    brick_slots_init(rel, pk, g, tid);
    __syncthreads();

    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    const int ln0 = brick_base_node(tid);
    int buf = 0;
    if (blockIdx.x < fg.nbricks) stage_brick64<N>(blockIdx.x, 0, x, w, fg, smem_raw, rel, pk, tid);
    asm volatile("cp.async.commit_group;" ::: "memory");
    for (int64_t brick = blockIdx.x; brick < fg.nbricks; brick += gridDim.x, buf ^= 1) {
        const int64_t next = brick + gridDim.x;
        const bool chk = brick_check_fixed(brick, fg);
        if (next < fg.nbricks) stage_brick64<N>(next, buf ^ 1, x, w, fg, smem_raw, rel, pk, tid);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();   // this brick's inputs landed; the previous write-out is done
        for (int i = tid; i < 2 * BRICK_NODES; i += BRICK_ELEMS)
            reinterpret_cast<double2 *>(ys)[i] = make_double2(0.0, 0.0);

        int bbx, bby, bbz;
        brick_xyz(brick, fg, bbx, bby, bbz);
        const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
        const bool valid = ex0 + lx < g.nelx && ey0 + ly < g.nely && ez0 + lz < g.nelz;
        const double *xs = reinterpret_cast<const double *>(smem_raw + L::OFF_XS) + buf * L::XS;
        const double *ws = reinterpret_cast<const double *>(smem_raw + L::OFF_WS) + buf * NS * BRICK_ELEMS;
        double acc[24];
#pragma unroll
        for (int i = 0; i < 24; ++i) acc[i] = 0.0;
        if (valid) {
            double u[24];
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
                const int ln = ln0 + (dz * NBX + dx) * NBY + dy;
                const double2 v01 = reinterpret_cast<const double2 *>(xs)[2 * ln];
                u[3 * a] = v01.x;
                u[3 * a + 1] = v01.y;
                u[3 * a + 2] = xs[4 * ln + 2];
            }
            if constexpr (N == 2) {
                double wh[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) wh[q] = ws[q * BRICK_ELEMS + tid];
#pragma unroll
                for (int bit = 1; bit < 8; bit <<= 1) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (!(q & bit)) {
                            const double a = wh[q], b = wh[q | bit];
                            wh[q] = a + b;
                            wh[q | bit] = a - b;
                        }
                    }
                }
                if constexpr (CONST_KE)
                    all_pairs_mr2c(ktc, wh, u, acc, std::make_integer_sequence<int, KE_PACK>{});
                else
                    all_pairs_mr2<double>(kt, wh, u, acc, std::make_integer_sequence<int, KE_PACK>{});
            } else {
                double wv[NSP];
#pragma unroll
                for (int q = 0; q < NSP; ++q) wv[q] = q < NS ? ws[q * BRICK_ELEMS + tid] : 0.0;
                all_pairs<double, NSP>(kt, wv, u, acc, std::make_integer_sequence<int, KE_PACK>{});
            }
        }
        __syncthreads();   // ys cleared by every thread
        brick_accumulate_pad(ys, acc, valid, ln0);
        brick_writeout_nodes<double>(ys, y, freemask, g, ex0, ey0, ez0, rel, pk, tid, chk);
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Diagonal of K(w): one thread per element, atomics (setup only).  Reads the
// row-major packed blocks ke[s*300 + rowmajor(i,i)].
template <int N>
__global__ void k_fine_diag(double *__restrict__ y, const double *__restrict__ w, const uint8_t *__restrict__ freemask,
                            const double *__restrict__ ke, FineGeom fg) {
    constexpr int NS = N * N * N;
    const Grid &g = fg.g;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < g.nelem;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int ey = (int)(e % g.nely), ex = (int)((e / g.nely) % g.nelx), ez = (int)(e / ((int64_t)g.nely * g.nelx));
        for (int i = 0; i < 24; ++i) {
            const int t = pair_rowmajor(i, i);
            double d = 0.0;
            for (int s = 0; s < NS; ++s) {
                const int sy = s % N, sx = (s / N) % N, sz = s / (N * N);
                d += w[((int64_t)(ez * N + sz) * fg.nelx_d + (ex * N + sx)) * fg.nely_d + (ey * N + sy)] *
                     ke[s * KE_PACK + t];
            }
            const int a = i / 3, c = i % 3;
            const int64_t node = ((int64_t)(ez + ((a >> 2) & 1)) * g.nx + (ex + ((a >> 1) & 1))) * g.ny + (ey + (a & 1));
            if (freemask[3 * node + c]) atomicAdd(&y[3 * node + c], d);
        }
    }
}

static int num_sms() {
    static int n = 0;
    if (!n) {
        int dev;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    }
    return n;
}

int fine_nsp(int n, int elem_bytes) {
    if (n == 1) return 1;
    const int ns = n * n * n, vw = elem_bytes == 8 ? 2 : 4;
    return (ns + vw - 1) / vw * vw;
}

// Host layout of the operator's block table (see FineShape::KT_LEN).
void fine_block_table(const std::vector<double> &packed_rowmajor, int n, int elem_bytes, std::vector<double> &kt) {
    const int ns = n * n * n;
    if (n == 2) {
        const int w = elem_bytes == 8 ? 2 : 4;
        kt.assign((size_t)mr2_off(KE_PACK, w), 0.0);
        for (int t = 0; t < KE_PACK; ++t) {
            const int rm = pair_rowmajor(pair_i(t), pair_j(t));
            int o = mr2_off(t, w);
            for (int m = 0; m < 8; ++m) {
                if (!((mr2_mask(t) >> m) & 1)) continue;
                double v = 0.0;
                for (int q = 0; q < 8; ++q) {
                    const int sign = (__builtin_popcount(m & q) & 1) ? -1 : 1;
                    v += sign * packed_rowmajor[(size_t)q * KE_PACK + rm];
                }
                kt[o++] = v / 8.0;
            }
        }
        return;
    }
    const int nsp = fine_nsp(n, elem_bytes);
    kt.assign((size_t)KE_PACK * nsp, 0.0);
    for (int t = 0; t < KE_PACK; ++t) {
        const int rm = pair_rowmajor(pair_i(t), pair_j(t));
        for (int s = 0; s < ns; ++s) kt[(size_t)t * nsp + s] = packed_rowmajor[(size_t)s * KE_PACK + rm];
    }
}

template <typename T, typename TW, int N>
static void launch_fine_t(const T *x, T *y, const TW *w, const uint8_t *fm, const T *kt, const FineGeom &fg,
                          cudaStream_t st) {
    const size_t smem = sizeof(T) * (FineShape<T, N>::KT_LEN + 2 * BRICK_NODES * 3);
    auto kern = k_fine_apply<T, TW, N>;
    static int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_dev = dev;
    }
    static int per_sm = 0;
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BRICK_ELEMS, smem);
        if (per_sm < 1) per_sm = 1;
    }
    int64_t grid = (int64_t)per_sm * num_sms();
    if (grid > fg.nbricks) grid = fg.nbricks;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, BRICK_ELEMS, smem, st>>>(x, y, w, fm, kt, fg); count_launch();
}

template <int N, typename KP>
static void launch_fine64_staged(const double *x, double *y, const double *w, const uint8_t *fm, const double *kt,
                                 const FineGeom &fg, cudaStream_t st, const KP &ktc) {
    const size_t smem = StagedLayout<N>::BYTES;
    auto kern = k_fine_apply64<N, KP>;
    static int attr_dev = -1, per_sm = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BRICK_ELEMS, smem);
        if (per_sm < 1) per_sm = 1;
        attr_dev = dev;
    }
    int64_t grid = (int64_t)per_sm * num_sms();
    if (grid > fg.nbricks) grid = fg.nbricks;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, BRICK_ELEMS, smem, st>>>(x, y, w, fm, kt, fg, ktc); count_launch();
}

// FP64 MR-2 operator with the coefficients passed in the launch (ktab: the
// kMr2Nonzeros non-zero Walsh-Hadamard coefficients, host memory).
void launch_fine_apply64_const(const double *x, double *y, const double *w, const uint8_t *freemask,
                               const double *ktab, const FineGeom &fg, cudaStream_t st) {
    Mr2Table t;
    memcpy(t.v, ktab, sizeof(t.v));
    launch_fine64_staged<2, Mr2Table>(x, y, w, freemask, nullptr, fg, st, t);
}

// The non-zero coefficients of the shared-memory table (padded to the vector
// width `elem_bytes`) in the unpadded order of Mr2Table.
void fine_mr2_const_table(const std::vector<double> &kt_padded, int elem_bytes, std::vector<double> &out) {
    const int wv = elem_bytes == 8 ? 2 : 4;
    out.clear();
    for (int t = 0; t < KE_PACK; ++t)
        for (int k = 0; k < mr2_nz(t); ++k) out.push_back(kt_padded[(size_t)mr2_off(t, wv) + k]);
}

template <typename T, typename TW>
void launch_fine_apply(const T *x, T *y, const TW *w, const uint8_t *freemask, const T *kt, const FineGeom &fg, int n,
                       cudaStream_t st) {
    if constexpr (sizeof(T) == 8) {
        if (n == 1) return launch_fine64_staged<1>(x, y, w, freemask, kt, fg, st, NoTable{});
        if (n == 2) return launch_fine64_staged<2>(x, y, w, freemask, kt, fg, st, NoTable{});
    }
    if (n == 1) launch_fine_t<T, TW, 1>(x, y, w, freemask, kt, fg, st);
    else if (n == 2) launch_fine_t<T, TW, 2>(x, y, w, freemask, kt, fg, st);
    else launch_fine_t<T, TW, 3>(x, y, w, freemask, kt, fg, st);
}

template void launch_fine_apply<double, double>(const double *, double *, const double *, const uint8_t *,
                                                const double *, const FineGeom &, int, cudaStream_t);
template void launch_fine_apply<float, __nv_bfloat16>(const float *, float *, const __nv_bfloat16 *, const uint8_t *,
                                                      const float *, const FineGeom &, int, cudaStream_t);

void launch_fine_diag(double *y, const double *w, const uint8_t *freemask, const double *ke64, const FineGeom &fg,
                      int n, cudaStream_t st) {
    int64_t blocks = (fg.g.nelem + 255) / 256;
    if (blocks > 16 * num_sms()) blocks = 16 * num_sms();
    if (blocks < 1) blocks = 1;
    if (n == 1) { k_fine_diag<1><<<(unsigned)blocks, 256, 0, st>>>(y, w, freemask, ke64, fg); count_launch(); }
    else if (n == 2) { k_fine_diag<2><<<(unsigned)blocks, 256, 0, st>>>(y, w, freemask, ke64, fg); count_launch(); }
    else { k_fine_diag<3><<<(unsigned)blocks, 256, 0, st>>>(y, w, freemask, ke64, fg); count_launch(); }
}

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

// wq (optional) receives the BF16-rounded factors widened back to FP64, so
// that the mixed V-cycle's Galerkin hierarchy matches its finest operator;
// w32 (optional) the factors rounded to FP32 (the CG's tensor-core product).
__global__ void k_simp(const double *rho, double *w64, __nv_bfloat16 *wbf, double *wq, float *w32, int64_t n,
                       double p, double emin, double E) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double w = emin + (E - emin) * powp(rho[i], p);
        w64[i] = w;
        if (w32) w32[i] = (float)w;
        if (wbf) {
            const __nv_bfloat16 b = __double2bfloat16(w);
            wbf[i] = b;
            if (wq) wq[i] = (double)__bfloat162float(b);
        }
    }
}

void launch_simp(const double *rho, double *w64, __nv_bfloat16 *wbf, double *wq, float *w32, int64_t n, double p,
                 double emin, double E, cudaStream_t st) {
    int64_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_simp<<<(unsigned)blocks, 256, 0, st>>>(rho, w64, wbf, wq, w32, n, p, emin, E); count_launch();
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
