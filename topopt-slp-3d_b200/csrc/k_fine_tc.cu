// Finest-level operator of the mixed-precision V-cycle, MR factor 2, with the
// element-matrix formation on the 5th-generation tensor cores.
//
// y_e = K_e u_e with K_e = sum_s w_s KE_s (I/WOK/KelemProd.m:57-100).  For a
// brick of 128 elements the 300 packed entries of every K_e form one GEMM,
//
//     D[e][t] = sum_k A[e][k] B[t][k],   A[e][8q+s] = w_s(e),
//                                        B[t][8q+s] = piece q of KE_s[t],
//
// with q = 0..2 the three BF16 pieces of each FP64 block value (hi, mid, lo;
// their sum carries 24 significant bits) and k = 24..31 zero.  The BF16 SIMP
// factors are exact in the A operand and every product of two BF16 values is
// exact, so D equals the FP32 formation of the CUDA-core kernel up to the
// order of the FP32 accumulation.  D lands in tensor memory (one lane per
// element, one column per entry); each thread reads its lane back in 32-column
// slices and applies y_i += k u_j, y_j += k u_i on the CUDA cores (576 FMAs per
// element instead of the 2148 of the Walsh-Hadamard CUDA-core formation).
//
// The entries are formed in three column chunks (128, 128, 48) through a
// 128-column tensor-memory allocation, so four CTAs share an SM's 512 columns;
// the dynamic shared memory per CTA is padded so that no fifth CTA can become
// resident and wait for columns.  Brick staging, the per-element output slots
// and the node gather with face atomics are those of the CUDA-core kernel.
// Every wait on the MMA-completion barrier is bounded; a timeout sets *err,
// leaves the brick loop and still frees the tensor memory.
#include <cuda_bf16.h>

#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

#include "tosp_internal.h"

namespace tosp {

namespace {

constexpr int TC_K = 32;                      // 3 BF16 pieces x 8 sub-cubes + 8 zero columns
constexpr int TC_ROWS_B = 304;                // 300 entries padded to a multiple of 16
constexpr int TC_ROW_BYTES = TC_K * 2;        // 64 B per K-major row
constexpr int TC_B_BYTES = TC_ROWS_B * TC_ROW_BYTES;          // 19456
constexpr int TC_A_BYTES = BRICK_ELEMS * TC_ROW_BYTES;        // 8192
constexpr int TC_COLS = 128;                  // tensor-memory columns per CTA
constexpr int TC_CTAS_PER_SM = 4;             // 4 x 128 = 512 columns
constexpr uint32_t TC_WAIT_LIMIT = 1u << 22;  // try_wait rounds before giving up

// Canonical no-swizzle K-major layout: 8-row x 16-byte core matrices, core
// matrices adjacent in K 128 B apart (leading byte offset), 8-row groups
// 512 B apart (stride byte offset).
__host__ __device__ constexpr int tc_offset(int row, int k) {
    return (row >> 3) * 512 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)((128 >> 4) & 0x3FFF) << 16;     // leading byte offset (K direction)
    d |= (uint64_t)((512 >> 4) & 0x3FFF) << 32;     // stride byte offset (M/N direction)
    d |= (uint64_t)1 << 46;                         // descriptor version for sm_100
    return d;                                       // base offset 0, no swizzle
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
    for (uint32_t it = 0; it < TC_WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Entry t (diagonal-major order) of K_e applied to u.
template <int t>
__device__ __forceinline__ void entry_step(float k, const float (&u)[24], float (&acc)[24]) {
    if constexpr (t < KE_PACK) {
        constexpr int i = pair_i(t), j = pair_j(t);
        if constexpr (i == j) {
            acc[i] = fmaf(k, u[i], acc[i]);
        } else {
            acc[i] = fmaf(k, u[j], acc[i]);
            acc[j] = fmaf(k, u[i], acc[j]);
        }
    }
}

template <int T0, int... J>
__device__ __forceinline__ void slice_steps(const uint32_t (&r)[32], const float (&u)[24], float (&acc)[24],
                                            std::integer_sequence<int, J...>) {
    (entry_step<T0 + J>(__uint_as_float(r[J]), u, acc), ...);
}

// Read the chunk's columns of this thread's lane and apply them.
template <int T0, int NC>
__device__ __forceinline__ void consume_chunk(uint32_t tlane, const float (&u)[24], float (&acc)[24]) {
    uint32_t r[32];
    if constexpr (NC >= 32) {
        tmem_ld32(tlane, r);
        slice_steps<T0>(r, u, acc, std::make_integer_sequence<int, 32>{});
        if constexpr (NC > 32) consume_chunk<T0 + 32, NC - 32>(tlane + 32, u, acc);
    } else {
        static_assert(NC == 16, "chunk tails are 16 columns");
        tmem_ld16(tlane, r);
        slice_steps<T0>(r, u, acc, std::make_integer_sequence<int, 16>{});
    }
}

}  // namespace

// Dynamic shared memory: B image, A tile, brick nodes, element output slots;
// padded so that at most four CTAs fit on an SM (228 KB, 1 KB reserved per
// CTA): 4 x 53.1 KB fit, 5 do not.  The MMA operands need 16-byte aligned
// starts; the barrier and the tensor-memory address are static (8-byte
// aligned) shared variables.
constexpr size_t TC_OFF_A = TC_B_BYTES;
constexpr size_t TC_OFF_XS = TC_OFF_A + TC_A_BYTES;
constexpr size_t TC_OFF_EO = TC_OFF_XS + sizeof(float) * ((BRICK_NODES * 3 + 3) / 4 * 4);
constexpr size_t TC_SMEM_USED = TC_OFF_EO + sizeof(float) * 24 * BRICK_ELEMS;
constexpr size_t TC_SMEM = 52 * 1024;
static_assert(TC_OFF_A % 16 == 0 && TC_OFF_XS % 16 == 0 && TC_OFF_EO % 16 == 0, "operand alignment");
static_assert(TC_SMEM_USED <= TC_SMEM, "tensor-core operator shared memory");

__global__ void __launch_bounds__(BRICK_ELEMS, TC_CTAS_PER_SM)
k_fine_apply_tc2(const float *__restrict__ x, float *__restrict__ y, const __nv_bfloat16 *__restrict__ w,
                 const uint8_t *__restrict__ freemask, const uint4 *__restrict__ bimg, FineGeom fg,
                 int *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *bs = smem_raw;                                   // B image (canonical layout)
    unsigned char *as = smem_raw + TC_OFF_A;                        // A tile (canonical layout)
    float *xs = reinterpret_cast<float *>(smem_raw + TC_OFF_XS);    // BRICK_NODES * 3
    float *eo = reinterpret_cast<float *>(smem_raw + TC_OFF_EO);    // 24 * BRICK_ELEMS
    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ __align__(8) uint32_t s_tmem;
    __shared__ int s_fail;
    uint64_t *mbar = &s_mbar;
    uint32_t *tmem_holder = &s_tmem;

    const int tid = threadIdx.x, warp = tid >> 5;
    if (smem_u32(smem_raw) & 15u) {   // operand tiles need 16-byte aligned starts
        if (tid == 0) atomicExch(err, 2);
        return;
    }
    for (int i = tid; i < TC_B_BYTES / 16; i += BRICK_ELEMS) reinterpret_cast<uint4 *>(bs)[i] = bimg[i];
    if (tid == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                     "r"(TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_holder;
    const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);    // this warp's 32 lanes, column 0
    const uint32_t mbar_a = smem_u32(mbar);
    const uint32_t a_base = smem_u32(as), b_base = smem_u32(bs);
    uint32_t phase = 0;

    const Grid &g = fg.g;
    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);

    for (int64_t brick = blockIdx.x; brick < fg.nbricks; brick += gridDim.x) {
        const int bby = (int)(brick % fg.nby);
        const int bbx = (int)((brick / fg.nby) % fg.nbx);
        const int bbz = (int)(brick / ((int64_t)fg.nby * fg.nbx));
        const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
        __syncthreads();   // previous brick done with xs / eo / A
        for (int i = tid; i < BRICK_NODES * 3; i += BRICK_ELEMS) {
            const int ln = i / 3, c = i - 3 * ln;
            const int ny_ = ln % NBY, nx_ = (ln / NBY) % NBX, nz_ = ln / (NBY * NBX);
            const int gx = ex0 + nx_, gy = ey0 + ny_, gz = ez0 + nz_;
            float v = 0.f;
            if (gx < g.nx && gy < g.ny && gz < g.nz) v = x[3 * (((int64_t)gz * g.nx + gx) * g.ny + gy) + c];
            xs[i] = v;
        }
        const int ex = ex0 + lx, ey = ey0 + ly, ez = ez0 + lz;
        const bool valid = ex < g.nelx && ey < g.nely && ez < g.nelz;
        // A row of this element: the 8 sub-cube factors three times, then zeros
        {
            uint32_t wp[4] = {0u, 0u, 0u, 0u};
            if (valid) {
#pragma unroll
                for (int s = 0; s < 8; s += 2) {
                    const int sx = (s >> 1) & 1, sz = s >> 2;
                    // sub-cubes s and s+1 differ in y only: adjacent in the density mesh
                    const int64_t di = ((int64_t)(ez * 2 + sz) * fg.nelx_d + (ex * 2 + sx)) * fg.nely_d + ey * 2;
                    const unsigned short lo = __bfloat16_as_ushort(w[di]);
                    const unsigned short hi = __bfloat16_as_ushort(w[di + 1]);
                    wp[s >> 1] = (uint32_t)lo | ((uint32_t)hi << 16);
                }
            }
            const uint4 row = make_uint4(wp[0], wp[1], wp[2], wp[3]);
            unsigned char *ar = as + tc_offset(tid, 0);
            *reinterpret_cast<uint4 *>(ar) = row;
            *reinterpret_cast<uint4 *>(ar + 128) = row;
            *reinterpret_cast<uint4 *>(ar + 256) = row;
            *reinterpret_cast<uint4 *>(ar + 384) = make_uint4(0u, 0u, 0u, 0u);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();

        float u[24], acc[24];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
            const int ln = ((lz + dz) * NBX + (lx + dx)) * NBY + (ly + dy);
#pragma unroll
            for (int c = 0; c < 3; ++c) u[3 * a + c] = xs[3 * ln + c];
        }
#pragma unroll
        for (int i = 0; i < 24; ++i) acc[i] = 0.f;

        bool ok = true;
#pragma unroll
        for (int chunk = 0; chunk < 3; ++chunk) {
            const int row0 = chunk * 128;
            const int nc = chunk < 2 ? 128 : 48;
            if (tid == 0) {
                fence_after();
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    const uint64_t ad = smem_desc(a_base + ks * 256);
                    const uint64_t bd = smem_desc(b_base + (row0 >> 3) * 512 + ks * 256);
                    mma_bf16(tmem, ad, bd, idesc_bf16(nc), ks);
                }
                mma_commit(mbar_a);
            }
            const bool got = mbar_wait(mbar_a, phase);
            phase ^= 1u;
            if (__syncthreads_or(!got)) {
                ok = false;
                break;
            }
            fence_after();
            if (chunk == 0) consume_chunk<0, 128>(tlane, u, acc);
            else if (chunk == 1) consume_chunk<128, 128>(tlane, u, acc);
            else consume_chunk<256, 48>(tlane, u, acc);
            fence_before();
            __syncthreads();   // all lanes read before the next chunk overwrites the columns
        }
        if (!ok) {
            if (tid == 0) {
                s_fail = 1;
                atomicExch(err, 1);
            }
            break;
        }

#pragma unroll
        for (int k = 0; k < 24; ++k) eo[k * BRICK_ELEMS + tid] = valid ? acc[k] : 0.f;
        __syncthreads();
        for (int i = tid; i < BRICK_NODES * 3; i += BRICK_ELEMS) {
            const int ln = i / 3, c = i - 3 * ln;
            const int ny_ = ln % NBY, nx_ = (ln / NBY) % NBX, nz_ = ln / (NBY * NBX);
            const int gx = ex0 + nx_, gy = ey0 + ny_, gz = ez0 + nz_;
            if (gx < g.nx && gy < g.ny && gz < g.nz) {
                const int64_t dof = 3 * (((int64_t)gz * g.nx + gx) * g.ny + gy) + c;
                if (freemask[dof]) {
                    float v = 0.f;
#pragma unroll
                    for (int a = 0; a < 8; ++a) {
                        const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
                        const int ex_ = nx_ - dx, ey_ = ny_ - dy, ez_ = nz_ - dz;
                        if (ex_ >= 0 && ex_ < BX && ey_ >= 0 && ey_ < BY && ez_ >= 0 && ez_ < BZ)
                            v += eo[(3 * a + c) * BRICK_ELEMS + (ez_ * BX + ex_) * BY + ey_];
                    }
                    const bool inner = nx_ > 0 && nx_ < BX && ny_ > 0 && ny_ < BY && nz_ > 0 && nz_ < BZ;
                    if (inner) y[dof] = v;
                    else atomicAdd(&y[dof], v);
                }
            }
        }
    }

    // An MMA still in flight after a timeout gets one more bounded wait
    // before its columns are released.
    if (s_fail && tid == 0) mbar_wait(mbar_a, phase ^ 1u);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_COLS) : "memory");
}

// B operand image for MR factor 2: row t (diagonal-major entry order) holds
// the hi / mid / lo BF16 pieces of KE_s[t] for s = 0..7; rows 300..303 and
// columns 24..31 are zero.
static uint16_t bf16_bits(double v) {
    const float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
static double bf16_value(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
}

void fine_tc_image(const std::vector<double> &packed_rowmajor, std::vector<uint16_t> &img) {
    img.assign(TC_B_BYTES / 2, 0);
    for (int t = 0; t < KE_PACK; ++t) {
        const int rm = pair_rowmajor(pair_i(t), pair_j(t));
        for (int s = 0; s < 8; ++s) {
            double r = packed_rowmajor[(size_t)s * KE_PACK + rm];
            for (int q = 0; q < 3; ++q) {
                const uint16_t b = bf16_bits(r);
                img[tc_offset(t, 8 * q + s) / 2] = b;
                r -= bf16_value(b);
            }
        }
    }
}

size_t fine_tc_image_bytes() { return TC_B_BYTES; }

static int num_sms_tc() {
    static int n = 0;
    if (!n) {
        int dev;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    }
    return n;
}

void launch_fine_apply_tc(const float *x, float *y, const __nv_bfloat16 *w, const uint8_t *fm, const void *bimg,
                          const FineGeom &fg, int *err, cudaStream_t st) {
    static int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaFuncSetAttribute(k_fine_apply_tc2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
        attr_dev = dev;
    }
    static int per_sm = 0;
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fine_apply_tc2, BRICK_ELEMS, TC_SMEM);
        if (per_sm < 1) per_sm = 1;
        if (per_sm > TC_CTAS_PER_SM) per_sm = TC_CTAS_PER_SM;   // 4 x 128 tensor-memory columns
    }
    int64_t grid = (int64_t)per_sm * num_sms_tc();
    if (grid > fg.nbricks) grid = fg.nbricks;
    if (grid < 1) grid = 1;
    k_fine_apply_tc2<<<(unsigned)grid, BRICK_ELEMS, TC_SMEM, st>>>(x, y, w, fm, (const uint4 *)bimg, fg, err);
    count_launch();
}

}  // namespace tosp
