// Finest-level operator of the mixed-precision V-cycle, MR factor 2, with the
// element-matrix formation on the 5th-generation tensor cores.
//
// y_e = K_e u_e with K_e = sum_s w_s KE_s (I/WOK/KelemProd.m:57-100).  For a
// brick of 128 elements the 300 packed entries of every K_e form one GEMM
// (M = 128 elements, N = 300 entries, kind::f16, FP32 accumulator):
//
//     D[e][t] = sum_k A[e][k] B1[t][k] + sum_k A[e][k] B2[t][k],
//     A[e][.] = (w_0..w_7, w_0..w_7),  B1[t][.] = (hi_s, mid_s),  B2[t][.] = (lo_s, 0)
//
// where hi/mid/lo are the three BF16 pieces of the FP64 block value KE_s[t]
// (their sum carries 24 significant bits).  The BF16 SIMP factors are exact
// in A and every product of two BF16 values is exact, so D is the FP32
// formation of K_e up to the order of the FP32 accumulation.  D lands in
// tensor memory (one lane per element, one column per entry); each thread
// reads its lane back in 32-column slices and applies y_i += k u_j,
// y_j += k u_i on the CUDA cores (576 FMAs per element instead of the 2148 of
// the Walsh-Hadamard CUDA-core formation).
//
// Pipelining inside a CTA: the next brick's nodal values and factors are
// staged with cp.async while the current brick computes; the entries are
// formed in 64-column chunks through two tensor-memory buffers, so the MMA of
// chunk c+1 runs while the threads consume chunk c, and the next brick's
// first two chunks run during the current brick's node sums and write-out.  Each CTA allocates 128
// tensor-memory columns; the dynamic shared memory per CTA is padded so that
// at most four CTAs (512 columns) are resident on an SM.  Every wait on an
// MMA-completion barrier is bounded; a timeout sets *err, leaves the brick
// loop and still frees the tensor memory.  Node sums and the write-out are
// those of the CUDA-core kernel (brick.cuh).
#include <cuda_bf16.h>

#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

#include "brick.cuh"
#include "tosp_internal.h"

namespace tosp {

namespace {

constexpr int TC_K = 16;                              // K of every MMA (kind::f16)
constexpr int TC_ROWS_B = 304;                        // 300 entries padded to a multiple of 16
constexpr int TC_GROUP = 8 * TC_K * 2;                // bytes of one 8-row group (256)
constexpr int TC_B_TILE = TC_ROWS_B / 8 * TC_GROUP;   // 9728 per B tile
constexpr int TC_B_BYTES = 2 * TC_B_TILE;             // B1 then B2
constexpr int TC_A_BYTES = BRICK_ELEMS / 8 * TC_GROUP;        // 4096 per A buffer
constexpr int TC_XS_FLOATS = BRICK_NODES * 4;                  // 900: nodes padded to float4
constexpr int TC_SLOTS_PAD = (BRICK_SLOTS + 3) / 4 * 4;       // slot table length
constexpr int TC_COLS = 128;                          // tensor-memory columns per CTA (2 x 64)
constexpr int TC_CHUNK = 64;
constexpr int TC_NCHUNK = 5;                          // 4 x 64 + 48 columns
constexpr int TC_CTAS_PER_SM = 4;                     // 4 x 128 = 512 columns
constexpr uint32_t TC_WAIT_LIMIT = 1u << 16;          // try_wait rounds before giving up
constexpr uint32_t TC_SUSPEND_NS = 20000;             // suspend-time hint of one try_wait round

// Canonical no-swizzle K-major layout with K = 16: 8-row x 16-byte core
// matrices, the two core matrices of a row group 128 B apart (leading byte
// offset), 8-row groups 256 B apart (stride byte offset).
__host__ __device__ constexpr int tc_offset(int row, int k) {
    return (row >> 3) * TC_GROUP + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);               // start address
    d |= (uint64_t)((128 >> 4) & 0x3FFF) << 16;          // leading byte offset (K direction)
    d |= (uint64_t)((TC_GROUP >> 4) & 0x3FFF) << 32;     // stride byte offset (M/N direction)
    d |= (uint64_t)1 << 46;                              // descriptor version for sm_100
    return d;                                            // base offset 0, no swizzle
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
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase), "r"(TC_SUSPEND_NS)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 4-byte asynchronous global -> shared copy; nbytes = 0 zero-fills.
__device__ __forceinline__ void cp_async4(void *dst, const void *src, int nbytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(nbytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

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

// Read NC columns of this thread's lane (entries T0..T0+NC-1) and apply them.
template <int T0, int NC>
__device__ __forceinline__ void consume(uint32_t taddr, const float (&u)[24], float (&acc)[24]) {
    uint32_t r[32];
    if constexpr (NC >= 32) {
        tmem_ld32(taddr, r);
        slice_steps<T0>(r, u, acc, std::make_integer_sequence<int, 32>{});
        if constexpr (NC > 32) consume<T0 + 32, NC - 32>(taddr + 32, u, acc);
    } else {
        static_assert(NC == 16, "chunk tails are 16 columns");
        tmem_ld16(taddr, r);
        slice_steps<T0>(r, u, acc, std::make_integer_sequence<int, 16>{});
    }
}

template <int C>
__device__ __forceinline__ void consume_chunk(uint32_t taddr, const float (&u)[24], float (&acc)[24]) {
    consume<C * TC_CHUNK, (C < TC_NCHUNK - 1) ? TC_CHUNK : TC_ROWS_B - C * TC_CHUNK>(taddr, u, acc);
}

// MMAs of chunk c into tensor-memory buffer (c & 1), then commit to its barrier.
__device__ __forceinline__ void issue_chunk(int c, uint32_t tmem, uint32_t a_addr, uint32_t b_addr, uint32_t mbar) {
    const int row0 = c * TC_CHUNK;
    const int nc = (c < TC_NCHUNK - 1) ? TC_CHUNK : TC_ROWS_B - row0;
    const uint32_t d = tmem + (uint32_t)((c & 1) * TC_CHUNK);
    const uint64_t ad = smem_desc(a_addr);
    const uint32_t boff = (uint32_t)((row0 >> 3) * TC_GROUP);
    mma_bf16(d, ad, smem_desc(b_addr + boff), idesc_bf16(nc), 0u);
    mma_bf16(d, ad, smem_desc(b_addr + TC_B_TILE + boff), idesc_bf16(nc), 1u);
    mma_commit(mbar);
}

}  // namespace

// Dynamic shared memory: B image, two A buffers, two node-input buffers, the
// node sums and the brick slot table; padded so that at most four CTAs fit on
// an SM (228 KB with 1 KB reserved per CTA: 4 x 53.1 KB fit, 5 do not).  The
// MMA operands need 16-byte aligned starts; the barriers and the
// tensor-memory address are static (8-byte aligned) shared variables.
constexpr size_t TC_OFF_A = TC_B_BYTES;
constexpr size_t TC_OFF_XS = TC_OFF_A + 2 * TC_A_BYTES;
constexpr size_t TC_OFF_YS = TC_OFF_XS + sizeof(float) * 2 * TC_XS_FLOATS;
constexpr size_t TC_OFF_REL = TC_OFF_YS + sizeof(float) * TC_XS_FLOATS;
constexpr size_t TC_OFF_PK = TC_OFF_REL + sizeof(int32_t) * TC_SLOTS_PAD;
constexpr size_t TC_SMEM_USED = TC_OFF_PK + sizeof(uint16_t) * TC_SLOTS_PAD;
constexpr size_t TC_SMEM = 52 * 1024;
static_assert(TC_OFF_A % 16 == 0 && TC_OFF_XS % 16 == 0 && TC_OFF_YS % 16 == 0, "operand alignment");
static_assert(TC_OFF_REL % 4 == 0 && TC_OFF_PK % 2 == 0, "slot table alignment");
static_assert(TC_SMEM_USED <= TC_SMEM, "tensor-core operator shared memory");
static_assert(TC_ROWS_B - (TC_NCHUNK - 1) * TC_CHUNK == 48, "last chunk");

// Stage brick `brick` (nodal values, A rows) into buffer `buf` with cp.async.
__device__ __forceinline__ void stage_brick(int64_t brick, int buf, const float *__restrict__ x,
                                            const __nv_bfloat16 *__restrict__ w, const FineGeom &fg,
                                            unsigned char *smem, const int32_t *rel, const uint16_t *pk,
                                            int tid) {
    const Grid &g = fg.g;
    int bbx, bby, bbz;
    brick_xyz(brick, fg, bbx, bby, bbz);
    const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
    float *xs = reinterpret_cast<float *>(smem + TC_OFF_XS) + buf * TC_XS_FLOATS;
    const float *xb = x + brick_base_dof(ex0, ey0, ez0, g);
    if (brick_interior(ex0, ey0, ez0, g)) {
        for (int i = tid; i < BRICK_SLOTS; i += BRICK_ELEMS) cp_async4(xs + i + i / 3, xb + rel[i], 4);
    } else {
        for (int i = tid; i < BRICK_SLOTS; i += BRICK_ELEMS) {
            const bool in = brick_slot_in(pk[i], ex0, ey0, ez0, g);
            cp_async4(xs + i + i / 3, in ? xb + rel[i] : x, in ? 4 : 0);
        }
    }
    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    const int ex = ex0 + lx, ey = ey0 + ly, ez = ez0 + lz;
    const bool valid = ex < g.nelx && ey < g.nely && ez < g.nelz;
    unsigned char *ar = smem + TC_OFF_A + buf * TC_A_BYTES + tc_offset(tid, 0);
    const __nv_bfloat16 *wb = w + ((int64_t)(ez * 2) * fg.nelx_d + ex * 2) * fg.nely_d + ey * 2;
#pragma unroll
    for (int s = 0; s < 8; s += 2) {
        // sub-cubes s and s+1 differ in y only: adjacent in the density mesh
        const int sx = (s >> 1) & 1, sz = s >> 2;
        const __nv_bfloat16 *src = valid ? wb + ((int64_t)sz * fg.nelx_d + sx) * fg.nely_d : w;
        cp_async4(ar + 2 * s, src, valid ? 4 : 0);
        cp_async4(ar + 128 + 2 * s, src, valid ? 4 : 0);
    }
}

__global__ void __launch_bounds__(BRICK_ELEMS, TC_CTAS_PER_SM)
k_fine_apply_tc2(const float *__restrict__ x, float *__restrict__ y, const __nv_bfloat16 *__restrict__ w,
                 const uint8_t *__restrict__ freemask, const uint4 *__restrict__ bimg, FineGeom fg,
                 int *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float *ys = reinterpret_cast<float *>(smem_raw + TC_OFF_YS);          // node sums
    int32_t *rel = reinterpret_cast<int32_t *>(smem_raw + TC_OFF_REL);    // slot table
    uint16_t *pk = reinterpret_cast<uint16_t *>(smem_raw + TC_OFF_PK);
    __shared__ __align__(8) uint64_t s_mbar[2];
    __shared__ __align__(8) uint32_t s_tmem;
    __shared__ int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5;
    if (smem_u32(smem_raw) & 15u) {   // operand tiles need 16-byte aligned starts
        if (tid == 0) atomicExch(err, 2);
        return;
    }
    const Grid &g = fg.g;
    for (int i = tid; i < TC_B_BYTES / 16; i += BRICK_ELEMS) reinterpret_cast<uint4 *>(smem_raw)[i] = bimg[i];
    brick_slots_init(rel, pk, g, tid);
    if (tid == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);    // this warp's 32 lanes
    const uint32_t mbar0 = smem_u32(&s_mbar[0]), mbar1 = smem_u32(&s_mbar[1]);
    const uint32_t b_addr = smem_u32(smem_raw);
    const uint32_t a_addr0 = smem_u32(smem_raw + TC_OFF_A);
    uint32_t ph0 = 0, ph1 = 0;

    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    const int ln0 = brick_base_node(tid);

    // Prologue: the first brick's inputs, then its first two chunks.  In the
    // loop, brick b+1's inputs are staged while brick b computes, and its
    // first two chunks are issued as soon as brick b's last chunk is read, so
    // they run during brick b's node sums and write-out.
    if (blockIdx.x < fg.nbricks) stage_brick(blockIdx.x, 0, x, w, fg, smem_raw, rel, pk, tid);
    cp_async_commit();
    cp_async_wait_0();
    fence_async_smem();
    __syncthreads();
    if (tid == 0 && blockIdx.x < fg.nbricks) {
        fence_after();
        issue_chunk(0, tmem, a_addr0, b_addr, mbar0);
        issue_chunk(1, tmem, a_addr0, b_addr, mbar1);
    }

    int buf = 0;
    for (int64_t brick = blockIdx.x; brick < fg.nbricks; brick += gridDim.x, buf ^= 1) {
        // the other buffers were last read by the previous brick, whose
        // threads have all passed its chunk barriers
        const int64_t next = brick + gridDim.x;
        const bool chk = brick_check_fixed(brick, fg);
        if (next < fg.nbricks) stage_brick(next, buf ^ 1, x, w, fg, smem_raw, rel, pk, tid);
        cp_async_commit();

        int bbx, bby, bbz;
        brick_xyz(brick, fg, bbx, bby, bbz);
        const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
        const bool valid = ex0 + lx < g.nelx && ey0 + ly < g.nely && ez0 + lz < g.nelz;
        const uint32_t a_addr = a_addr0 + (uint32_t)(buf * TC_A_BYTES);
        const float *xs = reinterpret_cast<const float *>(smem_raw + TC_OFF_XS) + buf * TC_XS_FLOATS;

        float u[24], acc[24];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
            const float4 v = reinterpret_cast<const float4 *>(xs)[ln0 + (dz * NBX + dx) * NBY + dy];
            u[3 * a] = v.x;
            u[3 * a + 1] = v.y;
            u[3 * a + 2] = v.z;
        }
#pragma unroll
        for (int i = 0; i < 24; ++i) acc[i] = 0.f;

        bool ok = true;
#pragma unroll
        for (int c = 0; c < TC_NCHUNK; ++c) {
            const bool got = (c & 1) ? mbar_wait(mbar1, ph1) : mbar_wait(mbar0, ph0);
            if (c & 1) ph1 ^= 1u;
            else ph0 ^= 1u;
            if (__syncthreads_or(!got)) {
                ok = false;
                break;
            }
            if (c == 0) {
                // every thread has finished the previous brick's write-out
                for (int i = tid; i < BRICK_NODES; i += BRICK_ELEMS)
                    reinterpret_cast<float4 *>(ys)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            fence_after();
            const uint32_t taddr = tlane + (uint32_t)((c & 1) * TC_CHUNK);
            if (c == 0) consume_chunk<0>(taddr, u, acc);
            else if (c == 1) consume_chunk<1>(taddr, u, acc);
            else if (c == 2) consume_chunk<2>(taddr, u, acc);
            else if (c == 3) consume_chunk<3>(taddr, u, acc);
            else consume_chunk<4>(taddr, u, acc);
            fence_before();
            __syncthreads();   // buffer (c & 1) fully read
            if (tid == 0 && c + 2 < TC_NCHUNK) {
                fence_after();
                issue_chunk(c + 2, tmem, a_addr, b_addr, (c & 1) ? mbar1 : mbar0);
            }
        }
        if (!ok) {
            if (tid == 0) {
                s_fail = 1;
                atomicExch(err, 1);
            }
            break;
        }
        // next brick's inputs complete and visible to the tensor cores
        cp_async_wait_0();
        fence_async_smem();
        __syncthreads();
        if (tid == 0 && next < fg.nbricks) {
            fence_after();
            const uint32_t a_next = a_addr0 + (uint32_t)((buf ^ 1) * TC_A_BYTES);
            issue_chunk(0, tmem, a_next, b_addr, mbar0);
            issue_chunk(1, tmem, a_next, b_addr, mbar1);
        }
        brick_accumulate4(reinterpret_cast<float4 *>(ys), acc, valid, ln0);
        brick_writeout_tab<float, 4>(ys, y, freemask, g, ex0, ey0, ez0, rel, pk, tid, chk);
    }
    cp_async_wait_0();

    // MMAs still in flight after a timeout get one more bounded wait each
    // before their columns are released.
    if (s_fail && tid == 0) {
        mbar_wait(mbar0, ph0);
        mbar_wait(mbar1, ph1);
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_COLS) : "memory");
}

// B operand image for MR factor 2: tile B1 row t (diagonal-major entry order)
// holds the hi and mid BF16 pieces of KE_s[t] for s = 0..7, tile B2 the lo
// pieces and zeros; rows 300..303 are zero.
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
                const int off = q < 2 ? tc_offset(t, 8 * q + s) : TC_B_TILE + tc_offset(t, s);
                img[off / 2] = b;
                r -= bf16_value(b);
            }
        }
    }
}

size_t fine_tc_image_bytes() { return TC_B_BYTES; }

// Resident CTAs per SM from the device limits (shared memory with the
// per-CTA reservation, registers at warp allocation granularity), capped by
// the 512 tensor-memory columns.
static int tc_ctas_per_sm() {
    int dev = 0, smem_sm = 0, smem_res = 0, regs_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, k_fine_apply_tc2) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const size_t per_cta = TC_SMEM + fa.sharedSizeBytes + (size_t)smem_res;
    const int by_smem = (int)(smem_sm / per_cta);
    const int regs_warp = (fa.numRegs * 32 + 255) / 256 * 256;
    const int by_regs = regs_sm / (regs_warp * (BRICK_ELEMS / 32));
    int n = by_smem < by_regs ? by_smem : by_regs;
    if (n > TC_CTAS_PER_SM) n = TC_CTAS_PER_SM;
    return n < 1 ? 1 : n;
}

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
    static int attr_dev = -1, per_sm = 1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaFuncSetAttribute(k_fine_apply_tc2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
        cudaFuncSetAttribute(k_fine_apply_tc2, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        per_sm = tc_ctas_per_sm();
        attr_dev = dev;
    }
    int64_t grid = (int64_t)per_sm * num_sms_tc();
    if (grid > fg.nbricks) grid = fg.nbricks;
    if (grid < 1) grid = 1;
    k_fine_apply_tc2<<<(unsigned)grid, BRICK_ELEMS, TC_SMEM, st>>>(x, y, w, fm, (const uint4 *)bimg, fg, err);
    count_launch();
}

}  // namespace tosp
