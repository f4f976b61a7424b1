// Finest-level operator of the mixed-precision V-cycle on the 5th-generation
// tensor cores, for multiresolution factors n = 1, 2 and 3.
//
// y_e = sum_s w_s KE_s u_e (I/WOK/KelemProd.m:57-100) over the n^3 density
// sub-cells s of displacement element e.  For a brick of 128 elements the
// products of the shared 24x24 sub-cell blocks with every element's nodal
// vector are one GEMM (M = 128 elements, N = 24 n^3 block rows, K = 24 element
// dofs, kind::f16, FP32 accumulator):
//
//     D[e][24 s + i] = sum_j KE_s[i][j] u_e[j],
//
// and each thread weights its element's 24 n^3 values with the element's n^3
// SIMP factors on the CUDA cores, two values per packed FMA (fma.rn.f32x2,
// the rounding of two FP32 FMAs):
//
//     y_e[i] = sum_s w_s D[e][24 s + i].
//
// 24 n^3 FMAs per element instead of the 300 (n^3 + 2) of forming K_e on the
// CUDA cores (n = 3: 648 against 8 700).
//
// FP16 operands carry each value in two pieces.  u_e is scaled by a power of
// two per element (largest entry in [2^13, 2^14)) and split into hi + lo; the
// blocks are scaled by one power of two (largest entry in [2^14, 2^15)) and
// split into hi + mid.  The products hi*hi, lo*hi and hi*mid are exact in the
// FP32 accumulator and carry about 22 significant bits of KE_s u_e; the
// neglected lo*mid term is below 2^-22 |KE_s| |u_e|.  The scale factors are
// undone on the weights.  K runs over five 16-wide steps:
//
//     step 0:  u_hi[0..15]                .  KE_hi[.][0..15]
//     step 1:  u_hi[16..23] u_lo[0..7]    .  KE_hi[.][16..23] KE_hi[.][0..7]
//     step 2:  u_lo[8..23]                .  KE_hi[.][8..23]
//     step 3:  u_hi[0..15]   (A tile 0)   .  KE_mid[.][0..15]
//     step 4:  (A tile 1)                 .  KE_mid[.][16..23] 0
//
// so A holds three 16-wide tiles per element row and the B image five.  The
// weights stay BF16 (exact in FP32), the same factors the coarse levels use.
//
// Pipelining inside a CTA: the accumulator columns are produced in chunks
// (64 columns; 32 for n = 1, whose 24 rows are one chunk) through two
// tensor-memory buffers, so the MMAs of chunk c+2 are issued as soon as chunk c
// is read and run while the threads consume chunk c+1.  Once the first chunk
// is read (every thread then holds the brick's factors and the A tiles are
// built), the next brick's nodal values and factors are staged with cp.async
// into the same buffers; once the last chunk is read, each thread stores its
// element's corner outputs, the A tiles are rebuilt for the next brick and
// that brick's first two chunks run during the current brick's node gather
// and write-out (brick.cuh: one node per thread sums the outputs of its up
// to eight elements in corner order, then stores it, or adds it atomically on
// the brick's faces).  Every wait on an MMA-completion barrier is bounded; a
// timeout sets *err, leaves the brick loop and still frees the tensor memory.
//
// A CTA runs NB such bricks side by side (two; three for n = 3), four warps
// each, so they share one copy of the B image (30 KB for n = 2, 103 KB for
// n = 3): two CTAs of eight warps per SM for n = 2, one of twelve for n = 3.
//
// The factors are staged as the brick's slab of the density mesh (rows along
// y of 8n BF16 values copied in 4-byte pieces), which needs n * nely even; the
// host uses the CUDA-core kernel otherwise.
//
// The same kernel with FP32 factors (one cell per 4-byte piece), the element's
// mean translation subtracted from u_e and, for n = 1, 2, the blocks in three
// FP16 pieces (eight MMA steps) is the product of the FP64 CG recurrence when
// the caller asks for it (cg_product 1).  Its larger B image is shared by four
// bricks per CTA at one CTA per SM, which keeps 16 warps per SM; for n = 3 it
// keeps the two-piece image at two bricks per CTA.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

#include "brick.cuh"
#include "tosp_internal.h"

namespace tosp {

namespace {

constexpr int TC_K = 16;                                  // K of every MMA (kind::f16)
constexpr int TC_GROUP = 8 * TC_K * 2;                    // bytes of one 8-row group (256)
constexpr int TC_A_TILE = BRICK_ELEMS / 8 * TC_GROUP;     // 4096 per A step
constexpr int TC_A_BYTES = 3 * TC_A_TILE;
constexpr int TC_XS_FLOATS = BRICK_NODES * 4;             // 900: nodes padded to float4
constexpr int TC_EO_BYTES = 8 * BRICK_ELEMS * 16;         // element outputs: one float4 per corner
constexpr int TC_SLOTS_PAD = (BRICK_SLOTS + 3) / 4 * 4;   // slot table length
constexpr uint32_t TC_WAIT_LIMIT = 1u << 16;              // try_wait rounds before giving up
constexpr uint32_t TC_SUSPEND_NS = 20000;                 // suspend-time hint of one try_wait round

// Sizes of the kernel for MR factor N and SIMP factors of type WT (BF16 for
// the V-cycle, FP32 for the CG's product).
template <int N, typename WT = __nv_bfloat16>
struct Tc {
    static constexpr int NS = N * N * N;                  // sub-cells per element
    static constexpr int NROWS = 24 * NS;                 // block rows (GEMM N)
    static constexpr int NPAD = (NROWS + 15) / 16 * 16;   // padded to the MMA's N granularity
    static constexpr int CH = N == 1 ? 32 : 64;           // accumulator columns per chunk
    static constexpr int NCH = (NPAD + CH - 1) / CH;
    static constexpr int COLS = 2 * CH;                   // tensor-memory columns per CTA
    static constexpr int B_TILE = NPAD / 8 * TC_GROUP;    // bytes of one B step
    // blocks in two FP16 pieces (hi + mid, five MMA steps) for the V-cycle's
    // BF16-factor kernel; the CG's FP32-factor kernel takes three (hi + mid +
    // lo, eight steps) for n = 1, 2 and two for n = 3, whose three-piece image
    // (166 KB) would leave room for one brick per SM (measured on the MR-3
    // bridge: two pieces at two bricks per CTA, 0.157 ms per launch and a
    // 14 % faster V-cycle solve for the same 124 iterations, against 0.287 ms)
    static constexpr bool K3 = sizeof(WT) == 4;
    static constexpr int B_STEPS = K3 && N != 3 ? 8 : 5;
    static constexpr int B_BYTES = B_STEPS * B_TILE;
    static constexpr int WY = BY * N, WX = BX * N, WZ = BZ * N;   // factor slab (density cells)
    static constexpr int CPP = 4 / (int)sizeof(WT);       // cells per 4-byte piece
    static constexpr int W_BYTES = (WY * WX * WZ * (int)sizeof(WT) + 15) / 16 * 16;
    static constexpr int UPR = WY / CPP;                  // 4-byte pieces per slab row
    // bricks processed side by side by one CTA, sharing the B image: four
    // warps each, their own A tiles, staging, outputs, barriers and
    // tensor-memory columns
    static constexpr int NB = K3 ? (N == 3 ? 2 : 4) : (N == 3 ? 3 : 2);
    static constexpr int THREADS = NB * BRICK_ELEMS;
    static constexpr int TMEM_COLS = NB * COLS <= 64 ? 64 : (NB * COLS <= 128 ? 128 : (NB * COLS <= 256 ? 256 : 512));
    // layout: B image, slot table, then one region per brick
    static constexpr size_t OFF_REL = B_BYTES;
    static constexpr size_t OFF_PK = OFF_REL + sizeof(int32_t) * TC_SLOTS_PAD;
    static constexpr size_t OFF_G = (OFF_PK + sizeof(uint16_t) * TC_SLOTS_PAD + 127) / 128 * 128;
    static constexpr size_t G_A = 0;                      // offsets inside a brick's region
    static constexpr size_t G_XS = G_A + TC_A_BYTES;
    static constexpr size_t G_EO = G_XS + sizeof(float) * TC_XS_FLOATS;
    static constexpr size_t G_W = G_EO + TC_EO_BYTES;
    static constexpr size_t G_BYTES = (G_W + W_BYTES + 127) / 128 * 128;
    static constexpr size_t SMEM = OFF_G + NB * G_BYTES;
    static constexpr int MINB = K3 || N == 3 ? 1 : (N == 2 ? 2 : 3);   // register cap: CTAs per SM aimed at
    static_assert(B_TILE % 16 == 0 && OFF_G % 16 == 0 && G_BYTES % 16 == 0 && G_XS % 16 == 0 &&
                      G_EO % 16 == 0 && G_W % 16 == 0, "operand alignment");
    static_assert(OFF_REL % 4 == 0 && OFF_PK % 2 == 0, "slot table alignment");
    static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
    static_assert(sizeof(WT) == 2 || sizeof(WT) == 4, "BF16 or FP32 factors");
    static_assert(NB * COLS <= 512, "tensor memory of an SM");
};

__host__ __device__ constexpr int chunk_width(int npad, int ch, int c) { return npad - c * ch < ch ? npad - c * ch : ch; }

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

// kind::f16 instruction descriptor: FP32 accumulator, FP16 A and B (format
// code 0), both K-major, M = 128, N = n (a multiple of 16, at most 256).
__host__ __device__ constexpr uint32_t idesc_f16(int n) {
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
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

// Barriers of one brick group (four warps, named barrier 1 + group; 0 is
// __syncthreads).
__device__ __forceinline__ void group_sync(int grp) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(BRICK_ELEMS) : "memory");
}
__device__ __forceinline__ bool group_sync_or(int grp, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(1 + grp), "r"(BRICK_ELEMS)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 4-byte asynchronous global -> shared copy; nbytes = 0 zero-fills.
__device__ __forceinline__ void cp_async4(void *dst, const void *src, int nbytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(nbytes)
                 : "memory");
}
// 16-byte asynchronous global -> shared copy (both addresses 16-byte
// aligned); nbytes = 0 zero-fills.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int nbytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(nbytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// W consecutive columns of this warp's 32 lanes (one column per register).
template <int W>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[W]);

template <>
__device__ __forceinline__ void tmem_ld<64>(uint32_t taddr, uint32_t (&r)[64]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, uint32_t (&r)[32]) {
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

template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Chunk C holds block rows C*CH .. C*CH + width - 1: row r is entry
// i = r % 24 of sub-cell s = r / 24 (rows from 24 n^3 on are padding).
// Columns t, t+1 (t even) are entries i, i+1 of the same sub-cell, weighted
// by one packed FMA.
template <int N, int C>
__device__ __forceinline__ void consume_chunk(uint32_t taddr, const float (&ws)[Tc<N>::NS], float2 (&acc)[12]) {
    constexpr int W = chunk_width(Tc<N>::NPAD, Tc<N>::CH, C);
    uint32_t r[W];
    tmem_ld<W>(taddr, r);
#pragma unroll
    for (int t = 0; t < W; t += 2) {
        const int row = C * Tc<N>::CH + t;
        if (row < Tc<N>::NROWS) {
            const float w = ws[row / 24];
            acc[(row % 24) / 2] = __ffma2_rn(make_float2(w, w),
                                             make_float2(__uint_as_float(r[t]), __uint_as_float(r[t + 1])),
                                             acc[(row % 24) / 2]);
        }
    }
}

// consume_chunk for a chunk index known after unrolling.
template <int N, int... Cs>
__device__ __forceinline__ void consume_any(int c, uint32_t taddr, const float (&ws)[Tc<N>::NS], float2 (&acc)[12],
                                            std::integer_sequence<int, Cs...>) {
    ((c == Cs ? consume_chunk<N, Cs>(taddr, ws, acc) : void()), ...);
}

// A tile of MMA step t: steps 0-2 run A tiles 0, 1, 2 ([u_hi u_lo]) against
// the hi piece of the blocks; steps 3-4 (two-piece image) run tiles 0, 1
// (u_hi) against the mid piece; in the three-piece image steps 3-5 run tiles
// 0, 1, 2 against the mid piece and steps 6-7 tiles 0, 1 against the lo piece.
__host__ __device__ constexpr int step_a_tile(int t) { return t < 6 ? t % 3 : t - 6; }

// The B_STEPS MMAs of chunk c into tensor-memory buffer (c & 1), then a commit
// to its barrier.
template <int N, typename WT>
__device__ __forceinline__ void issue_chunk(int c, uint32_t tmem, uint32_t a_addr, uint32_t b_addr, uint32_t mbar) {
    using K = Tc<N, WT>;
    const uint32_t d = tmem + (uint32_t)((c & 1) * K::CH);
    const uint32_t boff = (uint32_t)(c * K::CH / 8 * TC_GROUP);
    const uint32_t id = idesc_f16(chunk_width(K::NPAD, K::CH, c));
#pragma unroll
    for (int t = 0; t < K::B_STEPS; ++t)
        mma_f16(d, smem_desc(a_addr + step_a_tile(t) * TC_A_TILE), smem_desc(b_addr + t * K::B_TILE + boff), id,
                t ? 1u : 0u);
    mma_commit(mbar);
}

// Entry i of the 24 element outputs held as 12 pairs.
__device__ __forceinline__ float acc_at(const float2 (&acc)[12], int i) { return (i & 1) ? acc[i >> 1].y : acc[i >> 1].x; }

__device__ __forceinline__ uint32_t half2_bits(__half2 h) {
    uint32_t b;
    memcpy(&b, &h, 4);
    return b;
}

__device__ __forceinline__ float factor_value(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float factor_value(float v) { return v; }

// Stage brick `brick` (nodal values, and the brick's slab of SIMP factors on
// the density mesh) with cp.async; absent nodes and cells read as zero.
template <int N, typename WT>
__device__ __forceinline__ void stage_brick(int64_t brick, float *xs, WT *wslab, const float *__restrict__ x,
                                            const WT *__restrict__ w, const FineGeom &fg,
                                            const int32_t *rel, const uint16_t *pk, int tid) {
    using K = Tc<N, WT>;
    const Grid &g = fg.g;
    int bbx, bby, bbz;
    brick_xyz(brick, fg, bbx, bby, bbz);
    const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
    const float *xb = x + brick_base_dof(ex0, ey0, ez0, g);
    // node by node: three values into a node's float4 slot
    if (brick_interior(ex0, ey0, ez0, g)) {
        for (int ln = tid; ln < BRICK_NODES; ln += BRICK_ELEMS) {
            const float *src = xb + rel[3 * ln];
            float *dst = xs + 4 * ln;
            cp_async4(dst, src, 4);
            cp_async4(dst + 1, src + 1, 4);
            cp_async4(dst + 2, src + 2, 4);
        }
    } else {
        for (int ln = tid; ln < BRICK_NODES; ln += BRICK_ELEMS) {
            const bool in = brick_slot_in(pk[3 * ln], ex0, ey0, ez0, g);
            const float *src = in ? xb + rel[3 * ln] : x;
            float *dst = xs + 4 * ln;
            cp_async4(dst, src, in ? 4 : 0);
            cp_async4(dst + 1, in ? src + 1 : x, in ? 4 : 0);
            cp_async4(dst + 2, in ? src + 2 : x, in ? 4 : 0);
        }
    }
    // factor slab: rows along y of WY values, 4-byte pieces (two BF16 cells
    // or one FP32 cell); with BF16 the density mesh has n * nely cells along
    // y, an even number, so a piece is wholly inside or wholly outside the
    // mesh and 4-byte aligned
    const int nelz_d = g.nelz * N;
    const int xd0 = ex0 * N, yd0 = ey0 * N, zd0 = ez0 * N;
    // 16-byte pieces when the density mesh's rows along y are a whole number
    // of pieces: every row then starts 16-byte aligned (the brick's first
    // cell yd0 = 8 N bby is a multiple of a piece) and a piece lies wholly
    // inside or wholly outside the mesh
    constexpr int C16 = 16 / (int)sizeof(WT);             // cells per 16-byte piece
    static_assert((K::WY * (int)sizeof(WT)) % 16 == 0 && (BY * N) % C16 == 0, "16-byte slab pieces");
    if (fg.nely_d % C16 == 0) {
        constexpr int P16 = K::WY / C16;                  // pieces per slab row
        for (int u = tid; u < K::WZ * K::WX * P16; u += BRICK_ELEMS) {
            const int row = u / P16, k = u - row * P16;
            const int rz = row / K::WX, rx = row - rz * K::WX;
            const int zd = zd0 + rz, xd = xd0 + rx, yd = yd0 + C16 * k;
            const bool in = zd < nelz_d && xd < fg.nelx_d && yd < fg.nely_d;
            const WT *src = in ? w + ((int64_t)zd * fg.nelx_d + xd) * fg.nely_d + yd : w;
            cp_async16(wslab + row * K::WY + C16 * k, src, in ? 16 : 0);
        }
        return;
    }
    for (int u = tid; u < K::WZ * K::WX * K::UPR; u += BRICK_ELEMS) {
        const int row = u / K::UPR, k = u - row * K::UPR;
        const int rz = row / K::WX, rx = row - rz * K::WX;
        const int zd = zd0 + rz, xd = xd0 + rx, yd = yd0 + K::CPP * k;
        const bool in = zd < nelz_d && xd < fg.nelx_d && yd < fg.nely_d;
        const WT *src = in ? w + ((int64_t)zd * fg.nelx_d + xd) * fg.nely_d + yd : w;
        cp_async4(wslab + row * K::WY + K::CPP * k, src, in ? 4 : 0);
    }
}

// A tiles of this thread's element (row tid) from the staged nodal values;
// returns 2^(E - 140), the inverse of the element's scale factor.  SHIFT:
// the element's mean translation (one value per component) is subtracted
// first.  The blocks map a rigid translation to zero (in exact arithmetic), so
// the product is unchanged, while the FP16 pieces, the truncation of the
// blocks and the FP32 accumulation then err relative to the element's
// deformation instead of its displacement, which for smooth fields is the
// much smaller part.
template <bool SHIFT>
__device__ __forceinline__ float build_a(const float *xs, unsigned char *abuf, int ln0, int tid) {
    float u[24];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
        const float4 v = reinterpret_cast<const float4 *>(xs)[ln0 + (dz * NBX + dx) * NBY + dy];
        u[3 * a] = v.x;
        u[3 * a + 1] = v.y;
        u[3 * a + 2] = v.z;
    }
    if constexpr (SHIFT) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float t = 0.f;
#pragma unroll
            for (int a = 0; a < 8; ++a) t += u[3 * a + c];
            t *= 0.125f;
#pragma unroll
            for (int a = 0; a < 8; ++a) u[3 * a + c] -= t;
        }
    }
    float m = 0.f;
#pragma unroll
    for (int j = 0; j < 24; ++j) m = fmaxf(m, fabsf(u[j]));
    // biased exponent E of the largest entry, so that m 2^(140 - E) lies in
    // [2^13, 2^14); the clamp keeps both scale factors normal
    uint32_t E = __float_as_uint(m) >> 23;
    E = E < 14u ? 14u : (E > 254u ? 254u : E);
    const float su = __uint_as_float((267u - E) << 23);
    uint32_t hw[12], lw[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) {
        const float a0 = u[2 * q] * su, a1 = u[2 * q + 1] * su;
        const __half2 h = __floats2half2_rn(a0, a1);
        const float2 hf = __half22float2(h);
        hw[q] = half2_bits(h);
        lw[q] = half2_bits(__floats2half2_rn(a0 - hf.x, a1 - hf.y));   // differences exact in FP32
    }
    unsigned char *ar = abuf + tc_offset(tid, 0);
    *reinterpret_cast<uint4 *>(ar) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *reinterpret_cast<uint4 *>(ar + 128) = make_uint4(hw[4], hw[5], hw[6], hw[7]);
    *reinterpret_cast<uint4 *>(ar + TC_A_TILE) = make_uint4(hw[8], hw[9], hw[10], hw[11]);
    *reinterpret_cast<uint4 *>(ar + TC_A_TILE + 128) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    *reinterpret_cast<uint4 *>(ar + 2 * TC_A_TILE) = make_uint4(lw[4], lw[5], lw[6], lw[7]);
    *reinterpret_cast<uint4 *>(ar + 2 * TC_A_TILE + 128) = make_uint4(lw[8], lw[9], lw[10], lw[11]);
    return __uint_as_float((E - 13u) << 23);
}

}  // namespace

// Dynamic shared memory: the B image and the brick slot table (shared by the
// CTA's bricks), then per brick its A tiles, staged nodal values, element
// outputs and factor slab.  The MMA operands need 16-byte aligned starts; the
// barriers and the tensor-memory address are static (8-byte aligned) shared
// variables.  Threads 128 g .. 128 g + 127 (warps 4g .. 4g+3) form brick group
// g: bricks g, g + NB, ... of the CTA's share, with the group's own named
// barrier, MMA-completion barriers and tensor-memory columns (lanes 0-127 of
// columns COLS g .. COLS (g+1) - 1, which its warps reach as warps 0-3 would).
template <int N, typename WT>
__global__ void __launch_bounds__(Tc<N, WT>::THREADS, Tc<N, WT>::MINB)
k_fine_apply_tc(const float *__restrict__ x, float *__restrict__ y, const WT *__restrict__ w,
                const uint8_t *__restrict__ freemask, const uint4 *__restrict__ bimg, FineGeom fg,
                int *__restrict__ err) {
    using K = Tc<N, WT>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_mbar[2 * K::NB];
    __shared__ __align__(8) uint32_t s_tmem;
    __shared__ int s_fail[K::NB];

    const int ttid = threadIdx.x;
    const int grp = ttid / BRICK_ELEMS, tid = ttid - grp * BRICK_ELEMS;   // group, thread within it
    const int warp = tid >> 5;                                           // warp within the group
    if (smem_u32(smem_raw) & 15u) {   // operand tiles need 16-byte aligned starts
        if (ttid == 0) atomicExch(err, 2);
        return;
    }
    int32_t *rel = reinterpret_cast<int32_t *>(smem_raw + K::OFF_REL);    // slot table
    uint16_t *pk = reinterpret_cast<uint16_t *>(smem_raw + K::OFF_PK);
    unsigned char *gbase = smem_raw + K::OFF_G + grp * K::G_BYTES;
    unsigned char *abuf = gbase + K::G_A;
    float *xs = reinterpret_cast<float *>(gbase + K::G_XS);              // staged nodal values
    float4 *eo4 = reinterpret_cast<float4 *>(gbase + K::G_EO);           // element outputs per corner
    WT *wslab = reinterpret_cast<WT *>(gbase + K::G_W);                  // SIMP factors

    const Grid &g = fg.g;
    for (int i = ttid; i < K::B_BYTES / 16; i += K::THREADS) reinterpret_cast<uint4 *>(smem_raw)[i] = bimg[i];
    const float inv_ke = reinterpret_cast<const float *>(bimg)[K::B_BYTES / 4];   // undoes the block scale
    if (grp == 0) brick_slots_init(rel, pk, g, tid);
    if (tid == 0) {
        s_fail[grp] = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[2 * grp])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[2 * grp + 1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (ttid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(K::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = s_tmem + (uint32_t)(grp * K::COLS);           // this group's columns
    const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);        // this warp's 32 lanes
    const uint32_t mbar0 = smem_u32(&s_mbar[2 * grp]), mbar1 = smem_u32(&s_mbar[2 * grp + 1]);
    const uint32_t b_addr = smem_u32(smem_raw);
    const uint32_t a_addr = smem_u32(abuf);
    uint32_t ph0 = 0, ph1 = 0;

    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    const int ln0 = brick_base_node(tid);
    const int64_t first = (int64_t)blockIdx.x * K::NB + grp, stride = (int64_t)gridDim.x * K::NB;

    // Prologue: the first brick's inputs and A tiles, then its first two
    // chunks (a group without a brick skips the loop).
    float fsc = 1.f;
    if (first < fg.nbricks) {
        stage_brick<N, WT>(first, xs, wslab, x, w, fg, rel, pk, tid);
        cp_async_commit();
        cp_async_wait_0();
        group_sync(grp);
        fsc = build_a<K::K3>(xs, abuf, ln0, tid);
        fence_async_smem();
        group_sync(grp);
        if (tid == 0) {
            fence_after();
            issue_chunk<N, WT>(0, tmem, a_addr, b_addr, mbar0);
            if (K::NCH > 1) issue_chunk<N, WT>(1, tmem, a_addr, b_addr, mbar1);
        }
    }

    for (int64_t brick = first; brick < fg.nbricks; brick += stride) {
        const int64_t next = brick + stride;
        const bool chk = brick_check_fixed(brick, fg);

        int bbx, bby, bbz;
        brick_xyz(brick, fg, bbx, bby, bbz);
        const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
        const bool valid = ex0 + lx < g.nelx && ey0 + ly < g.nely && ez0 + lz < g.nelz;

        // this element's factors, with the two scale factors undone
        float ws[K::NS];
        {
            const float f = fsc * inv_ke;
#pragma unroll
            for (int s = 0; s < K::NS; ++s) {
                const int sy = s % N, sx = (s / N) % N, sz = s / (N * N);
                ws[s] = factor_value(wslab[((lz * N + sz) * K::WX + lx * N + sx) * K::WY + ly * N + sy]) * f;
            }
        }
        float2 acc[12];
#pragma unroll
        for (int i = 0; i < 12; ++i) acc[i] = make_float2(0.f, 0.f);

        bool ok = true;
#pragma unroll
        for (int c = 0; c < K::NCH; ++c) {
            // warp-uniform, so that the collective tensor-memory loads below
            // are executed by all or none of a warp's threads
            const bool got = __all_sync(0xffffffffu, (c & 1) ? mbar_wait(mbar1, ph1) : mbar_wait(mbar0, ph0));
            if (c & 1) ph1 ^= 1u;
            else ph0 ^= 1u;
            if (got) {
                fence_after();
                consume_any<N>(c, tlane + (uint32_t)((c & 1) * K::CH), ws, acc,
                               std::make_integer_sequence<int, K::NCH>{});
            }
            fence_before();
            if (group_sync_or(grp, !got)) {   // buffer (c & 1) fully read
                ok = false;
                break;
            }
            if (c == 0) {
                // past this barrier every thread of the group has read this
                // brick's factors and the A tiles were built: the next brick's
                // inputs go into the same buffers
                if (next < fg.nbricks) stage_brick<N, WT>(next, xs, wslab, x, w, fg, rel, pk, tid);
                cp_async_commit();
            }
            if (tid == 0 && c + 2 < K::NCH) {
                fence_after();
                issue_chunk<N, WT>(c + 2, tmem, a_addr, b_addr, (c & 1) ? mbar1 : mbar0);
            }
        }
        if (!ok) {
            if (tid == 0) {
                s_fail[grp] = 1;
                atomicExch(err, 1);
            }
            break;
        }
        // this element's corner outputs (zero outside the mesh); every thread
        // of the group finished the previous brick's gathers before the first
        // chunk's barrier
#pragma unroll
        for (int a = 0; a < 8; ++a)
            eo4[a * BRICK_ELEMS + tid] = valid ? make_float4(acc_at(acc, 3 * a), acc_at(acc, 3 * a + 1),
                                                             acc_at(acc, 3 * a + 2), 0.f)
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
        // every MMA of this brick has completed: the A tiles are free.  The
        // next brick's inputs and the corner outputs are complete and visible
        // after the barrier.
        cp_async_wait_0();
        group_sync(grp);
        if (next < fg.nbricks) {
            fsc = build_a<K::K3>(xs, abuf, ln0, tid);
            fence_async_smem();
        }
        group_sync(grp);
        if (tid == 0 && next < fg.nbricks) {
            fence_after();
            issue_chunk<N, WT>(0, tmem, a_addr, b_addr, mbar0);
            if (K::NCH > 1) issue_chunk<N, WT>(1, tmem, a_addr, b_addr, mbar1);
        }
        brick_gather_write(eo4, y, freemask, g, ex0, ey0, ez0, rel, pk, tid, chk);
    }
    cp_async_wait_0();

    // MMAs still in flight after a timeout get one more bounded wait each
    // before their columns are released.
    if (tid == 0 && s_fail[grp]) {
        mbar_wait(mbar0, ph0);
        if (K::NCH > 1) mbar_wait(mbar1, ph1);
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (ttid < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(K::TMEM_COLS)
                     : "memory");
}

// B image: step tiles of the scaled blocks' FP16 pieces in the K order of the
// MMAs above (row r = 24 s + i, entry KE_s[i][j] at k = j, j - 16 + 8 or j - 8
// as the step requires; rows beyond 24 n^3 zero), then the block scale record:
// the float 2^-sc in the first four bytes.  Steps 0-2 hold the hi piece against
// A = [u_hi u_lo].  Two-piece image: steps 3-4 the mid piece against u_hi
// (step 4: entries j >= 16 only).  Three-piece image: steps 3-5 the mid piece
// against [u_hi u_lo], steps 6-7 the lo piece (the rest v - hi - mid, rounded)
// against u_hi.  Two pieces carry about 22 bits of each block entry relative
// to the largest; that truncation, and the dropped u_lo * mid product, change
// the operator by about 2^-22 |KE| |u_e|, which slows a CG whose recurrence
// uses it (110 -> 173 iterations on the 192 x 96 x 96 MR-2 workload; the
// V-cycle tolerates it), so the CG's kernel for n = 1, 2 takes three pieces
// and five products (hi*hi, lo*hi, hi*mid, lo*mid, hi*lo); for n = 3 the
// two-piece image with the translation removed costs fewer solve seconds.
static uint16_t f16_bits(float v) {
    const __half h = __float2half_rn(v);
    uint16_t b;
    memcpy(&b, &h, 2);
    return b;
}
static double f16_value(uint16_t b) {
    __half h;
    memcpy(&h, &b, 2);
    return (double)__half2float(h);
}

template <int N, typename WT>
static void tc_image(const std::vector<double> &packed_rowmajor, std::vector<uint16_t> &img) {
    using K = Tc<N, WT>;
    auto ke = [&](int s, int i, int j) {
        const int a = i < j ? i : j, b = i < j ? j : i;
        return packed_rowmajor[(size_t)s * KE_PACK + pair_rowmajor(a, b)];
    };
    double kmax = 0.0;
    for (int s = 0; s < K::NS; ++s)
        for (int t = 0; t < KE_PACK; ++t) kmax = fmax(kmax, fabs(packed_rowmajor[(size_t)s * KE_PACK + t]));
    int e = 0;
    frexp(kmax > 0.0 ? kmax : 1.0, &e);
    const int sc = 15 - e;   // kmax 2^sc in [2^14, 2^15)
    img.assign((K::B_BYTES + 16) / 2, 0);   // + the block scale record
    auto put = [&](int step, int r, int k, uint16_t b) { img[(step * K::B_TILE + tc_offset(r, k)) / 2] = b; };
    for (int r = 0; r < K::NROWS; ++r) {
        const int s = r / 24, i = r % 24;
        for (int j = 0; j < 24; ++j) {
            const double v = ldexp(ke(s, i, j), sc);
            const uint16_t hi = f16_bits((float)v);
            const uint16_t mid = f16_bits((float)(v - f16_value(hi)));
            if (j < 16) put(0, r, j, hi);
            else put(1, r, j - 16, hi);
            if (j < 8) put(1, r, j + 8, hi);
            else put(2, r, j - 8, hi);
            if (K::B_STEPS == 5) {
                if (j < 16) put(3, r, j, mid);
                else put(4, r, j - 16, mid);
            } else {
                if (j < 16) put(3, r, j, mid);
                else put(4, r, j - 16, mid);
                if (j < 8) put(4, r, j + 8, mid);
                else put(5, r, j - 8, mid);
                const uint16_t lo = f16_bits((float)(v - f16_value(hi) - f16_value(mid)));
                if (j < 16) put(6, r, j, lo);
                else put(7, r, j - 16, lo);
            }
        }
    }
    const float inv = (float)ldexp(1.0, -sc);
    memcpy(&img[K::B_BYTES / 2], &inv, sizeof(float));
}

bool fine_tc_supported(int n, int nely) { return n >= 1 && n <= 3 && (n * nely) % 2 == 0; }

void fine_tc_image(const std::vector<double> &packed_rowmajor, int n, std::vector<uint16_t> &img) {
    if (n == 1) tc_image<1, __nv_bfloat16>(packed_rowmajor, img);
    else if (n == 2) tc_image<2, __nv_bfloat16>(packed_rowmajor, img);
    else tc_image<3, __nv_bfloat16>(packed_rowmajor, img);
}

void fine_tc_image_w32(const std::vector<double> &packed_rowmajor, int n, std::vector<uint16_t> &img) {
    if (n == 1) tc_image<1, float>(packed_rowmajor, img);
    else if (n == 2) tc_image<2, float>(packed_rowmajor, img);
    else tc_image<3, float>(packed_rowmajor, img);
}

// Resident CTAs per SM from the device limits (shared memory with the
// per-CTA reservation, registers at warp allocation granularity), capped by
// the 512 tensor-memory columns.
template <int N, typename WT>
static int tc_ctas_per_sm() {
    int dev = 0, smem_sm = 0, smem_res = 0, regs_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, k_fine_apply_tc<N, WT>) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    using K = Tc<N, WT>;
    const size_t per_cta = K::SMEM + fa.sharedSizeBytes + (size_t)smem_res;
    const int by_smem = (int)(smem_sm / per_cta);
    const int regs_warp = (fa.numRegs * 32 + 255) / 256 * 256;
    const int by_regs = regs_sm / (regs_warp * (K::THREADS / 32));
    int m = by_smem < by_regs ? by_smem : by_regs;
    if (m > 512 / K::TMEM_COLS) m = 512 / K::TMEM_COLS;
    return m < 1 ? 1 : m;
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

template <int N, typename WT>
static void launch_tc(const float *x, float *y, const WT *w, const uint8_t *fm, const void *bimg,
                      const FineGeom &fg, int *err, cudaStream_t st) {
    using K = Tc<N, WT>;
    static int attr_dev = -1, per_sm = 1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaFuncSetAttribute(k_fine_apply_tc<N, WT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::SMEM);
        cudaFuncSetAttribute(k_fine_apply_tc<N, WT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        per_sm = tc_ctas_per_sm<N, WT>();
        attr_dev = dev;
    }
    int64_t grid = (int64_t)per_sm * num_sms_tc();
    const int64_t need = (fg.nbricks + K::NB - 1) / K::NB;   // NB bricks side by side per CTA
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    k_fine_apply_tc<N, WT><<<(unsigned)grid, K::THREADS, K::SMEM, st>>>(x, y, w, fm, (const uint4 *)bimg, fg, err);
    count_launch();
}

void launch_fine_apply_tc(const float *x, float *y, const __nv_bfloat16 *w, const uint8_t *fm, const void *bimg,
                          const FineGeom &fg, int n, int *err, cudaStream_t st) {
    if (n == 1) launch_tc<1>(x, y, w, fm, bimg, fg, err, st);
    else if (n == 2) launch_tc<2>(x, y, w, fm, bimg, fg, err, st);
    else launch_tc<3>(x, y, w, fm, bimg, fg, err, st);
}

bool fine_tc_w32_supported(int n) { return n >= 1 && n <= 3; }

void launch_fine_apply_tc_w32(const float *x, float *y, const float *w, const uint8_t *fm, const void *bimg,
                              const FineGeom &fg, int n, int *err, cudaStream_t st) {
    if (n == 1) launch_tc<1>(x, y, w, fm, bimg, fg, err, st);
    else if (n == 2) launch_tc<2>(x, y, w, fm, bimg, fg, err, st);
    else launch_tc<3>(x, y, w, fm, bimg, fg, err, st);
}

}  // namespace tosp
