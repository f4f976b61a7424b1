// Finest-level operator of the mixed-precision V-cycle, MR factor 2, on the
// 5th-generation tensor cores.
//
// y_e = sum_s w_s KE_s u_e (I/WOK/KelemProd.m:57-100).  For a brick of 128
// elements the products of the eight shared 24x24 sub-cell blocks with every
// element's nodal vector are one GEMM (M = 128 elements, N = 8 x 24 = 192 block
// rows, K = 24 element dofs, kind::f16, FP32 accumulator):
//
//     D[e][24 s + i] = sum_j KE_s[i][j] u_e[j],
//
// and each thread weights its element's 192 values with the element's eight
// SIMP factors on the CUDA cores (192 FMAs per element):
//
//     y_e[i] = sum_s w_s D[e][24 s + i].
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
// Pipelining inside a CTA: the 192 accumulator columns are produced in three
// 64-column chunks through two tensor-memory buffers, so the MMAs of chunk
// c+1 run while the threads consume chunk c.  Once the first chunk is read
// (every thread then holds the brick's factors and the A tiles are built), the
// next brick's nodal values and factors are staged with cp.async into the same
// buffers; once the last chunk is read, the A tiles are rebuilt for the next
// brick and that brick's first two chunks run during the current brick's node
// sums and write-out.  Single node, factor and A buffers keep a CTA at 55 KB of
// shared memory, so four CTAs (4 x 128 tensor-memory columns) share an SM.
// Every wait on an MMA-completion barrier is bounded; a timeout sets *err,
// leaves the brick loop and still frees the tensor memory.  Node sums and the
// write-out are those of the CUDA-core kernels (brick.cuh).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "brick.cuh"
#include "tosp_internal.h"

namespace tosp {

namespace {

constexpr int TC_K = 16;                                  // K of every MMA (kind::f16)
constexpr int TC_NROWS = 192;                             // B rows: 8 sub-cells x 24 block rows
constexpr int TC_GROUP = 8 * TC_K * 2;                    // bytes of one 8-row group (256)
constexpr int TC_B_TILE = TC_NROWS / 8 * TC_GROUP;        // 6144 per B step
constexpr int TC_B_STEPS = 5;
constexpr int TC_B_BYTES = TC_B_STEPS * TC_B_TILE;        // 30720
constexpr int TC_IMG_BYTES = TC_B_BYTES + 16;             // + the block scale record
constexpr int TC_A_TILE = BRICK_ELEMS / 8 * TC_GROUP;     // 4096 per A step
constexpr int TC_A_BYTES = 3 * TC_A_TILE;
constexpr int TC_XS_FLOATS = BRICK_NODES * 4;             // 900: nodes padded to float4
constexpr int TC_EO_BYTES = 8 * BRICK_ELEMS * 16;         // element outputs: one float4 per corner
constexpr int TC_W_BYTES = BRICK_ELEMS * 16;              // eight BF16 factors per element
constexpr int TC_SLOTS_PAD = (BRICK_SLOTS + 3) / 4 * 4;   // slot table length
constexpr int TC_CHUNK = 64;
constexpr int TC_NCHUNK = TC_NROWS / TC_CHUNK;            // 3
constexpr int TC_COLS = 2 * TC_CHUNK;                     // tensor-memory columns per CTA
constexpr int TC_CTAS_PER_SM = 512 / TC_COLS;
constexpr uint32_t TC_WAIT_LIMIT = 1u << 16;              // try_wait rounds before giving up
constexpr uint32_t TC_SUSPEND_NS = 20000;                 // suspend-time hint of one try_wait round

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
// code 0), both K-major, M = 128.
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

// 64 consecutive columns of this warp's 32 lanes (one column per register).
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&r)[64]) {
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

// Chunk C holds block rows 64C..64C+63: row n is entry i = n % 24 of
// sub-cell s = n / 24.  Columns t, t+1 (t even) are entries i, i+1 of the
// same sub-cell, weighted by one packed FMA (two FP32 FMAs, same rounding).
template <int C>
__device__ __forceinline__ void consume_chunk(uint32_t taddr, const float2 (&ws2)[8], float2 (&acc)[12]) {
    uint32_t r[64];
    tmem_ld64(taddr, r);
#pragma unroll
    for (int t = 0; t < TC_CHUNK; t += 2) {
        const int n = C * TC_CHUNK + t;
        acc[(n % 24) / 2] = __ffma2_rn(ws2[n / 24], make_float2(__uint_as_float(r[t]), __uint_as_float(r[t + 1])),
                                       acc[(n % 24) / 2]);
    }
}

// The five MMAs of chunk c into tensor-memory buffer (c & 1), then a commit to
// its barrier.
__device__ __forceinline__ void issue_chunk(int c, uint32_t tmem, uint32_t a_addr, uint32_t b_addr, uint32_t mbar) {
    const uint32_t d = tmem + (uint32_t)((c & 1) * TC_CHUNK);
    const uint32_t boff = (uint32_t)(c * TC_CHUNK / 8 * TC_GROUP);
    constexpr uint32_t id = idesc_f16(TC_CHUNK);
    mma_f16(d, smem_desc(a_addr), smem_desc(b_addr + boff), id, 0u);
    mma_f16(d, smem_desc(a_addr + TC_A_TILE), smem_desc(b_addr + TC_B_TILE + boff), id, 1u);
    mma_f16(d, smem_desc(a_addr + 2 * TC_A_TILE), smem_desc(b_addr + 2 * TC_B_TILE + boff), id, 1u);
    mma_f16(d, smem_desc(a_addr), smem_desc(b_addr + 3 * TC_B_TILE + boff), id, 1u);
    mma_f16(d, smem_desc(a_addr + TC_A_TILE), smem_desc(b_addr + 4 * TC_B_TILE + boff), id, 1u);
    mma_commit(mbar);
}

// Entry i of the 24 element outputs held as 12 pairs.
__device__ __forceinline__ float acc_at(const float2 (&acc)[12], int i) { return (i & 1) ? acc[i >> 1].y : acc[i >> 1].x; }

__device__ __forceinline__ uint32_t half2_bits(__half2 h) {
    uint32_t b;
    memcpy(&b, &h, 4);
    return b;
}

}  // namespace

// Dynamic shared memory: the B image, the A tiles, the staged nodal values,
// the node sums, the factors and the brick slot table.  The MMA
// operands need 16-byte aligned starts; the barriers and the tensor-memory
// address are static (8-byte aligned) shared variables.
constexpr size_t TC_OFF_A = TC_B_BYTES;
constexpr size_t TC_OFF_XS = TC_OFF_A + TC_A_BYTES;
constexpr size_t TC_OFF_EO = TC_OFF_XS + sizeof(float) * TC_XS_FLOATS;
constexpr size_t TC_OFF_W = TC_OFF_EO + TC_EO_BYTES;
constexpr size_t TC_OFF_REL = TC_OFF_W + TC_W_BYTES;
constexpr size_t TC_OFF_PK = TC_OFF_REL + sizeof(int32_t) * TC_SLOTS_PAD;
constexpr size_t TC_SMEM = (TC_OFF_PK + sizeof(uint16_t) * TC_SLOTS_PAD + 127) / 128 * 128;
static_assert(TC_OFF_A % 16 == 0 && TC_OFF_XS % 16 == 0 && TC_OFF_EO % 16 == 0 && TC_OFF_W % 16 == 0,
              "operand alignment");
static_assert(TC_OFF_REL % 4 == 0 && TC_OFF_PK % 2 == 0, "slot table alignment");
static_assert(TC_NCHUNK * TC_CHUNK == TC_NROWS && TC_NCHUNK == 3, "three chunks through two buffers");

// Stage brick `brick` (nodal values, SIMP factors) with cp.async.
__device__ __forceinline__ void stage_brick(int64_t brick, float *xs, unsigned char *wbuf, const float *__restrict__ x,
                                            const __nv_bfloat16 *__restrict__ w, const FineGeom &fg,
                                            const int32_t *rel, const uint16_t *pk, int tid) {
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
    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    const int ex = ex0 + lx, ey = ey0 + ly, ez = ez0 + lz;
    const bool valid = ex < g.nelx && ey < g.nely && ez < g.nelz;
    unsigned char *wr = wbuf + 16 * tid;
    const __nv_bfloat16 *wb = w + ((int64_t)(ez * 2) * fg.nelx_d + ex * 2) * fg.nely_d + ey * 2;
#pragma unroll
    for (int s = 0; s < 8; s += 2) {
        // sub-cubes s and s+1 differ in y only: adjacent in the density mesh
        const int sx = (s >> 1) & 1, sz = s >> 2;
        const __nv_bfloat16 *src = valid ? wb + ((int64_t)sz * fg.nelx_d + sx) * fg.nely_d : w;
        cp_async4(wr + 2 * s, src, valid ? 4 : 0);
    }
}

// A tiles of this thread's element (row tid) from the staged nodal values;
// returns 2^(E - 140), the inverse of the element's scale factor.
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

__global__ void __launch_bounds__(BRICK_ELEMS, 4)
k_fine_apply_tc2(const float *__restrict__ x, float *__restrict__ y, const __nv_bfloat16 *__restrict__ w,
                 const uint8_t *__restrict__ freemask, const uint4 *__restrict__ bimg, FineGeom fg,
                 int *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float *xs = reinterpret_cast<float *>(smem_raw + TC_OFF_XS);          // staged nodal values
    float4 *eo4 = reinterpret_cast<float4 *>(smem_raw + TC_OFF_EO);       // element outputs per corner
    unsigned char *abuf = smem_raw + TC_OFF_A;
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
    const float inv_ke = reinterpret_cast<const float *>(bimg)[TC_B_BYTES / 4];   // undoes the block scale
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
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);    // this warp's 32 lanes
    const uint32_t mbar0 = smem_u32(&s_mbar[0]), mbar1 = smem_u32(&s_mbar[1]);
    const uint32_t b_addr = smem_u32(smem_raw);
    const uint32_t a_addr = smem_u32(abuf);
    uint32_t ph0 = 0, ph1 = 0;

    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    const int ln0 = brick_base_node(tid);

    // Prologue: the first brick's inputs and A tiles, then its first two
    // chunks.  The grid never exceeds the brick count.
    stage_brick(blockIdx.x, xs, smem_raw + TC_OFF_W, x, w, fg, rel, pk, tid);
    cp_async_commit();
    cp_async_wait_0();
    __syncthreads();
    float fsc = build_a(xs, abuf, ln0, tid);
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
        fence_after();
        issue_chunk(0, tmem, a_addr, b_addr, mbar0);
        issue_chunk(1, tmem, a_addr, b_addr, mbar1);
    }

    for (int64_t brick = blockIdx.x; brick < fg.nbricks; brick += gridDim.x) {
        const int64_t next = brick + gridDim.x;
        const bool chk = brick_check_fixed(brick, fg);

        int bbx, bby, bbz;
        brick_xyz(brick, fg, bbx, bby, bbz);
        const int ex0 = bbx * BX, ey0 = bby * BY, ez0 = bbz * BZ;
        const bool valid = ex0 + lx < g.nelx && ey0 + ly < g.nely && ez0 + lz < g.nelz;

        float2 ws2[8], acc[12];
        {
            const uint4 wv = *reinterpret_cast<const uint4 *>(smem_raw + TC_OFF_W + 16 * tid);
            const uint32_t wq[4] = {wv.x, wv.y, wv.z, wv.w};
            const float f = fsc * inv_ke;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float w0 = __uint_as_float(wq[q] << 16) * f, w1 = __uint_as_float(wq[q] & 0xFFFF0000u) * f;
                ws2[2 * q] = make_float2(w0, w0);
                ws2[2 * q + 1] = make_float2(w1, w1);
            }
        }
#pragma unroll
        for (int i = 0; i < 12; ++i) acc[i] = make_float2(0.f, 0.f);

        bool ok = true;
#pragma unroll
        for (int c = 0; c < TC_NCHUNK; ++c) {
            // warp-uniform, so that the collective tensor-memory loads below
            // are executed by all or none of a warp's threads
            const bool got = __all_sync(0xffffffffu, (c & 1) ? mbar_wait(mbar1, ph1) : mbar_wait(mbar0, ph0));
            if (c & 1) ph1 ^= 1u;
            else ph0 ^= 1u;
            if (got) {
                fence_after();
                const uint32_t taddr = tlane + (uint32_t)((c & 1) * TC_CHUNK);
                if (c == 0) consume_chunk<0>(taddr, ws2, acc);
                else if (c == 1) consume_chunk<1>(taddr, ws2, acc);
                else consume_chunk<2>(taddr, ws2, acc);
            }
            fence_before();
            if (__syncthreads_or(!got)) {   // buffer (c & 1) fully read
                ok = false;
                break;
            }
            if (c == 0) {
                // past this barrier every thread has read this brick's factors
                // and the A tiles were built: the next brick's inputs go into
                // the same buffers
                if (next < fg.nbricks) stage_brick(next, xs, smem_raw + TC_OFF_W, x, w, fg, rel, pk, tid);
                cp_async_commit();
                if (tid == 0) {
                    fence_after();
                    issue_chunk(2, tmem, a_addr, b_addr, mbar0);
                }
            }
        }
        if (!ok) {
            if (tid == 0) {
                s_fail = 1;
                atomicExch(err, 1);
            }
            break;
        }
        // this element's corner outputs (zero outside the mesh); every thread
        // finished the previous brick's gathers before the first chunk's barrier
#pragma unroll
        for (int a = 0; a < 8; ++a)
            eo4[a * BRICK_ELEMS + tid] = valid ? make_float4(acc_at(acc, 3 * a), acc_at(acc, 3 * a + 1),
                                                             acc_at(acc, 3 * a + 2), 0.f)
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
        // every MMA of this brick has completed: the A tiles are free.  The
        // next brick's inputs and the corner outputs are complete and visible
        // after the barrier.
        cp_async_wait_0();
        __syncthreads();
        if (next < fg.nbricks) {
            fsc = build_a(xs, abuf, ln0, tid);
            fence_async_smem();
        }
        __syncthreads();
        if (tid == 0 && next < fg.nbricks) {
            fence_after();
            issue_chunk(0, tmem, a_addr, b_addr, mbar0);
            issue_chunk(1, tmem, a_addr, b_addr, mbar1);
        }
        brick_gather_write(eo4, y, freemask, g, ex0, ey0, ez0, rel, pk, tid, chk);
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

// B image for MR factor 2: step tiles of the scaled blocks' FP16 hi and mid
// pieces in the K order of the MMAs above (row n = 24 s + i, entry KE_s[i][j]
// at k = j, j - 16 + 8 or j - 8 as the step requires), then the block scale
// record: the float 2^-sc in the first four bytes.
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

void fine_tc_image(const std::vector<double> &packed_rowmajor, std::vector<uint16_t> &img) {
    auto ke = [&](int s, int i, int j) {
        const int a = i < j ? i : j, b = i < j ? j : i;
        return packed_rowmajor[(size_t)s * KE_PACK + pair_rowmajor(a, b)];
    };
    double kmax = 0.0;
    for (int s = 0; s < 8; ++s)
        for (int t = 0; t < KE_PACK; ++t) kmax = fmax(kmax, fabs(packed_rowmajor[(size_t)s * KE_PACK + t]));
    int e = 0;
    frexp(kmax > 0.0 ? kmax : 1.0, &e);
    const int sc = 15 - e;   // kmax 2^sc in [2^14, 2^15)
    img.assign(TC_IMG_BYTES / 2, 0);
    auto put = [&](int step, int n, int k, uint16_t b) { img[(step * TC_B_TILE + tc_offset(n, k)) / 2] = b; };
    for (int n = 0; n < TC_NROWS; ++n) {
        const int s = n / 24, i = n % 24;
        for (int j = 0; j < 24; ++j) {
            const double v = ldexp(ke(s, i, j), sc);
            const uint16_t hi = f16_bits((float)v);
            const uint16_t mid = f16_bits((float)(v - f16_value(hi)));
            if (j < 16) put(0, n, j, hi);
            else put(1, n, j - 16, hi);
            if (j < 8) put(1, n, j + 8, hi);
            else put(2, n, j - 8, hi);
            if (j < 16) put(3, n, j, mid);
            else put(4, n, j - 16, mid);
        }
    }
    const float inv = (float)ldexp(1.0, -sc);
    memcpy(&img[TC_B_BYTES / 2], &inv, sizeof(float));
}

size_t fine_tc_image_bytes() { return TC_IMG_BYTES; }

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
