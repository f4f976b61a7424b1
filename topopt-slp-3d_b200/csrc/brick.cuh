// Node accumulation and write-out of a BX x BY x BZ element brick, shared by
// the finest-level operator kernels.
//
// The brick's (BX+1)(BY+1)(BZ+1) nodes hold three values each in shared
// memory (ys, y fastest, the layout of the staged inputs).  Element outputs
// are added corner by corner: in pass a every element adds its corner-a
// values to the node at offset a from its base node, and no two elements of
// one pass reach the same node, so plain read-modify-writes separated by
// barriers give each node the deterministic sum over corners 0..7.  The
// write-out stores nodes that only this brick touches and adds the brick's
// face nodes atomically; fixed dofs are skipped.
#pragma once

#include "tosp_internal.h"

namespace tosp {

__device__ __forceinline__ void brick_atomic_add(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void brick_atomic_add(float *p, float v) { atomicAdd(p, v); }

// Brick coordinates of brick b (y fastest); bricks number far below 2^31.
__device__ __forceinline__ void brick_xyz(int64_t b, const FineGeom &fg, int &bx, int &by, int &bz) {
    const int i = (int)b, q = i / fg.nby;
    by = i - q * fg.nby;
    bz = q / fg.nbx;
    bx = q - bz * fg.nbx;
}

// Whether brick b's write-out must read the free-dof mask.
__device__ __forceinline__ bool brick_check_fixed(int64_t b, const FineGeom &fg) {
    return fg.bfix == nullptr || fg.bfix[b] != 0;
}

// Base node of thread tid's element within the brick.
__device__ __forceinline__ int brick_base_node(int tid) {
    const int ly = tid % BY, lx = (tid / BY) % BX, lz = tid / (BY * BX);
    return (lz * NBX + lx) * NBY + ly;
}

// Adds acc (24 values, local node a = dz*4 + dx*2 + dy, 3 components each)
// into ys.  Every thread of the CTA must call it (it contains barriers);
// ys must be zero on entry and is complete on return.
template <typename T>
__device__ __forceinline__ void brick_accumulate(T *ys, const T (&acc)[24], bool valid, int ln0) {
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
        const int ln = ln0 + (dz * NBX + dx) * NBY + dy;
        if (valid) {
            ys[3 * ln] += acc[3 * a];
            ys[3 * ln + 1] += acc[3 * a + 1];
            ys[3 * ln + 2] += acc[3 * a + 2];
        }
        __syncthreads();
    }
}

// Same with the brick's nodes padded to float4 (ys4[ln] = (x, y, z, -)): one
// vector read-modify-write per corner.
__device__ __forceinline__ void brick_accumulate4(float4 *ys4, const float (&acc)[24], bool valid, int ln0) {
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
        const int ln = ln0 + (dz * NBX + dx) * NBY + dy;
        if (valid) {
            float4 v = ys4[ln];
            v.x += acc[3 * a];
            v.y += acc[3 * a + 1];
            v.z += acc[3 * a + 2];
            ys4[ln] = v;
        }
        __syncthreads();
    }
}

// FP64 nodes padded to 4 values: a 16-byte pair and a scalar per corner.
__device__ __forceinline__ void brick_accumulate_pad(double *ys, const double (&acc)[24], bool valid, int ln0) {
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
        const int ln = ln0 + (dz * NBX + dx) * NBY + dy;
        if (valid) {
            double2 v = reinterpret_cast<double2 *>(ys)[2 * ln];
            v.x += acc[3 * a];
            v.y += acc[3 * a + 1];
            reinterpret_cast<double2 *>(ys)[2 * ln] = v;
            ys[4 * ln + 2] += acc[3 * a + 2];
        }
        __syncthreads();
    }
}

constexpr int BRICK_SLOTS = BRICK_NODES * 3;

// Per-CTA table of the brick's node-value slots (i = 3 * local node + c):
// offset of slot i from the brick's first dof, and its local node coordinates
// packed as bits 0-2 x, 3-6 y, 7-9 z, bit 10 set when only this brick touches
// the node.  Built once per CTA; valid for every brick of the grid.
__device__ __forceinline__ void brick_slots_init(int32_t *rel, uint16_t *pk, const Grid &g, int tid) {
    for (int i = tid; i < BRICK_SLOTS; i += BRICK_ELEMS) {
        const int ln = i / 3, c = i - 3 * ln;
        const int ny_ = ln % NBY, nx_ = (ln / NBY) % NBX, nz_ = ln / (NBY * NBX);
        rel[i] = 3 * ((nz_ * g.nx + nx_) * g.ny + ny_) + c;
        const bool inner = nx_ > 0 && nx_ < BX && ny_ > 0 && ny_ < BY && nz_ > 0 && nz_ < BZ;
        pk[i] = (uint16_t)(nx_ | (ny_ << 3) | (nz_ << 7) | (inner ? 1 << 10 : 0));
    }
}

// All nodes of the brick with first element (ex0, ey0, ez0) lie in the mesh.
__device__ __forceinline__ bool brick_interior(int ex0, int ey0, int ez0, const Grid &g) {
    return ex0 + BX < g.nx && ey0 + BY < g.ny && ez0 + BZ < g.nz;
}

__device__ __forceinline__ bool brick_slot_in(uint16_t p, int ex0, int ey0, int ez0, const Grid &g) {
    return ex0 + (p & 7) < g.nx && ey0 + ((p >> 3) & 15) < g.ny && ez0 + ((p >> 7) & 7) < g.nz;
}

__device__ __forceinline__ int64_t brick_base_dof(int ex0, int ey0, int ez0, const Grid &g) {
    return 3 * (((int64_t)ez0 * g.nx + ex0) * g.ny + ey0);
}

// Write-out through the slot table; NP values per node in ys (3, or 4 when
// the nodes are padded).  check = false: no node of the brick has a fixed
// dof, so the free-dof mask is not read.
template <typename T, int NP = 3>
__device__ __forceinline__ void brick_writeout_tab(const T *ys, T *__restrict__ y, const uint8_t *__restrict__ freemask,
                                                   const Grid &g, int ex0, int ey0, int ez0, const int32_t *rel,
                                                   const uint16_t *pk, int tid, bool check = true) {
    const int64_t base = brick_base_dof(ex0, ey0, ez0, g);
    const bool interior = brick_interior(ex0, ey0, ez0, g);
    for (int i = tid; i < BRICK_SLOTS; i += BRICK_ELEMS) {
        const uint16_t p = pk[i];
        if (!interior && !brick_slot_in(p, ex0, ey0, ez0, g)) continue;
        const int64_t dof = base + rel[i];
        if (!check || freemask[dof]) {
            const T v = ys[NP == 3 ? i : i + i / 3];
            if (p >> 10) y[dof] = v;
            else brick_atomic_add(&y[dof], v);
        }
    }
}

// The same write-out node by node, for nodes padded to four values in ys:
// one slot-table lookup, one range test and one address per node instead of
// per value (BRICK_NODES / BRICK_ELEMS = 1.8 trips per thread instead of 5.3).
template <typename T>
__device__ __forceinline__ void brick_writeout_nodes(const T *ys, T *__restrict__ y,
                                                     const uint8_t *__restrict__ freemask, const Grid &g, int ex0,
                                                     int ey0, int ez0, const int32_t *rel, const uint16_t *pk, int tid,
                                                     bool check) {
    const int64_t base = brick_base_dof(ex0, ey0, ez0, g);
    const bool interior = brick_interior(ex0, ey0, ez0, g);
    for (int ln = tid; ln < BRICK_NODES; ln += BRICK_ELEMS) {
        const uint16_t p = pk[3 * ln];
        if (!interior && !brick_slot_in(p, ex0, ey0, ez0, g)) continue;
        const int64_t dof = base + rel[3 * ln];
        const T v[3] = {ys[4 * ln], ys[4 * ln + 1], ys[4 * ln + 2]};
        if constexpr (sizeof(T) == 4) {
            if (!check) {
                // FP32: one 8-byte access for the two of the node's three values
                // that share an 8-byte-aligned pair (decided from the address)
                // and one 4-byte access for the third
                float *a = reinterpret_cast<float *>(y + dof);
                const bool lo = (reinterpret_cast<uintptr_t>(a) & 7u) == 0;
                float *pair = lo ? a : a + 1;
                float *one = lo ? a + 2 : a;
                const float p0 = lo ? v[0] : v[1], p1 = lo ? v[1] : v[2], s1 = lo ? v[2] : v[0];
                if (p >> 10) {
                    asm volatile("st.global.v2.f32 [%0], {%1, %2};" ::"l"(pair), "f"(p0), "f"(p1) : "memory");
                    *one = s1;
                } else {
                    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(pair), "f"(p0), "f"(p1) : "memory");
                    atomicAdd(one, s1);
                }
                continue;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (check && !freemask[dof + c]) continue;
            if (p >> 10) y[dof + c] = v[c];
            else brick_atomic_add(&y[dof + c], v[c]);
        }
    }
}

// Node sums gathered from per-element corner outputs (eo4[a * BRICK_ELEMS + e]
// = element e's values at its corner a, zero for elements outside the mesh)
// and written out node by node.  Each node adds its contributions in corner
// order 0..7, the order of brick_accumulate4, so the sums are the same; one
// barrier (eo4 complete) replaces the eight of the corner passes.
__device__ __forceinline__ void brick_gather_write(const float4 *eo4, float *__restrict__ y,
                                                   const uint8_t *__restrict__ freemask, const Grid &g, int ex0,
                                                   int ey0, int ez0, const int32_t *rel, const uint16_t *pk, int tid,
                                                   bool check) {
    const int64_t base = brick_base_dof(ex0, ey0, ez0, g);
    const bool interior = brick_interior(ex0, ey0, ez0, g);
    for (int ln = tid; ln < BRICK_NODES; ln += BRICK_ELEMS) {
        const uint16_t p = pk[3 * ln];
        if (!interior && !brick_slot_in(p, ex0, ey0, ez0, g)) continue;
        const int ny_ = ln % NBY, nx_ = (ln / NBY) % NBX, nz_ = ln / (NBY * NBX);
        float v0 = 0.f, v1 = 0.f, v2 = 0.f;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int dx = (a >> 1) & 1, dy = a & 1, dz = (a >> 2) & 1;
            const int lx = nx_ - dx, ly = ny_ - dy, lz = nz_ - dz;
            if (lx >= 0 && lx < BX && ly >= 0 && ly < BY && lz >= 0 && lz < BZ) {
                const float4 c = eo4[a * BRICK_ELEMS + (lz * BX + lx) * BY + ly];
                v0 += c.x;
                v1 += c.y;
                v2 += c.z;
            }
        }
        const int64_t dof = base + rel[3 * ln];
        const float v[3] = {v0, v1, v2};
        if (!check) {
            // one 8-byte access for the two of the node's three values that
            // share an 8-byte-aligned pair (decided from the address) and one
            // 4-byte access for the third
            float *a = y + dof;
            const bool lo = (reinterpret_cast<uintptr_t>(a) & 7u) == 0;
            float *pair = lo ? a : a + 1;
            float *one = lo ? a + 2 : a;
            const float p0 = lo ? v[0] : v[1], p1 = lo ? v[1] : v[2], s1 = lo ? v[2] : v[0];
            if (p >> 10) {
                asm volatile("st.global.v2.f32 [%0], {%1, %2};" ::"l"(pair), "f"(p0), "f"(p1) : "memory");
                *one = s1;
            } else {
                asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(pair), "f"(p0), "f"(p1) : "memory");
                atomicAdd(one, s1);
            }
            continue;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (!freemask[dof + c]) continue;
            if (p >> 10) y[dof + c] = v[c];
            else atomicAdd(&y[dof + c], v[c]);
        }
    }
}

template <typename T>
__device__ __forceinline__ void brick_writeout(const T *ys, T *__restrict__ y, const uint8_t *__restrict__ freemask,
                                               const Grid &g, int ex0, int ey0, int ez0, int tid) {
    for (int i = tid; i < BRICK_NODES * 3; i += BRICK_ELEMS) {
        const int ln = i / 3, c = i - 3 * ln;
        const int ny_ = ln % NBY, nx_ = (ln / NBY) % NBX, nz_ = ln / (NBY * NBX);
        const int gx = ex0 + nx_, gy = ey0 + ny_, gz = ez0 + nz_;
        if (gx < g.nx && gy < g.ny && gz < g.nz) {
            const int64_t dof = 3 * (((int64_t)gz * g.nx + gx) * g.ny + gy) + c;
            if (freemask[dof]) {
                const bool inner = nx_ > 0 && nx_ < BX && ny_ > 0 && ny_ < BY && nz_ > 0 && nz_ < BZ;
                if (inner) y[dof] = ys[i];
                else brick_atomic_add(&y[dof], ys[i]);
            }
        }
    }
}

}  // namespace tosp
