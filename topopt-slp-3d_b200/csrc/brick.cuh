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
