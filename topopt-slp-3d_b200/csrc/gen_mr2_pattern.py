"""Generate mr2_pattern.h: which Walsh-Hadamard modes of the 8 sub-element
blocks are non-zero for each upper-triangle entry (MR factor 2, hex8).

For MR factor 2 the element matrix is K_e = sum_s w_s KE_s over the 8
sub-cubes s = (sz, sx, sy).  With the 8-point Walsh-Hadamard matrix H
(H H = 8 I) this equals sum_b (H w)_b Khat_b with Khat = H KE / 8.  The modes
that are odd in one or more directions cancel in many entries; the zero
pattern is structural (the same for every box element and Poisson ratio), so
the kernel skips those terms at compile time: 1548 instead of 2400 FMAs to
form the 300 entries.

    python topopt-slp-3d_b200/csrc/gen_mr2_pattern.py > topopt-slp-3d_b200/csrc/mr2_pattern.h

The blocks are computed here directly from the 2-point Gauss rule per
sub-cube (the integrand of ElemStiffMatrixGQMR) for a few generic box shapes;
an entry/mode pair is kept if it is non-zero for any of them.  The entry
order is the kernel's (diagonal-major, even rows first; see pair_i/pair_j in
tosp_internal.h).
"""
import numpy as np

SX = np.array([-1, -1, 1, 1, -1, -1, 1, 1])
SY = np.array([-1, 1, -1, 1, -1, 1, -1, 1])
SZ = np.array([-1, -1, -1, -1, 1, 1, 1, 1])


def blocks(a, b, c, nu, n=2):
    d0 = 1.0 / ((1 + nu) * (1 - 2 * nu))
    D = np.zeros((6, 6))
    D[:3, :3] = nu
    np.fill_diagonal(D[:3, :3], 1 - nu)
    D[3, 3] = D[4, 4] = D[5, 5] = (1 - 2 * nu) / 2
    D *= d0
    g = 1 / np.sqrt(3)
    out = []
    for sz in range(n):
        for sx in range(n):
            for sy in range(n):
                k = np.zeros((24, 24))
                cx, cy, cz = (-1 + (2 * sx + 1) / n, -1 + (2 * sy + 1) / n, -1 + (2 * sz + 1) / n)
                for p3 in (-g, g):
                    for p1 in (-g, g):
                        for p2 in (-g, g):
                            x1, x2, x3 = cx + p1 / n, cy + p2 / n, cz + p3 / n
                            dx = SX * (1 + SY * x2) * (1 + SZ * x3) / (8 * a)
                            dy = SY * (1 + SX * x1) * (1 + SZ * x3) / (8 * b)
                            dz = SZ * (1 + SX * x1) * (1 + SY * x2) / (8 * c)
                            B = np.zeros((6, 24))
                            B[0, 0::3], B[1, 1::3], B[2, 2::3] = dx, dy, dz
                            B[3, 0::3], B[3, 1::3] = dy, dx
                            B[4, 1::3], B[4, 2::3] = dz, dy
                            B[5, 0::3], B[5, 2::3] = dz, dx
                            k += B.T @ D @ B
                out.append(k)
    return out


def pair_order():
    pairs = []
    for d in range(24):
        rows = list(range(0, 24 - d, 2)) + list(range(1, 24 - d, 2))
        pairs += [(i, i + d) for i in rows]
    return pairs


def main():
    H1 = np.array([[1, 1], [1, -1]])
    H = np.kron(np.kron(H1, H1), H1)
    pairs = pair_order()
    mask = np.zeros(300, dtype=int)
    for shape in ((0.7, 1.3, 2.1, 0.27), (2.0, 0.5, 1.0, 0.41), (1.0, 1.0, 1.0, 0.3)):
        ks = blocks(*shape)
        P = np.array([[k[i, j] for (i, j) in pairs] for k in ks])
        Ph = H @ P / 8
        nz = np.abs(Ph) > 1e-12 * np.abs(Ph).max()
        for t in range(300):
            for m in range(8):
                if nz[m, t]:
                    mask[t] |= 1 << m
    print("// Generated by gen_mr2_pattern.py - do not edit.")
    print("// Bit m of mr2_mask(t): Walsh-Hadamard mode m of entry t (kernel order) is non-zero.")
    print("#pragma once")
    print(f"constexpr int kMr2Nonzeros = {int(sum(bin(v).count('1') for v in mask))};")
    print("__host__ __device__ constexpr unsigned mr2_mask(int t) {")
    print("    constexpr unsigned char m[300] = {")
    for r in range(0, 300, 20):
        print("        " + ", ".join(str(v) for v in mask[r:r + 20]) + ",")
    print("    };")
    print("    return m[t];")
    print("}")


if __name__ == "__main__":
    main()
