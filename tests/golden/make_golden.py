"""Generate the golden fixtures under tests/golden/ from the reference sources.

Run in a container that has the reference checkout (read-only) at
``/root/reference`` (or pass its path as the first argument):

    python tests/golden/make_golden.py [/path/to/TopOpt-SLP-3D]

Outputs (committed; tests read only these files, never the reference):
  * ``ke_closed_form.npz`` - the 24x24 hex8 stiffness of
    ``Implementation/ElemStiffMatrix.m`` for several element shapes and
    Poisson ratios.  The MATLAB file is a straight list of scalar assignments
    (``k(i,j) = expr;``) followed by a symmetric fill and a row/column
    permutation; this script evaluates those statements one by one in Python
    (``^`` -> ``**``, 1-based ``k(i,j)`` -> ``k[i-1, j-1]``).  No reference
    code is copied into the repository, only the resulting numbers.
  * ``fixtures.npz`` - for a few small saved problems of
    ``Implementation/Tests/*.mat``: the support/load/region rows and the
    ``freedofs`` / ``f`` / ``fixedDens`` arrays the reference's EnterData
    stored beside them.
"""
import os
import re
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))

SHAPES = [(1.0, 1.0, 1.0, 0.3), (0.5, 0.5, 0.5, 0.3), (1.0, 0.5, 2.0, 0.3),
          (2.0, 1.0, 0.75, 0.25), (1.0, 1.0, 1.0, 0.45)]

FIXTURES = ["cb48x16x16", "mbb96x16x1half", "hc32x16x32quarter", "tt16x80x16quarter",
            "bd96x24x12quarter", "bt16x64x16", "ls48x48x16half", "mbb96x16x16quarter"]


def eval_closed_form(src, el, eh, ew, nu):
    ns = {"str_el": el, "str_eh": eh, "str_ew": ew, "str_nu": nu, "pi": np.pi}
    k = np.zeros((24, 24))
    ns["k"] = k
    body = src.split("\n")
    perm2 = None
    for raw in body:
        line = raw.split("%")[0].strip()
        if not line or line.startswith("function") or line == "end":
            continue
        m = re.match(r"^perm2\s*=\s*\[(.*)\];$", line)
        if m:
            perm2 = np.array([int(v) for v in m.group(1).split(",")]) - 1
            continue
        if line.startswith("k(perm2,perm2)"):
            kn = np.zeros_like(k)
            kn[np.ix_(perm2, perm2)] = k
            k[:] = kn
            continue
        if line.startswith("for") or line.startswith("k(i,j) = k(j,i)"):
            continue
        if line.startswith("k = zeros"):
            continue
        expr = line.rstrip(";")
        expr = expr.replace("str.el", "str_el").replace("str.eh", "str_eh")
        expr = expr.replace("str.ew", "str_ew").replace("str.nu", "str_nu")
        expr = re.sub(r"k\((\d+),(\d+)\)", lambda mm: f"k[{int(mm.group(1)) - 1},{int(mm.group(2)) - 1}]", expr)
        expr = expr.replace("^", "**")
        exec(expr, ns)
        if line.startswith("k(24,24)"):
            # symmetric fill of the reference (lower triangle from the upper)
            iu = np.triu_indices(24, 1)
            k[(iu[1], iu[0])] = k[iu]
    return k


def main():
    src = open(os.path.join(REF, "Implementation", "ElemStiffMatrix.m")).read()
    kes = np.stack([eval_closed_form(src, *s) for s in SHAPES])
    np.savez_compressed(os.path.join(HERE, "ke_closed_form.npz"), shapes=np.array(SHAPES), ke=kes)

    import scipy.io as sio
    out = {}
    for name in FIXTURES:
        s = sio.loadmat(os.path.join(REF, "Implementation", "Tests", name + ".mat"),
                        squeeze_me=True, struct_as_record=False)["str"]
        nnodes = int(s.nnodes)
        fd = np.asarray(s.freedofs, dtype=np.int64).ravel() - 1
        mask = np.zeros(3 * nnodes, dtype=bool)
        mask[fd] = True
        f = np.asarray(s.f, dtype=np.float64).ravel()
        nzf = np.nonzero(f)[0]
        out[name + "/dims"] = np.array([s.nelx, s.nely, s.nelz], dtype=np.int64)
        out[name + "/sizes"] = np.array([s.el, s.eh, s.ew, s.E, s.nu], dtype=np.float64)
        out[name + "/supp"] = np.atleast_2d(np.asarray(s.supp, dtype=np.float64))
        out[name + "/loads"] = np.atleast_2d(np.asarray(s.loads, dtype=np.float64))
        out[name + "/freemask"] = np.packbits(mask)
        out[name + "/f_idx"] = nzf.astype(np.int64)
        out[name + "/f_val"] = f[nzf]
        out[name + "/nfree"] = np.array([fd.size], dtype=np.int64)
        if "fix" in s._fieldnames:
            out[name + "/fix"] = np.atleast_2d(np.asarray(s.fix, dtype=np.int64))
            out[name + "/fixedDens"] = np.asarray(s.fixedDens, dtype=np.int64).ravel() - 1
            out[name + "/fixedDensVal"] = np.asarray(s.fixedDensVal, dtype=np.float64).ravel()
    np.savez_compressed(os.path.join(HERE, "fixtures.npz"), **out)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
