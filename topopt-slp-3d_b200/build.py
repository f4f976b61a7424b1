"""Build recipe for the tosp CUDA library (sm_100a) and the C oracle.

    python topopt-slp-3d_b200/build.py            # library only
    python topopt-slp-3d_b200/build.py --oracle   # plus the C oracle libraries in oracle/

The library is compiled in-tree to ``topopt-slp-3d_b200/tosp/libtosp.so`` with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo``.  Objects are
rebuilt only when a source or header is newer than the object.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "tosp", "libtosp.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
         "-I" + CSRC, "--expt-relaxed-constexpr"]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "tosp.h"))
    return hs


def _compile(src, extra):
    out = os.path.join(OBJ, src + ".o")
    srcp = os.path.join(CSRC, src)
    newest = max([os.path.getmtime(srcp)] + [os.path.getmtime(h) for h in _headers()])
    if os.path.exists(out) and os.path.getmtime(out) >= newest and not extra:
        return out
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", srcp, "-o", out]
    if src.endswith(".cpp"):
        cmd = [NVCC] + FLAGS + extra + ["-x", "cu", "-c", srcp, "-o", out] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return out


def build_library(verbose_ptxas=False):
    os.makedirs(OBJ, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), _sources()))
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s" % r.stderr)
    return LIB


def build_oracle():
    """The C restatements under oracle/ (test infrastructure, CPU baseline)."""
    outs = []
    for name in ("kelem_omp", "assembled_omp"):
        src = os.path.join(ROOT, "oracle", name + ".c")
        out = os.path.join(ROOT, "oracle", "lib%s.so" % name)
        if not os.path.exists(src):
            continue
        outs.append(out)
        if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
            continue
        cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", src, "-o", out, "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("gcc failed for the oracle:\n%s" % r.stderr)
    return outs


if __name__ == "__main__":
    print(build_library(verbose_ptxas="-v" in sys.argv))
    if "--oracle" in sys.argv:
        print(build_oracle())
