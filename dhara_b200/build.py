"""Builds the CUDA library dhara_b200/libdhara_b200.so for sm_100a (in-tree)."""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libdhara_b200.so")
SRC = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
HDRS = sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))
              + glob.glob(os.path.join(HERE, "..", "include", "*.h")))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-O3",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in SRC + HDRS)


def build(force=False, verbose=False, extra=(), out=None):
    """Compiles every csrc/*.cu for sm_100a and links the library (to `out`,
    default dhara_b200/libdhara_b200.so); `extra` adds nvcc flags."""
    if out is None and not force and not stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    bdir = os.path.join(HERE, "_build")
    if out is not None:
        bdir = os.path.join(bdir, os.path.splitext(os.path.basename(out))[0])
    os.makedirs(bdir, exist_ok=True)
    cmds = []
    objs = []
    for src in SRC:
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        cmds.append([nvcc(), *NVCC_FLAGS, *extra, "-c", src, "-o", obj])
        objs.append(obj)
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), file=sys.stderr)
    # the translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for r in pool.map(lambda c: subprocess.run(c, capture_output=not verbose, text=True), cmds):
            if r.returncode != 0:
                sys.stderr.write((r.stdout or "") + (r.stderr or ""))
                raise subprocess.CalledProcessError(r.returncode, r.args)
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", out or LIB, *objs]
    subprocess.run(cmd, check=True)
    return out or LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
