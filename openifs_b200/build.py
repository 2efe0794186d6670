"""Build libcloudsc_b200.so (sm_100a) in-tree with nvcc.

    python -m openifs_b200.build            # build if sources changed
    python -m openifs_b200.build --force    # rebuild

The kernels are compiled with --fmad=false: the FP64 kernel must perform the
reference's operations with one rounding each (no multiply-add contraction).
"""
import argparse
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcloudsc_b200.so")
STAMP = os.path.join(HERE, ".libcloudsc_b200.stamp")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false (device) and -ffp-contract=off (host): no multiply-add
# contraction anywhere, so the kernels, the host-side constant set-up and
# plibm.h evaluate exactly the operations written.
NVCC_FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O2", "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]


def _nvcc():
    cand = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    deps = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".cu")))
    return [os.path.join(CSRC, f) for f in srcs], [os.path.join(CSRC, f) for f in deps]


def _digest(paths):
    h = hashlib.sha256()
    inc = os.path.join(ROOT, "include")
    for p in paths + sorted(os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")):
        with open(p, "rb") as f:
            h.update(p.encode())
            h.update(f.read())
    h.update(" ".join(ARCH + NVCC_FLAGS).encode())
    return h.hexdigest()


def build(force=False, verbose=False):
    srcs, deps = _sources()
    dig = _digest(deps)
    if not force and os.path.exists(LIB) and os.path.exists(STAMP):
        if open(STAMP).read().strip() == dig:
            return LIB
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s)[:-3] + ".o")
        cmds.append([nvcc] + ARCH + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-c", s, "-o", o])
        objs.append(o)
    # the translation units compile independently: one nvcc per source, in parallel
    from concurrent.futures import ThreadPoolExecutor

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(run, cmds))
    tmp = LIB + ".tmp"
    # static CUDA runtime: the library does not depend on whichever libcudart
    # another component of the process (e.g. torch) brings along
    cmd = [nvcc] + ARCH + ["-shared", "--cudart", "static", "-o", tmp] + objs
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    with open(STAMP, "w") as f:
        f.write(dig)
    return LIB


def build_oracle(verbose=False):
    """Build the CPU checker (oracle/liboracle_cloudsc.so) with its Makefile."""
    od = os.path.join(ROOT, "oracle")
    r = subprocess.run(["make", "-s", "-C", od], capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + (r.stdout or "") + (r.stderr or ""))
    return os.path.join(od, "liboracle_cloudsc.so")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
