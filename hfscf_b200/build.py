"""Build the hfgpu engine in-tree: hfscf_b200/libhfgpu.so for sm_100a.

Steps: run the class-code generator (csrc/gen_eri.py) into csrc/generated/,
compile every translation unit with nvcc (one per shell-quartet class, in
parallel), link one shared library.  Objects are rebuilt only when their
source or a header changed (content hash stamps).

Usage: python -m hfscf_b200.build [-j N] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import hashlib
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "generated")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhfgpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE]


def _hash_files(paths):
    h = hashlib.sha1()
    for p in sorted(paths):
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def _common_headers():
    return [os.path.join(CSRC, f) for f in ("hfgpu_common.cuh", "hfgpu_kernels.cuh", "hfgpu_launch.h")] + \
        [os.path.join(GEN, "common.cuh"), os.path.join(INCLUDE, "hfgpu.h")]


def generate():
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_eri.py"), GEN], check=True, stdout=subprocess.DEVNULL)


def _compile(src, verbose):
    base = os.path.splitext(os.path.basename(src))[0]
    obj = os.path.join(OBJ, base + ".o")
    deps = [src] + _common_headers() + [os.path.join(CSRC, "hfgpu_onee.h")]
    if base.startswith("inst_"):
        deps.append(os.path.join(GEN, "class_" + base[5:] + ".cuh"))
    elif base.startswith("hess_") and base != "hess_dispatch":
        deps += [os.path.join(GEN, base + ".cuh"), os.path.join(GEN, "class_" + base[5:] + ".cuh"),
                 os.path.join(CSRC, "hfgpu_hess_kernels.cuh"), os.path.join(CSRC, "hfgpu_hess_launch.h")]
    else:  # hand-written sources: every hand-written header counts
        deps += sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")))
    stamp = obj + ".sha1"
    key = _hash_files(deps) + " ".join(FLAGS + ARCH)
    if os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == key:
        return base, 0.0, ""
    t = time.time()
    cmd = [NVCC] + ARCH + FLAGS + (["-Xcompiler", "-fopenmp"] if src.endswith(".cpp") else []) + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-6000:]}")
    with open(stamp, "w") as f:
        f.write(key)
    return base, time.time() - t, r.stderr if verbose else ""


def build(jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    generate()
    srcs = sorted(glob.glob(os.path.join(GEN, "inst_*.cu"))) + sorted(glob.glob(os.path.join(GEN, "hess_*.cu"))) + \
        [os.path.join(GEN, "dispatch.cu"),
                                                                 os.path.join(CSRC, "hfgpu_host.cu"),
                                                                 os.path.join(CSRC, "hfgpu_noalloc.cu"),
                                                                 os.path.join(CSRC, "hfgpu_onee.cpp")]
    # largest classes first so they do not finish last
    def _size(s):
        b = os.path.basename(s)
        if b.startswith("inst_"):
            return os.path.getsize(os.path.join(GEN, "class_" + b[5:-3] + ".cuh"))
        if b.startswith("hess_") and b != "hess_dispatch.cu":
            return os.path.getsize(os.path.join(GEN, b[:-3] + ".cuh"))
        return 0
    srcs.sort(key=lambda s: -_size(s))
    jobs = jobs or os.cpu_count() or 4
    changed = False
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for base, dt, log in ex.map(lambda s: _compile(s, verbose), srcs):
            if dt > 0:
                changed = True
                print(f"  compiled {base:>12s} in {dt:6.1f}s", flush=True)
            if log:
                print(log)
    objs = [os.path.join(OBJ, os.path.splitext(os.path.basename(s))[0] + ".o") for s in srcs]
    if changed or not os.path.exists(LIB):
        subprocess.run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-Xcompiler", "-fopenmp"], check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    t = time.time()
    print(build(a.j, a.verbose), f"{time.time() - t:.1f}s")
