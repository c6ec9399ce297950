"""Build libwamgpu.so (sm_100a) in-tree with nvcc.

    python -m wam_b200.build          # incremental
    python -m wam_b200.build --force  # rebuild everything

The propagation unit is compiled without FMA contraction so that the
recomputed propagation coefficients round exactly like the reference's stored
coefficient arrays; the source-term unit keeps FMA (compute-bound kernel).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwamgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]
UNITS = {
    "implsch.cu": [],
    "propags.cu": ["-fmad=false"],
    "api.cu": [],
    "adjoint.cu": [],
    "output.cu": ["-fmad=false"],
}
HEADERS = ["implsch.cuh", "propags.cuh", "propargs.hpp", "devmath.cuh", "kernels.hpp", "adjoint.cuh", "adjoint_warp.cuh", "spectral_tables.hpp", "wamgpu_config.hpp"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _newest_dep():
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "wamgpu.h")]
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    dep = _newest_dep()
    jobs = []
    for src, extra in UNITS.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), dep):
            cmd = [nvcc] + ARCH + COMMON + extra + ["-c", s, "-o", o]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return cmd

    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        list(ex.map(run, jobs))
    objs = [os.path.join(BUILD, s.replace(".cu", ".o")) for s in UNITS]
    if jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
