"""Build libtct_b200.so in-tree for sm_100a.

    python tectosaur_b200/build.py [-j N] [--force]

(run as a script: importing the package loads the library this builds)

Each CUDA source compiles to its own object in parallel (nvcc
-gencode arch=compute_100a,code=sm_100a -lineinfo -O3), the host C++ source
with g++ (OpenMP, -ffp-contract=off), and nvcc links the shared library next
to this file, where tectosaur_b200._lib loads it.
"""
import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtct_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# The image's CXX may point at a compiler without libgomp; the system g++ has it.
HOST_CXX = shutil.which("g++", path="/usr/bin:/bin") or "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-ccbin", HOST_CXX,
    "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC,
    "-Xptxas", "-warn-spills",
]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
             "-I" + INCLUDE, "-I" + os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["pairs.cu", "pairs_batched.cu", "farfield.cu", "bsr.cu", "probe.cu", "noalloc.cu",
              "fmm.cu", "csr.cu", "far_mrhs.cu", "qd.cu", "interior.cu", "near.cu", "tune.cu", "tree_dev.cu", "pts_mrhs.cu",
              "rt_mrhs.cu", "qd_batch.cu"]
CXX_SOURCES = ["host.cpp"]
HEADERS = ["common.cuh", "pair_math.cuh", "far_common.cuh", "near_plan.h", "octree.h", "tc_common.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, r.returncode, r.stdout + r.stderr


def build(jobs=None, force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "tct_b200.h")]
    cmds = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            cmds.append([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            cmds.append([HOST_CXX] + CXX_FLAGS + ["-c", s, "-o", o])
    failed = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for cmd, rc, out in ex.map(_compile, cmds):
            if verbose or rc != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + out)
            if rc != 0:
                failed.append(cmd[-3])
    if failed:
        raise RuntimeError("tct_b200 build failed: " + ", ".join(failed))
    if force or cmds or _newer(LIB, objs):
        link = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", LIB] + objs + \
               ["-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("tct_b200 link failed:\n" + r.stdout + r.stderr)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, a.v))


if __name__ == "__main__":
    main()
