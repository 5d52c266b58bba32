"""Builds libphc_b200.so in-tree: the sm_100a CUDA kernels and the C ABI.

    python -m polyhomocont_b200.build [--force] [-j JOBS]

Every .cu unit is compiled by nvcc for sm_100a (-gencode
arch=compute_100a,code=sm_100a) in parallel, the host C++ with g++
(no floating-point contraction), and everything is linked into
polyhomocont_b200/libphc_b200.so next to this file.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libphc_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = GENCODE + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                        "-I", INCLUDE, "-I", CSRC]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", INCLUDE, "-I", CSRC,
             "-I", os.path.join(CUDA_HOME, "include")]


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                     + glob.glob(os.path.join(INCLUDE, "*.h")))
    return cu, cpp, headers


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def _obj(src):
    return os.path.join(BUILD, os.path.basename(src) + ".o")


def _compile(src, hdr_time, force, extra):
    obj = _obj(src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(
            os.path.getmtime(src), hdr_time):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    else:
        cmd = [os.environ.get("CXX", "g++")] + CXX_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, (r.stdout + r.stderr)


def build(force=False, jobs=None, verbose=False, ptxas_verbose=False):
    """Compiles what changed and links the library. Returns its path."""
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp, headers = _sources()
    hdr_time = _newest(headers)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    jobs = jobs or min(8, os.cpu_count() or 4)
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, s, hdr_time, force, extra) for s in cu + cpp]
        objs = []
        for f in futs:
            o, log = f.result()
            objs.append(o)
            if log:
                logs.append(log)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC] + GENCODE + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        shutil.move(LIB + ".tmp", LIB)
    if verbose:
        for log in logs:
            sys.stdout.write(log)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    path = build(force=a.force, jobs=a.jobs, verbose=True, ptxas_verbose=a.ptxas_verbose)
    print(path)


if __name__ == "__main__":
    main()
