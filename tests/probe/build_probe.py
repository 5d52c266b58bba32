"""Builds tests/probe/libphc_probe.so, the device probe of the tracker's
reciprocal helpers (test infrastructure), for sm_100a."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SRC = os.path.join(HERE, "phc_probe.cu")
LIB = os.path.join(HERE, "libphc_probe.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(force=False):
    headers = [os.path.join(ROOT, "polyhomocont_b200", "csrc", "phc_device.cuh"),
               os.path.join(ROOT, "polyhomocont_b200", "csrc", "phc_internal.h")]
    newest = max(os.path.getmtime(p) for p in [SRC] + headers)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    cmd = [os.path.join(CUDA_HOME, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a",
           "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "polyhomocont_b200", "csrc"), SRC, "-o", LIB + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"probe build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
