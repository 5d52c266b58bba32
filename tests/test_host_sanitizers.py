"""The library's host C++ under AddressSanitizer and
UndefinedBehaviorSanitizer, on CPU (compute-sanitizer, the device-side
counterpart, is not available on the GPU pool; device-side indices come
from the compiled table, which verify_plan checks before every launch).

tests/sanitize/host_fuzz.cpp is compiled with -fsanitize=address,undefined
together with every host source of the library (the CUDA objects are linked
uninstrumented and never called) and run on random systems. It covers the
table compiler and its verifier, corrupted tables, the request codec with
damaged requests, the bookkeeping at the dedup tolerance boundaries, and the
user-system sampler; once more under ThreadSanitizer for the sampler's
threaded least squares. tests/sanitize/oracle_fuzz.cpp runs the CPU
restatement the same way, and once more under ThreadSanitizer, since its
solve uses worker threads. Any memory error, undefined behaviour, data race
or broken invariant fails the run."""
import glob
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _sanitizer_cxx():
    """A C++ compiler whose AddressSanitizer runtime is installed (the
    compiler named by CXX may be a wrapper without it)."""
    for c in (os.environ.get("CXX"), "g++", "/usr/bin/g++", "clang++"):
        if not c or shutil.which(c) is None:
            continue
        r = subprocess.run([c, "-print-file-name=libasan.so"], capture_output=True, text=True)
        path = r.stdout.strip()
        if r.returncode == 0 and os.path.isabs(path) and os.path.exists(path):
            return c
    return None


def _build_fuzz(tmp_path_factory, sanitize):
    from polyhomocont_b200 import build as B
    B.build()
    cxx = _sanitizer_cxx()
    if cxx is None:
        pytest.fail("no C++ compiler with the AddressSanitizer runtime found")
    out = str(tmp_path_factory.mktemp("san") / "host_fuzz")
    csrc = os.path.join(ROOT, "polyhomocont_b200", "csrc")
    cmd = ([cxx, "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-pthread",
            f"-fsanitize={sanitize}", "-ffp-contract=off",
            "-I", os.path.join(ROOT, "include"), "-I", csrc, "-I", os.path.join(CUDA, "include"),
            os.path.join(ROOT, "tests", "sanitize", "host_fuzz.cpp")]
           + sorted(glob.glob(os.path.join(csrc, "*.cpp")))
           + sorted(glob.glob(os.path.join(B.BUILD, "*.cu.o")))
           + ["-L", os.path.join(CUDA, "lib64"), "-lcudart", "-lpthread", "-ldl", "-lrt",
              "-o", out])
    if sanitize != "thread":
        cmd.insert(6, "-fno-sanitize-recover=all")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    return out


@pytest.fixture(scope="module")
def fuzz_binary(tmp_path_factory):
    return _build_fuzz(tmp_path_factory, "address,undefined")


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_host_code_under_sanitizers(fuzz_binary, seed):
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = os.path.join(CUDA, "lib64") + ":" + env.get("LD_LIBRARY_PATH", "")
    env["ASAN_OPTIONS"] = "protect_shadow_gap=0:abort_on_error=0:halt_on_error=1"
    env["UBSAN_OPTIONS"] = "print_stacktrace=1:halt_on_error=1"
    r = subprocess.run([fuzz_binary, "600", str(seed)], capture_output=True, text=True,
                       timeout=900, env=env)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-6000:])
    assert "iterations ok" in r.stdout
    assert "runtime error" not in r.stderr  # UBSan reports


def test_host_code_under_thread_sanitizer(tmp_path_factory):
    """The same driver under ThreadSanitizer: the sampler's least squares
    runs its column updates on several threads for designs of 192
    monomials or more (one such design every 150 iterations)."""
    exe = _build_fuzz(tmp_path_factory, "thread")
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = os.path.join(CUDA, "lib64") + ":" + env.get("LD_LIBRARY_PATH", "")
    env["TSAN_OPTIONS"] = "halt_on_error=1"
    r = subprocess.run([exe, "300", "4"], capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-6000:])
    assert "iterations ok" in r.stdout
    assert "WARNING: ThreadSanitizer" not in r.stderr


def _build_oracle_driver(tmp_path_factory, cxx, sanitize, name):
    out = str(tmp_path_factory.mktemp("san") / name)
    cmd = [cxx, "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-pthread",
           f"-fsanitize={sanitize}", "-ffp-contract=off", "-I", os.path.join(ROOT, "oracle"),
           os.path.join(ROOT, "tests", "sanitize", "oracle_fuzz.cpp"),
           os.path.join(ROOT, "oracle", "phc_oracle.cpp"), "-o", out]
    if sanitize != "thread":
        cmd.insert(-2, "-fno-sanitize-recover=all")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    return out


@pytest.mark.parametrize("sanitize", ["address,undefined", "thread"])
def test_restatement_under_sanitizers(tmp_path_factory, sanitize):
    """The CPU restatement (two worker threads per solve) on random small
    systems: no memory error, no undefined behaviour, no data race."""
    cxx = _sanitizer_cxx()
    if cxx is None:
        pytest.fail("no C++ compiler with the sanitizer runtimes found")
    exe = _build_oracle_driver(tmp_path_factory, cxx, sanitize, "oracle_fuzz")
    env = dict(os.environ)
    env["ASAN_OPTIONS"] = "halt_on_error=1"
    env["UBSAN_OPTIONS"] = "print_stacktrace=1:halt_on_error=1"
    env["TSAN_OPTIONS"] = "halt_on_error=1"
    r = subprocess.run([exe, "40", "5"], capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-6000:])
    assert "iterations ok" in r.stdout
    assert "WARNING: ThreadSanitizer" not in r.stderr and "runtime error" not in r.stderr
