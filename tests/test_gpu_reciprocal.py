"""The tracker's own reciprocals against CUDA's (phc_device.cuh):

  rcp_nr(d)  the hardware reciprocal approximation (rcp.approx) refined by
             Newton-Raphson steps r <- r + r (1 - d r) (two in FP64, one in
             FP32); every pivot of the Gauss-Jordan elimination goes
             through it;
  crcp(a)    1/a = conj(a) / |a|^2 with rcp_nr, and Smith's division
             (R. L. Smith, CACM 5 (1962) 435) where |a|^2 would leave
             [1e-290, 1e290] ([1e-36, 1e36] in FP32).

rcp_nr must be within 1 ulp of CUDA's correctly rounded 1/d over its
range, both signs. crcp must agree with the exact reciprocal (computed on
the host in extended precision) to 4 units of the precision, relative to
|1/a|, and with CUDA's complex division cuCdiv(1, a) to 8, on random
values, at the ends of the range and across the Smith fallback boundary."""
import ctypes

import numpy as np
import pytest

from tests.probe import build_probe

pytestmark = pytest.mark.gpu

EPS64 = np.finfo(np.float64).eps
EPS32 = np.finfo(np.float32).eps


@pytest.fixture(scope="module")
def probe():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    L = ctypes.CDLL(build_probe.build())
    for name, t in (("phc_probe_rcp64", ctypes.c_double), ("phc_probe_crcp64", ctypes.c_double),
                    ("phc_probe_rcp32", ctypes.c_float), ("phc_probe_crcp32", ctypes.c_float)):
        f = getattr(L, name)
        p = ctypes.POINTER(t)
        f.argtypes = [p, ctypes.c_int32, p, p]
        f.restype = ctypes.c_int
    return L


def _call(fn, x, values, dtype):
    """fn on x (values entries); returns its two output arrays, x.size each."""
    x = np.ascontiguousarray(x, dtype=dtype)
    a = np.zeros(x.size, dtype=dtype)
    b = np.zeros(x.size, dtype=dtype)
    p = ctypes.POINTER(ctypes.c_double if dtype == np.float64 else ctypes.c_float)
    st = fn(x.ctypes.data_as(p), values, a.ctypes.data_as(p), b.ctypes.data_as(p))
    assert st == 0, f"CUDA error {st}"
    return a, b


def _ulps(a, b):
    """Distance in units in the last place between same-signed finite floats."""
    it = np.int64 if a.dtype == np.float64 else np.int32
    assert np.all(np.sign(a) == np.sign(b))
    return np.abs(a.view(it).astype(np.int64) - b.view(it).astype(np.int64))


def _log_uniform(rng, lo, hi, size, dtype):
    v = 10.0 ** rng.uniform(lo, hi, size)
    v *= rng.choice([-1.0, 1.0], size)
    return v.astype(dtype)


def test_rcp_nr_fp64_within_one_ulp(probe):
    rng = np.random.default_rng(11)
    d = _log_uniform(rng, -290, 290, 200000, np.float64)
    edges = np.array([1e-290, 1e290, 1.0, 2.0, 0.5, 3.0, 1.0 + EPS64, 2.0 - 2 * EPS64,
                      np.nextafter(1.0, 0.0), 7.0, 1e-100, 1e100], dtype=np.float64)
    d = np.concatenate([d, edges, -edges])
    nr, div = _call(probe.phc_probe_rcp64, d, d.size, np.float64)
    assert np.all(np.isfinite(nr))
    assert _ulps(nr, div).max() <= 1


def test_rcp_nr_fp32_within_one_ulp(probe):
    rng = np.random.default_rng(12)
    d = _log_uniform(rng, -36, 36, 200000, np.float32)
    edges = np.array([1e-36, 1e36, 1.0, 2.0, 0.5, 3.0, 7.0], dtype=np.float32)
    d = np.concatenate([d, edges, -edges])
    nr, div = _call(probe.phc_probe_rcp32, d, d.size, np.float32)
    assert np.all(np.isfinite(nr))
    assert _ulps(nr, div).max() <= 1


def _exact_reciprocal(a):
    """1/a in extended precision (x87 long double: 64-bit significand), a
    interleaved complex."""
    re = a[0::2].astype(np.longdouble)
    im = a[1::2].astype(np.longdouble)
    # scale by a power of two so that |a|^2 neither overflows nor underflows
    e = np.floor(np.log2(np.maximum(np.abs(re), np.abs(im)))).astype(np.longdouble)
    s = np.exp2(-e)
    rs, is_ = re * s, im * s
    den = rs * rs + is_ * is_
    return (rs / den) * s, (-is_ / den) * s


def _complex_cases(rng, lo, hi, size, dtype):
    mag = 10.0 ** rng.uniform(lo, hi, size)
    ang = rng.uniform(0.0, 2 * np.pi, size)
    a = np.empty(2 * size)
    a[0::2] = mag * np.cos(ang)
    a[1::2] = mag * np.sin(ang)
    return a.astype(dtype)


def _edge_cases(mags, dtype):
    out = []
    for m in mags:
        for ang in (0.0, 0.3, np.pi / 4, np.pi / 2, 2.0, np.pi, 4.0, 5.5):
            out += [m * np.cos(ang), m * np.sin(ang)]
    return np.array(out, dtype=dtype)


def _rel_err(got, ref_re, ref_im):
    g_re = got[0::2].astype(np.longdouble)
    g_im = got[1::2].astype(np.longdouble)
    scale = np.maximum(np.abs(ref_re), np.abs(ref_im))
    return np.maximum(np.abs(g_re - ref_re), np.abs(g_im - ref_im)) / scale


def test_crcp_fp64(probe):
    rng = np.random.default_rng(13)
    # |a|^2 across the fallback boundaries 1e-290 and 1e290 (Smith's
    # division outside), and far outside them (|a|^2 under- or overflows)
    a = np.concatenate([_complex_cases(rng, -140, 140, 100000, np.float64),
                        _edge_cases((1e-145, 0.99e-145, 1.01e-145, 1e145, 0.99e145, 1.01e145,
                                     1e-200, 1e200, 1e-300, 1e300), np.float64)])
    out, div = _call(probe.phc_probe_crcp64, a, a.size // 2, np.float64)
    ref_re, ref_im = _exact_reciprocal(a)
    assert np.all(np.isfinite(out))
    # conj(a) * rcp_nr(|a|^2): |a|^2 (1 ulp), the reciprocal (1 ulp), the
    # products (1/2 ulp): a few eps; Smith's division is within that too
    assert _rel_err(out, ref_re, ref_im).max() <= 4 * EPS64
    assert _rel_err(out, div[0::2].astype(np.longdouble),
                    div[1::2].astype(np.longdouble)).max() <= 8 * EPS64


def test_crcp_fp32(probe):
    rng = np.random.default_rng(14)
    a = np.concatenate([_complex_cases(rng, -17, 17, 100000, np.float32),
                        _edge_cases((1e-18, 0.99e-18, 1.01e-18, 1e18, 0.99e18, 1.01e18,
                                     1e-25, 1e25), np.float32)])
    out, div = _call(probe.phc_probe_crcp32, a, a.size // 2, np.float32)
    ref_re, ref_im = _exact_reciprocal(a.astype(np.float64))
    assert np.all(np.isfinite(out))
    assert _rel_err(out, ref_re, ref_im).max() <= 4 * EPS32
    assert _rel_err(out, div[0::2].astype(np.longdouble),
                    div[1::2].astype(np.longdouble)).max() <= 8 * EPS32
