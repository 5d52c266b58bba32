"""Compact request format of the serving path (phc_request_encode /
phc_request_decode): encode -> decode gives back the same packed table
(term order, exponents, degrees, coefficients bit for bit) and options;
malformed requests are refused with err_invalid_input, never accepted or
read past their end. Runs without a GPU."""
import ctypes

import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import workloads as W


def _table(s):
    t, st = s.table()
    assert st == 0
    n, T = t.n, t.nterms
    first = np.ctypeslib.as_array(t.first, shape=(n + 1,)).copy()
    deg = np.ctypeslib.as_array(t.deg, shape=(n,)).copy()
    hexps = np.ctypeslib.as_array(t.hexps, shape=(T * (n + 1),)).copy()
    coefs = np.ctypeslib.as_array(t.coefs, shape=(2 * T,)).copy()
    return n, first, deg, hexps, coefs


CASES = {
    "cfg2": lambda: W.cfg2(),
    "katsura4": lambda: W.katsura(4),
    "cyclic5": lambda: W.cyclic(5),
    "stream7": lambda: W.stream_system(7),
    "stream31": lambda: W.stream_system(31),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_round_trip(name):
    s = W.build(P.SparseSystem, *CASES[name]())
    o = P.default_options()
    o.seed = 7
    o.tracker.step_max = 0.05
    o.endgame.nsamples = 6
    data = P.encode_request(s, o)
    t, _ = s.table()
    assert len(data) == P._abi.lib().phc_request_size(ctypes.byref(t), 1)
    s2, o2, st = P.decode_request(data)
    assert st == 0
    a, b = _table(s), _table(s2)
    assert a[0] == b[0]
    for x, y in zip(a[1:], b[1:]):
        assert np.array_equal(x, y)
    assert bytes(o2) == bytes(o)
    # without options the decoder returns the defaults
    s3, o3, st = P.decode_request(P.encode_request(s))
    assert st == 0 and bytes(o3) == bytes(P.default_options())
    assert np.array_equal(_table(s3)[3], a[3])


def test_sparse_terms_are_smaller_than_dense_exponents():
    s = W.build(P.SparseSystem, *W.cyclic(6))
    n, first, deg, hexps, coefs = _table(s)
    dense = len(coefs) * 8 + len(hexps) * 4
    assert len(P.encode_request(s)) < dense


def test_malformed_requests_are_refused():
    s = W.build(P.SparseSystem, *W.katsura(3))
    data = P.encode_request(s, P.default_options())
    for cut in range(len(data)):
        _, _, st = P.decode_request(data[:cut])
        assert st == P.ERR_INVALID_INPUT, cut
    _, _, st = P.decode_request(data + b"\x00")
    assert st == P.ERR_INVALID_INPUT
    bad = bytearray(data)
    bad[0:4] = b"XXXX"
    assert P.decode_request(bytes(bad))[2] == P.ERR_INVALID_INPUT
    bad = bytearray(data)
    bad[4] = 2  # version
    assert P.decode_request(bytes(bad))[2] == P.ERR_INVALID_INPUT
    # first term's first pair: variable index out of range
    n = s.nvars()
    off = 24 + ctypes.sizeof(P.SolveOptions) + 4 * n + 16 + 2
    bad = bytearray(data)
    bad[off:off + 2] = (n).to_bytes(2, "little")
    assert P.decode_request(bytes(bad))[2] == P.ERR_INVALID_INPUT
    bad[off:off + 2] = (0).to_bytes(2, "little")
    bad[off + 2:off + 4] = (0).to_bytes(2, "little")  # zero exponent
    assert P.decode_request(bytes(bad))[2] == P.ERR_INVALID_INPUT
