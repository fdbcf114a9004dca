"""Direct GPU test of the device field arithmetic (gl.cuh) that every
transform kernel inlines, through b2m_field_eval_host.

The reference defines the field in include/goldilocks.h:90-189 and checks it
in its self-test (tests/self_test.cu:46-62). Here the device functions are
compared with
  * the reference's own outputs (tests/golden/field.json, made by the
    reference's compiled field functions in oracle/_ref),
  * exact Python integers on edge values (0, 1, p-1, p-2, 2^32-1, 2^32,
    2^64-2^32, 2^63 and neighbours) crossed with each other, every shift
    amount 0..191 on those values, and 10^5 random pairs,
  * a direct O(64) evaluation of the 8-point DFT (root 2^24) and its inverse.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = 0xFFFFFFFF00000001
GOLD = os.path.join(os.path.dirname(__file__), "golden", "field.json")

EDGE = [0, 1, 2, 3, P - 1, P - 2, P - 3, 0xFFFFFFFF, 0x100000000, 0x100000001, 0xFFFFFFFE,
        0xFFFFFFFF00000000, 0xFFFFFFFEFFFFFFFF, 1 << 63, (1 << 63) - 1, (1 << 63) + 1, 1 << 48, (1 << 32) * 3,
        0x8000000080000000, 0x7FFFFFFF7FFFFFFF, 0xDEADBEEFCAFEBABE % P]


def arr(x):
    return np.array(x, dtype=np.uint64)


def ints(x):
    return [int(v) for v in x]


def test_field_ops_against_reference_rows(b2m_gpu):
    rows = json.load(open(GOLD))["rows"]
    a = arr([r["a"] for r in rows])
    b = arr([r["b"] for r in rows])
    assert ints(b2m_gpu.field_eval("add", a, b)) == [r["add"] for r in rows]
    assert ints(b2m_gpu.field_eval("sub", a, b)) == [r["sub"] for r in rows]
    assert ints(b2m_gpu.field_eval("mul", a, b)) == [r["mul"] for r in rows]
    e = arr([r["b"] % 1000003 for r in rows])
    assert ints(b2m_gpu.field_eval("pow", a, e)) == [r["pow"] for r in rows]
    nz = [i for i, r in enumerate(rows) if r["a"]]
    inv = b2m_gpu.field_eval("inv", a[nz])
    assert ints(inv) == [rows[i]["inv"] for i in nz]


def test_field_ops_edge_values_crossed(b2m_gpu):
    xs = [x for x in EDGE for _ in EDGE]
    ys = [y for _ in EDGE for y in EDGE]
    a, b = arr(xs), arr(ys)
    assert ints(b2m_gpu.field_eval("add", a, b)) == [(x + y) % P for x, y in zip(xs, ys)]
    assert ints(b2m_gpu.field_eval("sub", a, b)) == [(x - y) % P for x, y in zip(xs, ys)]
    assert ints(b2m_gpu.field_eval("mul", a, b)) == [(x * y) % P for x, y in zip(xs, ys)]


def test_every_shift_amount(b2m_gpu):
    """x * 2^s for s = 0..191 on the edge values and on random elements."""
    rng = np.random.default_rng(192)
    vals = EDGE + [int(v) % P for v in rng.integers(0, 2**63, 40, dtype=np.uint64)]
    xs = [x for x in vals for _ in range(192)]
    ss = [s for _ in vals for s in range(192)]
    want = [(x << s) % P for x, s in zip(xs, ss)]
    assert ints(b2m_gpu.field_eval("shl", arr(xs), arr(ss))) == want
    # the run-time (warp-uniform) shift of the level-1 twiddles
    assert ints(b2m_gpu.field_eval("shl_rt", arr(xs), arr(ss))) == want
    # the carry's scale by N^-1 = 2^(192 - k): x * 2^(160 + t), t < 32
    ts = [s % 32 for s in ss]
    assert ints(b2m_gpu.field_eval("shl_160", arr(xs), arr(ts))) == [(x << (160 + t)) % P for x, t in zip(xs, ts)]


def test_paired_run_time_shift(b2m_gpu):
    """The paired run-time shift of the inverse tile tasks: elements 2k and
    2k+1 shifted together by b[2k], every amount 0..191, crossed edge values."""
    rng = np.random.default_rng(193)
    vals = EDGE + [int(v) % P for v in rng.integers(0, 2**63, 24, dtype=np.uint64)]
    xs, ss = [], []
    for i, x in enumerate(vals):
        y = vals[(7 * i + 3) % len(vals)]
        for s in range(192):
            xs += [x, y]
            ss += [s, 191 - s]  # the second amount is ignored: both take b[2k]
    want = [(x << ss[i & ~1]) % P for i, x in enumerate(xs)]
    assert ints(b2m_gpu.field_eval("shl_rt2", arr(xs), arr(ss))) == want
    # odd length: the last element is shifted alone
    got = ints(b2m_gpu.field_eval("shl_rt2", arr(xs[:5]), arr(ss[:5])))
    assert got == want[:5]


def test_random_pairs(b2m_gpu):
    rng = np.random.default_rng(100000)
    n = 100000
    a = rng.integers(0, 2**63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    b = rng.integers(0, 2**63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    a = arr([int(x) % P for x in a])
    b = arr([int(x) % P for x in b])
    xs, ys = ints(a), ints(b)
    assert ints(b2m_gpu.field_eval("add", a, b)) == [(x + y) % P for x, y in zip(xs, ys)]
    assert ints(b2m_gpu.field_eval("sub", a, b)) == [(x - y) % P for x, y in zip(xs, ys)]
    assert ints(b2m_gpu.field_eval("mul", a, b)) == [(x * y) % P for x, y in zip(xs, ys)]
    s = arr(rng.integers(0, 192, n))
    assert ints(b2m_gpu.field_eval("shl", a, s)) == [(x << int(k)) % P for x, k in zip(xs, ints(s))]


def _brev3(i):
    return ((i & 1) << 2) | (i & 2) | (i >> 2)


def test_dft8_and_inverse(b2m_gpu):
    rng = np.random.default_rng(8)
    groups = [EDGE[:8], EDGE[8:16], [P - 1] * 8, [0] * 7 + [1]]
    groups += [[int(v) % P for v in rng.integers(0, 2**63, 8, dtype=np.uint64)] for _ in range(200)]
    flat = [v for g in groups for v in g]
    fwd = ints(b2m_gpu.field_eval("dft8", arr(flat)))
    w = pow(2, 24, P)
    want = []
    for g in groups:
        y = [sum(g[n] * pow(w, n * k, P) for n in range(8)) % P for k in range(8)]
        want += [y[_brev3(i)] for i in range(8)]  # bit-reversed order out
    assert fwd == want
    back = ints(b2m_gpu.field_eval("idft8", arr(fwd)))
    assert back == [(8 * v) % P for v in flat]  # unscaled inverse
