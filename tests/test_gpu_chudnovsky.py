"""GPU tests of the device binary-splitting tree (b2m_chudnovsky_bs) and of
compute_pi on top of it, bit-exact against the reference: (P, Q, T) of small
ranges against the oracle restatement, roots of the 1k/100k/1M/10M-digit
trees against the reference's own runs (tests/golden/chudnovsky.json), and
digit strings against the reference's compute_pi_chudnovsky
(tests/golden/pi_digits.json)."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from golden_util import sha_limbs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("a,b", [(0, 1), (1, 2), (0, 2), (0, 3), (2, 7), (5, 90), (0, 300), (123, 1500)])
def test_small_ranges_match_oracle(b2m_gpu, a, b):
    r = b2m_gpu.chudnovsky_bs(a, b)
    got = r.signed()
    want = oracle.bs_port(a, b)
    for (sg, mg), (sw, mw) in zip(got, want):
        assert sg == sw and np.array_equal(mg, mw)
    r.free()


@pytest.mark.parametrize("digits", [1000, 100000, 1000000, 10000000])
def test_tree_roots_match_reference(b2m_gpu, digits):
    trees = {t["digits"]: t for t in json.load(open(os.path.join(GOLD, "chudnovsky.json")))["trees"]}
    if digits not in trees:
        pytest.skip("tree not in the fixtures")
    tr = trees[digits]
    r = b2m_gpu.chudnovsky_bs(0, tr["terms"])
    for which, nm in enumerate("PQT"):
        assert r.lengths[which] == tr[nm]["len"], nm
        assert sha_limbs(r.limbs(which)) == tr[nm]["sha256"], nm
    assert r.t_sign == tr["T"]["sign"]
    r.free()


@pytest.mark.parametrize("digits", [1000, 100000, 1000000])
def test_compute_pi_matches_reference_digits(b2m_gpu, digits):
    runs = {r["digits"]: r for r in json.load(open(os.path.join(GOLD, "pi_digits.json")))["runs"]}
    if digits not in runs:
        pytest.skip("digit string not in the fixtures")
    s = b2m_gpu.compute_pi(digits)
    assert s[:102] == runs[digits]["head"]
    assert hashlib.sha256(s.encode()).hexdigest() == runs[digits]["sha256"]
