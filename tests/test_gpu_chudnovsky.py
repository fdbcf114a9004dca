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
import ranks
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


@pytest.mark.parametrize("digits", [1000, 100000, 1000000, 3000000])
def test_compute_pi_matches_reference_digits(b2m_gpu, digits):
    runs = {r["digits"]: r for r in json.load(open(os.path.join(GOLD, "pi_digits.json")))["runs"]}
    if digits not in runs:
        pytest.skip("digit string not in the fixtures")
    s = b2m_gpu.compute_pi(digits)
    assert s[:102] == runs[digits]["head"]
    assert hashlib.sha256(s.encode()).hexdigest() == runs[digits]["sha256"]


def test_ten_million_digit_string_prefix_matches_reference(b2m_gpu):
    """The 10,000,000-digit string (the Chudnovsky config): its leading
    3,000,000 digits equal the reference's own 3,000,000-digit run
    (src/chudnovsky.cpp:107-164 via oracle/_ref, 4,220 s on one core)."""
    runs = {r["digits"]: r for r in json.load(open(os.path.join(GOLD, "pi_digits.json")))["runs"]}
    d = max(runs)
    s = b2m_gpu.compute_pi(10000000)
    assert len(s) == 10000002 and s[:102] == runs[d]["head"]
    assert hashlib.sha256(s[: 2 + d].encode()).hexdigest() == runs[d]["sha256"]


@pytest.mark.parametrize("digits", [1000, 100000, 1000000])
def test_split_and_merged_trees_equal_the_reference_root(b2m_gpu, digits):
    """The tree split into subtrees (as ranks.py splits it over GPUs) and
    merged with b2m_pqt_merge, subtree roots moved through b2m_pqt_import on
    the way, equals the reference's root."""
    tr = next(t for t in json.load(open(os.path.join(GOLD, "chudnovsky.json")))["trees"] if t["digits"] == digits)
    n = tr["terms"]
    for world in (2, 3, 8):
        nodes = []
        for a, b in ranks.term_ranges(n, world):
            r = b2m_gpu.chudnovsky_bs(a, b)
            moved = b2m_gpu.pqt_import([b2m_gpu.lib.b2m_pqt_device(r.handle, f) for f in range(3)],
                                       r.lengths, r.t_sign)
            r.free()
            nodes.append(moved)
        # the same pairwise order as ranks.merge_schedule
        held = dict(enumerate(nodes))
        for step in ranks.merge_schedule(world):
            for dst, src in step:
                m = b2m_gpu.pqt_merge(held[dst], held[src])
                held[dst].free()
                held.pop(src).free()
                held[dst] = m
        root = held[0]
        for which, nm in enumerate("PQT"):
            assert root.lengths[which] == tr[nm]["len"], (world, nm)
            assert sha_limbs(root.limbs(which)) == tr[nm]["sha256"], (world, nm)
        assert root.t_sign == tr["T"]["sign"]
        root.free()


def test_pqt_merge_small_ranges_match_oracle(b2m_gpu):
    for a, b, c in [(0, 1, 2), (0, 5, 9), (3, 4, 40), (10, 200, 201)]:
        left, right = b2m_gpu.chudnovsky_bs(a, b), b2m_gpu.chudnovsky_bs(b, c)
        m = b2m_gpu.pqt_merge(left, right)
        for (sg, mg), (sw, mw) in zip(m.signed(), oracle.bs_port(a, c)):
            assert sg == sw and np.array_equal(mg, mw)
        for x in (left, right, m):
            x.free()
