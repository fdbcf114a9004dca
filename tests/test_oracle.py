"""CPU tests: pin the oracle (our C restatement of the reference's CPU path)
against the reference's own compiled code and the golden fixtures."""
import json
import os

import numpy as np
import pytest

import oracle
from golden_util import GL_P, gen_operand, selftest_pairs, sha_limbs

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return json.load(open(os.path.join(GOLD, name)))


def test_field_ops_match_reference_vectors():
    lib = oracle.port_lib()
    for r in load("field.json")["rows"]:
        a, b = r["a"], r["b"]
        assert lib.orc_gl_add(a, b) == r["add"]
        assert lib.orc_gl_sub(a, b) == r["sub"]
        assert lib.orc_gl_mul(a, b) == r["mul"] == lib.orc_gl_mul_def(a, b)
        assert lib.orc_gl_pow(a, b % 1000003) == r["pow"]
        if a:
            assert lib.orc_gl_inv(a) == r["inv"]
            assert lib.orc_gl_mul(a, r["inv"]) == 1


def test_roots_of_unity_match_reference_vectors():
    lib = oracle.port_lib()
    for k, w in load("field.json")["roots_g7"].items():
        n = 1 << int(k)
        assert lib.orc_gl_root_of_unity(n) == w
        assert lib.orc_gl_pow(w, n) == 1
        assert lib.orc_gl_pow(w, n // 2) == GL_P - 1


def test_field_identities_like_reference_selftest():
    # tests/self_test.cu:46-62 on a smaller sample
    lib = oracle.port_lib()
    rng = np.random.default_rng(5)
    for _ in range(2000):
        a, b, c = (int(x) % GL_P for x in rng.integers(0, 2**63, 3, dtype=np.uint64))
        assert lib.orc_gl_add(a, b) == lib.orc_gl_add(b, a)
        assert lib.orc_gl_sub(lib.orc_gl_add(a, b), b) == a
        assert lib.orc_gl_mul(a, lib.orc_gl_add(b, c)) == lib.orc_gl_add(lib.orc_gl_mul(a, b), lib.orc_gl_mul(a, c))


def test_selftest_pairs_match_reference_products():
    gold = load("selftest_multiply.json")["pairs"]
    assert len(gold) == 120
    for g, (na, nb, a, b) in zip(gold, selftest_pairs()):
        assert (g["na"], g["nb"], g["la"], g["lb"]) == (na, nb, a.size, b.size)
        p = oracle.mul_port(a, b)
        assert sha_limbs(p) == g["sha256"]
    # schoolbook restatement on a subset
    for i, (na, nb, a, b) in enumerate(selftest_pairs()):
        if i % 10 == 0:
            assert sha_limbs(oracle.mul_port(a, b, schoolbook=True)) == gold[i]["sha256"]


@pytest.mark.parametrize("entry", [e for e in json.load(open(os.path.join(GOLD, "sweep_small.json")))["products"]
                                   if e["na"] <= (1 << 16)], ids=lambda e: e["name"])
def test_sweep_products_match_reference(entry):
    a = gen_operand(entry["seed_a"], entry["na"], entry["kind_a"])
    b = gen_operand(entry["seed_b"], entry["nb"], entry["kind_b"])
    p = oracle.mul_port(a, b)
    assert p.size == entry["len"] and sha_limbs(p) == entry["sha256"]


def test_operand_generator_numpy_matches_c():
    for seed, n in [(1, 1), (7, 1000), (123456789, 4097)]:
        assert np.array_equal(gen_operand(seed, n), oracle.gen_operand(seed, n))
    assert np.array_equal(gen_operand(0, 10, 1), oracle.gen_operand(0, 10, 1))


def test_operand_generator_product_copy_matches():
    b200mul = pytest.importorskip("b200mul")
    for seed, n in [(1, 1), (99, 5000)]:
        assert np.array_equal(b200mul.gen_operand(seed, n), gen_operand(seed, n))


def test_carry_propagate_restatement_edge_cases():
    # coefficient vectors with long carry chains (include/ntt.h:70-91)
    lib = oracle.port_lib()
    conv = np.array([0xFFFF, 0xFFFF, 0xFFFF, 1 << 40, 0, 0, 0, 0], np.uint64)
    out = np.zeros(8, np.uint32)
    n = lib.orc_carry_propagate(conv.ctypes.data_as(oracle.ctypes.POINTER(oracle.ctypes.c_uint64)), conv.size,
                                out.ctypes.data_as(oracle._u32p), out.size)
    val = sum(int(c) << (16 * i) for i, c in enumerate(conv))
    got = sum(int(x) << (32 * i) for i, x in enumerate(out[:n]))
    assert got == val


def _bs_equal(x, y):
    return all(sx == sy and np.array_equal(mx, my) for (sx, mx), (sy, my) in zip(x, y))


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (needs the reference tree)")
def test_binary_splitting_restatement_matches_reference():
    for a, b in [(0, 1), (1, 2), (0, 2), (0, 37), (5, 90), (0, 300)]:
        assert _bs_equal(oracle.bs_port(a, b), oracle.bs_ref(a, b))


def test_binary_splitting_restatement_matches_golden():
    tree = [t for t in load("chudnovsky.json")["trees"] if t["digits"] == 1000][0] \
        if os.path.exists(os.path.join(GOLD, "chudnovsky.json")) else None
    if tree is None:
        pytest.skip("chudnovsky.json not generated")
    pqt = oracle.bs_port(0, tree["terms"])
    for nm, (sg, mag) in zip("PQT", pqt):
        assert sg == tree[nm]["sign"] and sha_limbs(mag) == tree[nm]["sha256"]


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (needs the reference tree)")
def test_reference_library_agrees_with_port_on_random_sizes():
    rng = np.random.default_rng(11)
    for _ in range(20):
        na, nb = (int(x) for x in rng.integers(1, 3000, 2))
        a = rng.integers(0, 2**32, na, dtype=np.uint64).astype(np.uint32)
        b = rng.integers(0, 2**32, nb, dtype=np.uint64).astype(np.uint32)
        r = oracle.mul_ref(a, b, "ntt-cpu")
        assert np.array_equal(r, oracle.mul_port(a, b))
        assert np.array_equal(r, oracle.mul_ref(a, b, "karatsuba"))
