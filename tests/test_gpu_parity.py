"""GPU parity tests: the CUDA path, called through the C ABI, against the
reference's products (golden fixtures made by the reference's compiled CPU
code) and against the oracle restatement, bit for bit.

Sizes cover every transform plan: the single-CTA path (N = 2^2 .. 2^13), the
two-pass plans (2^14 .. 2^26) and, through size-independent properties, the
three-pass plans. Edge cases follow the reference's tests (tests/self_test.cu
:64-78) and add what they lack: all-0xFFFFFFFF operands (longest carry runs),
1:8 unbalanced operands, leading zero limbs, zero operands, empty operands.
"""
import json
import os

import numpy as np
import pytest

import oracle
from golden_util import gen_operand, selftest_pairs, sha_limbs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    path = os.path.join(GOLD, name)
    return json.load(open(path)) if os.path.exists(path) else None


def test_selftest_pairs(b2m_gpu):
    """The reference self-test's 120 multiply pairs (tests/self_test.cu:64-78)."""
    gold = load("selftest_multiply.json")["pairs"]
    for g, (na, nb, a, b) in zip(gold, selftest_pairs()):
        p = b2m_gpu.mul_ntt_cuda(a, b)
        assert sha_limbs(p) == g["sha256"], (na, nb)


# N = ntt_length(na, nb) for each case; every plan and boundary is hit.
EDGE = [(1, 1), (1, 2), (2, 1), (1, 3), (3, 5), (7, 9), (15, 16), (16, 16), (31, 33), (64, 64), (100, 28),
        (511, 512), (1024, 1024), (1024, 1025), (2047, 2048), (2048, 2048), (2048, 2049), (4095, 4096),
        (4096, 4096), (4096, 1), (1, 8191), (8192, 8192), (8193, 10000), (16384, 16384), (30000, 2),
        (65536, 65536), (100000, 31000), (131072, 131072), (200000, 200001)]


@pytest.mark.parametrize("na,nb", EDGE)
@pytest.mark.parametrize("kind", [0, 1])
def test_edge_sizes_against_oracle(b2m_gpu, na, nb, kind):
    a = gen_operand(na * 31 + 7, na, kind)
    b = gen_operand(nb * 17 + 3, nb, kind)
    p = b2m_gpu.mul_ntt_cuda(a, b)
    q = oracle.mul_port(a, b)
    assert p.size == q.size and np.array_equal(p, q)


def runs_operand(seed, n):
    """n limbs in runs of 0xFFFFFFFF, zero and random limbs, run lengths
    1..6000 (so runs cross the carry kernel's 2048-limb chunks), top limb
    non-zero."""
    rng = np.random.default_rng(seed)
    out = np.empty(n, np.uint32)
    i, run = 0, int(rng.integers(0, 3))
    while i < n:
        k = min(n - i, int(rng.integers(1, 6001)))
        kind = run % 3  # all ones, zeros, random in turn
        out[i:i + k] = (0xFFFFFFFF if kind == 0 else 0) if kind < 2 else rng.integers(0, 1 << 32, k, np.uint64)
        i += k
        run += 1
    out[-1] |= 1
    return out


def ones_plus(n, m):
    """(2^(32n) - 1, 2^(32m) + 1): their product has 0xFFFFFFFF runs of n - m
    limbs between sparse limbs, so whole carry chunks are all ones while
    their neighbours are not."""
    a = np.full(n, 0xFFFFFFFF, np.uint32)
    b = np.zeros(m + 1, np.uint32)
    b[0] = b[m] = 1
    return a, b


@pytest.mark.parametrize("na,nb", [(1 << 14, 1 << 14), (1 << 16, 1 << 15), (1 << 17, 1 << 17), (50000, 70001),
                                   (262144, 8192)])
def test_structured_runs_against_oracle(b2m_gpu, na, nb):
    """Carry stress: operands made of long runs, so that some chunks of the
    carry resolve by the scan-free path, others by the full scan, and the
    lookback crosses both kinds of aggregate (include/ntt.h:70-91)."""
    a, b = runs_operand(na, na), runs_operand(nb + 1, nb)
    p = b2m_gpu.mul_ntt_cuda(a, b)
    q = oracle.mul_port(a, b)
    assert p.size == q.size and np.array_equal(p, q)


@pytest.mark.parametrize("n,m", [(20000, 3000), (70000, 65536), (131072, 1), (150000, 40000)])
def test_all_ones_run_products_against_oracle(b2m_gpu, n, m):
    a, b = ones_plus(n, m)
    p = b2m_gpu.mul_ntt_cuda(a, b)
    q = oracle.mul_port(a, b)
    assert p.size == q.size and np.array_equal(p, q)


@pytest.mark.parametrize("entry", (load("sweep_small.json") or {"products": []})["products"],
                         ids=lambda e: e["name"])
def test_sweep_against_reference_hashes(b2m_gpu, entry):
    a = gen_operand(entry["seed_a"], entry["na"], entry["kind_a"])
    b = gen_operand(entry["seed_b"], entry["nb"], entry["kind_b"])
    p = b2m_gpu.mul_ntt_cuda(a, b)
    assert p.size == entry["len"] and sha_limbs(p) == entry["sha256"]


def _sweep_entries(*names):
    out = []
    for nm in names:
        out += (load(nm) or {"products": []})["products"]
    return out


# Every power of two from 2^17 to 2^27 limbs (transforms of 2^19 .. 2^29
# points: two- and three-pass plans, the largest the default sweep reaches),
# random, all-0xFFFFFFFF and 1:8 unbalanced, against the reference's own
# mul_ntt_cpu hashes.
@pytest.mark.parametrize("entry", _sweep_entries("sweep_odd.json", "sweep_large.json", "sweep_xl.json"),
                         ids=lambda e: e["name"])
def test_large_sweep_against_reference_hashes(b2m_gpu, entry):
    a = gen_operand(entry["seed_a"], entry["na"], entry["kind_a"])
    b = gen_operand(entry["seed_b"], entry["nb"], entry["kind_b"])
    p = b2m_gpu.mul_ntt_cuda(a, b)
    assert p.size == entry["len"] and sha_limbs(p) == entry["sha256"]


def test_leading_zero_limbs_are_trimmed(b2m_gpu):
    a = np.concatenate([gen_operand(5, 3000), np.zeros(500, np.uint32)])
    b = np.concatenate([gen_operand(6, 20000), np.zeros(7, np.uint32)])
    p = b2m_gpu.mul_ntt_cuda(a, b)
    q = oracle.mul_port(np.trim_zeros(a, "b"), np.trim_zeros(b, "b"))
    assert np.array_equal(p, q)


def test_zero_and_empty_operands(b2m_gpu):
    z = np.zeros(40000, np.uint32)
    assert b2m_gpu.mul_ntt_cuda(z, gen_operand(1, 40000)).size == 0
    assert b2m_gpu.mul_ntt_cuda(np.zeros(3, np.uint32), np.ones(2, np.uint32)).size == 0
    assert b2m_gpu.mul_ntt_cuda(np.zeros(0, np.uint32), np.ones(2, np.uint32)).size == 0


def test_output_too_small_is_an_error(b2m_gpu):
    a = gen_operand(1, 10)
    with pytest.raises(b2m_gpu.B2MError) as ei:
        b2m_gpu.mul_ntt_cuda(a, a, out=np.zeros(19, np.uint32))
    assert ei.value.status == b2m_gpu.OUTPUT_TOO_SMALL


def test_product_properties_three_pass_plan(b2m_gpu):
    """2^27 x 2^27 limbs: N = 2^29, the three-pass plan. Checked through
    size-independent properties: (x * y) mod m for small m equals
    ((x mod m)(y mod m)) mod m, the product is symmetric, and the low/high
    limbs agree with exact partial products."""
    n = 1 << 27
    a = gen_operand(71, n)
    b = gen_operand(72, n)
    p = b2m_gpu.mul_ntt_cuda(a, b)
    assert p.size in (2 * n, 2 * n - 1)
    # low 64 limbs: (a mod B^64)(b mod B^64) mod B^64
    low = oracle.mul_port(a[:64], b[:64])[:64]
    assert np.array_equal(p[:64], low)
    # residues modulo 2^32-1 and 2^32+1 via limb sums
    def mod_m(x, m, sign):
        # x mod (2^32 - 1) is the limb sum; x mod (2^32 + 1) the alternating limb sum
        acc = 0
        for i in range(0, x.size, 1 << 20):
            chunk = x[i:i + (1 << 20)].astype(np.int64)
            if sign < 0:
                chunk = chunk * np.where((np.arange(chunk.size) + i) % 2 == 0, 1, -1)
            acc = (acc + int(chunk.sum())) % m
        return acc
    for m, sign in [((1 << 32) - 1, 1), ((1 << 32) + 1, -1)]:
        assert mod_m(p, m, sign) == (mod_m(a, m, sign) * mod_m(b, m, sign)) % m


def test_device_pointer_entry_point(b2m_gpu):
    torch = pytest.importorskip("torch")
    na, nb = 70000, 50000
    a = gen_operand(3, na)
    b = gen_operand(4, nb)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    dout = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
    dlen = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    b2m_gpu.mul_device(da.data_ptr(), na, db.data_ptr(), nb, dout.data_ptr(), na + nb, dlen.data_ptr(),
                       s.cuda_stream)
    b2m_gpu.stream_check(s.cuda_stream)
    n = int(dlen.item())
    p = dout.cpu().numpy().view(np.uint32)
    q = oracle.mul_port(a, b)
    assert n == q.size and np.array_equal(p[:n], q) and not p[n:].any()


def test_repeated_calls_are_deterministic(b2m_gpu):
    a = gen_operand(9, 300000)
    b = gen_operand(10, 123457)
    p1 = b2m_gpu.mul_ntt_cuda(a, b).copy()
    p2 = b2m_gpu.mul_ntt_cuda(b, a).copy()
    p3 = b2m_gpu.mul_ntt_cuda(a, b).copy()
    assert np.array_equal(p1, p2) and np.array_equal(p1, p3)
