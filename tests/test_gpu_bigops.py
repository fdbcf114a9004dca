"""Division and square root on the device (b2m_divmod_device,
b2m_isqrt_device) against exact host integers.

The reference's divmod_knuth / div_fast and isqrt (src/bignum_div.cpp:162-204)
define floor quotient, remainder and floor root; Python's integers compute the
same three exactly, so they are the oracle here: exact equality up to a few
thousand limbs, and at large sizes the defining identities (a = q b + r with
0 <= r < b, checked exactly for r < b and modulo several 61-bit primes for the
identity; s^2 <= a < (s+1)^2, checked exactly)."""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRIMES = [(1 << 61) - 1, (1 << 61) - 507, (1 << 60) - 93, (1 << 59) - 55]


def to_limbs(v: int, n: int | None = None) -> np.ndarray:
    k = max(1, (v.bit_length() + 31) // 32) if n is None else n
    return np.frombuffer(v.to_bytes(4 * k, "little"), dtype="<u4").copy()


def to_int(a) -> int:
    return int.from_bytes(np.ascontiguousarray(a, dtype="<u4").tobytes(), "little")


def dev(b2m, arr):
    import torch

    return torch.from_numpy(np.ascontiguousarray(arr).view(np.int32)).cuda()


def gpu_divmod(b2m, a: int, b: int, pad_a: int = 0):
    import torch

    la = to_limbs(a)
    if pad_a:
        la = np.concatenate([la, np.zeros(pad_a, np.uint32)])
    lb = to_limbs(b)
    da, db = dev(b2m, la), dev(b2m, lb)
    qc, rc = max(1, la.size - lb.size + 1), lb.size
    dq = torch.zeros(qc, dtype=torch.int32, device="cuda")
    dr = torch.zeros(rc, dtype=torch.int32, device="cuda")
    ql, rl = b2m.divmod_device(da.data_ptr(), la.size, db.data_ptr(), lb.size, dq.data_ptr(), qc, dr.data_ptr(), rc)
    q = to_int(dq.cpu().numpy().view(np.uint32)[:ql])
    r = to_int(dr.cpu().numpy().view(np.uint32)[:rl])
    return q, r


def gpu_isqrt(b2m, a: int) -> int:
    import torch

    la = to_limbs(a)
    da = dev(b2m, la)
    cap = (la.size + 1) // 2 + 1
    do = torch.zeros(cap, dtype=torch.int32, device="cuda")
    n = b2m.isqrt_device(da.data_ptr(), la.size, do.data_ptr(), cap)
    return to_int(do.cpu().numpy().view(np.uint32)[:n])


def rand_int(rng: random.Random, limbs: int, top_bits: int = 32) -> int:
    v = rng.getrandbits(32 * limbs)
    top = rng.getrandbits(top_bits) | (1 << (top_bits - 1))
    return (v & ((1 << (32 * (limbs - 1))) - 1)) | (top << (32 * (limbs - 1)))


@pytest.mark.parametrize("na,nb", [(1, 1), (2, 1), (5, 3), (9, 9), (40, 1), (100, 99), (300, 17), (1000, 500),
                                   (2500, 2400), (4000, 130), (6000, 3000)])
def test_divmod_matches_python_exactly(b2m_gpu, na, nb):
    rng = random.Random(1000 * na + nb)
    for top_bits in (32, 1, 17):
        a, b = rand_int(rng, na), rand_int(rng, nb, top_bits)
        assert gpu_divmod(b2m_gpu, a, b) == divmod(a, b), (na, nb, top_bits)


def test_divmod_edge_cases(b2m_gpu):
    rng = random.Random(7)
    b = rand_int(rng, 300)
    cases = [(0, 5), (5, 7), (7, 7), (b, b), (b - 1, b), (b * 12345, b), (b * b, b), (b * b - 1, b),
             ((1 << (32 * 700)) - 1, (1 << (32 * 300)) - 1), ((1 << (32 * 700)) - 1, 1 << (32 * 299)),
             (1 << (32 * 500), 3), (rand_int(rng, 900), 1), (rand_int(rng, 50), (1 << 32) - 1)]
    for a, d in cases:
        assert gpu_divmod(b2m_gpu, a, d) == divmod(a, d), (a.bit_length(), d.bit_length())
    # operands with leading zero limbs, as the reference's BigInt may carry
    a = rand_int(rng, 77)
    assert gpu_divmod(b2m_gpu, a, b, pad_a=5) == divmod(a, b)


@pytest.mark.parametrize("na,nb", [(1 << 16, 1 << 15), (1 << 18, 1 << 10), (1 << 20, 1 << 19), (300000, 299999)])
def test_divmod_large_identities(b2m_gpu, na, nb):
    rng = random.Random(na ^ (nb << 3))
    a, b = rand_int(rng, na), rand_int(rng, nb, 5)
    q, r = gpu_divmod(b2m_gpu, a, b)
    assert 0 <= r < b
    for p in PRIMES:
        assert (q % p) * (b % p) % p == (a - r) % p


@pytest.mark.parametrize("limbs", [1, 2, 3, 4, 5, 8, 9, 33, 100, 1001, 4096, 20000, 1 << 17])
def test_isqrt_matches_definition(b2m_gpu, limbs):
    import math

    rng = random.Random(limbs)
    for top_bits in (32, 1, 9):
        a = rand_int(rng, limbs, top_bits)
        s = gpu_isqrt(b2m_gpu, a)
        if limbs <= 4096:
            assert s == math.isqrt(a)
        else:
            assert s * s <= a < (s + 1) * (s + 1)


def test_isqrt_edge_cases(b2m_gpu):
    import math

    rng = random.Random(3)
    x = rand_int(rng, 400)
    for a in [0, 1, 2, 3, 4, 15, 16, 17, (1 << 64) - 1, 1 << 64, (1 << 128) - 1, 1 << 128, x * x, x * x - 1,
              x * x + 1, (x + 1) * (x + 1) - 1, (1 << (32 * 801)) - 1, 10005 * 10 ** 2032]:
        assert gpu_isqrt(b2m_gpu, a) == math.isqrt(a), a.bit_length()


def gpu_decimal(b2m, a: int, pad: int = 0) -> str:
    la = to_limbs(a)
    if pad:
        la = np.concatenate([la, np.zeros(pad, np.uint32)])
    da = dev(b2m, la)
    return b2m.to_decimal_device(da.data_ptr(), la.size)


@pytest.mark.parametrize("limbs", [1, 2, 7, 8, 9, 30, 250, 1000, 3333, 20000, 100000])
def test_to_decimal_matches_python(b2m_gpu, limbs):
    import sys

    sys.set_int_max_str_digits(0)
    rng = random.Random(limbs + 99)
    for top_bits in (32, 1):
        a = rand_int(rng, limbs, top_bits)
        assert gpu_decimal(b2m_gpu, a) == str(a)


def test_to_decimal_edge_cases(b2m_gpu):
    import sys

    sys.set_int_max_str_digits(0)
    for a in [0, 1, 9, 10, 999999999, 10 ** 9, 10 ** 18 - 1, 10 ** 18, 10 ** 72 - 1, 10 ** 72, 10 ** 72 + 1,
              10 ** 144 - 1, 10 ** 144, 10 ** 1152, 10 ** 1152 - 1, 10 ** 4608 + 7, (1 << 32 * 500) - 1,
              3 * 10 ** 20000 + 1]:
        assert gpu_decimal(b2m_gpu, a) == str(a), len(str(a))
    assert gpu_decimal(b2m_gpu, 12345, pad=9) == "12345"


def test_compute_pi_short_strings(b2m_gpu):
    import json
    import os

    head = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pi_digits.json")))["runs"][0]["head"]
    assert b2m_gpu.compute_pi(0) == "3"
    for d in (1, 2, 5, 50, 100):
        assert b2m_gpu.compute_pi(d) == head[: 2 + d]


def test_host_buffer_forms(b2m_gpu):
    """b2m_divmod_host / b2m_isqrt_host / b2m_to_decimal_host: the shapes the
    reference's BigInt seams (div_fast, isqrt, to_decimal) would call."""
    import math
    import sys

    sys.set_int_max_str_digits(0)
    rng = random.Random(11)
    for na, nb in [(1, 1), (50, 7), (3000, 1000)]:
        a, b = rand_int(rng, na), rand_int(rng, nb, 9)
        q, r = b2m_gpu.divmod_host(to_limbs(a), to_limbs(b))
        assert (to_int(q), to_int(r)) == divmod(a, b)
        assert to_int(b2m_gpu.isqrt_host(to_limbs(a))) == math.isqrt(a)
        assert b2m_gpu.to_decimal_host(to_limbs(a)) == str(a)
    assert b2m_gpu.to_decimal_host(np.zeros(3, np.uint32)) == "0"
