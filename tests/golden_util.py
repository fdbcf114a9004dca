"""Shared helpers of the tests and of tests/golden/make_golden.py.

* ``selftest_pairs()`` replays the reference self-test's deterministic stream
  (tests/self_test.cu:38-44 xorshift64, seed 0x9e3779b97f4a7c15): 60,000 draws
  by the field test (:48-54, three per iteration), then 120 multiply pairs with
  na, nb = 1 + rnd32() % 1500 and limbs from rnd32(), normalised (:64-72).
* ``gen_operand`` is the seeded operand generator (numpy copy; the product has
  one in b200mul.py and the oracle one in C -- the tests compare all three).
* ``SWEEP_SMALL`` / ``SWEEP_LARGE`` / ``SWEEP_ODD`` / ``SWEEP_XL`` name the
  single-product workloads: the 60,000-limb product and the size sweep over
  every power of two from 2^12 to 2^27 limbs, each with random,
  all-0xFFFFFFFF and 1:8 unbalanced operands.
"""
from __future__ import annotations

import hashlib

import numpy as np

GL_P = 0xFFFFFFFF00000001
_M64 = (1 << 64) - 1
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def sha_limbs(p: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(p, dtype="<u4").tobytes()).hexdigest()


def gen_operand(seed: int, n: int, kind: int = 0) -> np.ndarray:
    if kind == 1:
        return np.full(n, 0xFFFFFFFF, np.uint32)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(1, n + 1, dtype=np.uint64) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    out = (z >> np.uint64(32)).astype(np.uint32)
    if n and out[-1] == 0:
        out[-1] = 1
    return out


class XorShift:
    """tests/self_test.cu:38-40."""

    def __init__(self, state: int = 0x9E3779B97F4A7C15):
        self.s = state

    def rnd64(self) -> int:
        s = self.s
        s ^= (s << 13) & _M64
        s ^= s >> 7
        s ^= (s << 17) & _M64
        self.s = s
        return s

    def rnd32(self) -> int:
        return self.rnd64() & 0xFFFFFFFF


def selftest_pairs():
    """Yield (na, nb, a, b) exactly as test_multiply draws them."""
    rng = XorShift()
    for _ in range(60000):
        rng.rnd64()
    for _ in range(120):
        na = 1 + rng.rnd32() % 1500
        nb = 1 + rng.rnd32() % 1500
        a = np.array([rng.rnd32() for _ in range(na)], np.uint32)
        b = np.array([rng.rnd32() for _ in range(nb)], np.uint32)
        a = np.trim_zeros(a, "b")
        b = np.trim_zeros(b, "b")
        yield na, nb, a, b


def _sweep(logs, seed0):
    out = []
    for lg in logs:
        n = 1 << lg
        out.append({"name": f"rand_2^{lg}", "na": n, "nb": n, "seed_a": seed0 + 2 * lg, "seed_b": seed0 + 2 * lg + 1,
                    "kind_a": 0, "kind_b": 0})
        out.append({"name": f"ones_2^{lg}", "na": n, "nb": n, "seed_a": 0, "seed_b": 0, "kind_a": 1, "kind_b": 1})
        out.append({"name": f"unbal_2^{lg}", "na": n, "nb": n // 8, "seed_a": seed0 + 2 * lg + 100,
                    "seed_b": seed0 + 2 * lg + 101, "kind_a": 0, "kind_b": 0})
    return out


C1 = {"name": "c1_60000", "na": 60000, "nb": 60000, "seed_a": 1, "seed_b": 2, "kind_a": 0, "kind_b": 0}
SWEEP_SMALL = [C1] + _sweep([12, 14, 16, 18, 20], 1000)
SWEEP_LARGE = _sweep([22, 24], 1000)
# The odd powers between (2^17 .. 2^23 limbs) and the top of the sweep
# (2^25 .. 2^27 limbs: transforms of 2^27 .. 2^29 points).
SWEEP_ODD = _sweep([17, 19, 21, 23], 1000)
SWEEP_XL = _sweep([25, 26, 27], 1000)
