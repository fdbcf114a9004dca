"""Generate the golden fixtures in this directory from the reference's own
compiled CPU code (oracle/_ref/libpidigits_ref.so, built by `make -C oracle ref`
from the reference sources).

    python tests/golden/make_golden.py small      # field, self-test pairs, C1, sweep <= 2^20
    python tests/golden/make_golden.py large      # sweep 2^22 and 2^24 (minutes)
    python tests/golden/make_golden.py odd        # sweep 2^17, 2^19, 2^21, 2^23 (minutes)
    python tests/golden/make_golden.py xl         # sweep 2^25 .. 2^27 (about an hour of CPU,
                                                  # three worker processes, ~13 GB each at 2^27)
    python tests/golden/make_golden.py chudnovsky # P/Q/T of the binary-splitting trees
    python tests/golden/make_golden.py pi         # digit strings of compute_pi_chudnovsky

Fixtures hold seeds, sizes and SHA-256 hashes of products (little-endian u32
limbs, trimmed), never the large operands themselves: operands are re-made
from their seeds by the generator in b200mul.gen_operand (the same generator
exists in C in oracle/gl_oracle.c, and the tests check that the two agree).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from golden_util import (gen_operand, selftest_pairs, sha_limbs, SWEEP_SMALL, SWEEP_LARGE,  # noqa: E402
                         SWEEP_ODD, SWEEP_XL, GL_P)


def dump(name, obj):
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, indent=1)
    print("wrote", name)


def make_field():
    ref = oracle.ref_lib()
    rng = np.random.default_rng(20261203)
    vals = [int(x) % GL_P for x in rng.integers(0, 2**63, 200, dtype=np.uint64)]
    vals += [0, 1, 2, GL_P - 1, GL_P - 2, 0xFFFFFFFF, 0x100000000, 0xFFFFFFFF00000000, 2**63]
    rows = []
    for i, a in enumerate(vals):
        b = vals[(i * 7 + 3) % len(vals)]
        rows.append({"a": a, "b": b, "add": ref.ref_gl_add(a, b), "sub": ref.ref_gl_sub(a, b),
                     "mul": ref.ref_gl_mul(a, b), "pow": ref.ref_gl_pow(a, b % 1000003),
                     "inv": ref.ref_gl_inv(a) if a else 0})
    roots = {str(k): ref.ref_gl_root_of_unity(1 << k) for k in range(1, 33)}
    dump("field.json", {"source": "include/goldilocks.h via oracle/_ref", "rows": rows, "roots_g7": roots})


def make_selftest():
    rows = []
    for na, nb, a, b in selftest_pairs():
        p = oracle.mul_ref(a, b, "schoolbook")
        assert np.array_equal(p, oracle.mul_ref(a, b, "ntt-cpu"))
        rows.append({"na": na, "nb": nb, "la": int(a.size), "lb": int(b.size), "len": int(p.size),
                     "sha256": sha_limbs(p)})
    dump("selftest_multiply.json", {
        "source": "tests/self_test.cu:38-78 RNG stream, products by the reference's mul_schoolbook "
                  "(== mul_ntt_cpu) via oracle/_ref", "pairs": rows})


def make_sweep(entries, name):
    out = []
    for e in entries:
        a = gen_operand(e["seed_a"], e["na"], e["kind_a"])
        b = gen_operand(e["seed_b"], e["nb"], e["kind_b"])
        t = time.time()
        p = oracle.mul_ref(a, b, "ntt-cpu")
        dt = time.time() - t
        r = dict(e)
        r.update({"len": int(p.size), "sha256": sha_limbs(p), "ref_ntt_cpu_s": round(dt, 3)})
        out.append(r)
        print(e["name"], p.size, f"{dt:.2f}s", flush=True)
    dump(name, {"source": "reference mul_ntt_cpu (src/ntt_cpu.cpp:111-129) via oracle/_ref, "
                          "1 thread of this container's host", "products": out})


def _sweep_row(e):
    a = gen_operand(e["seed_a"], e["na"], e["kind_a"])
    b = gen_operand(e["seed_b"], e["nb"], e["kind_b"])
    t = time.time()
    p = oracle.mul_ref(a, b, "ntt-cpu")
    dt = time.time() - t
    r = dict(e)
    r.update({"len": int(p.size), "sha256": sha_limbs(p), "ref_ntt_cpu_s": round(dt, 3)})
    print(e["name"], p.size, f"{dt:.2f}s", flush=True)
    return r


def make_sweep_parallel(entries, name, workers):
    """The same rows as make_sweep, one reference product per worker process
    (each product is single-threaded), largest first."""
    import multiprocessing as mp

    order = sorted(range(len(entries)), key=lambda i: -(entries[i]["na"] + entries[i]["nb"]))
    with mp.get_context("spawn").Pool(workers) as pool:
        rows = pool.map(_sweep_row, [entries[i] for i in order], chunksize=1)
    out = [None] * len(entries)
    for i, r in zip(order, rows):
        out[i] = r
    dump(name, {"source": "reference mul_ntt_cpu (src/ntt_cpu.cpp:111-129) via oracle/_ref, "
                          "1 thread of this container's host per product", "products": out})


def make_chudnovsky(digit_list):
    ref = oracle.ref_lib()
    rows = []
    for d in digit_list:
        n = ref.ref_chudnovsky_terms_for_digits(d + 16)
        t = time.time()
        pqt = oracle.bs_ref(0, n, "ntt-cpu" if n > 2000 else "auto")
        dt = time.time() - t
        row = {"digits": d, "terms": int(n), "ref_s": round(dt, 2)}
        for nm, (sg, mag) in zip("PQT", pqt):
            row[nm] = {"sign": int(sg), "len": int(mag.size), "sha256": sha_limbs(mag)}
        rows.append(row)
        print("bs", d, n, f"{dt:.1f}s", flush=True)
    path = os.path.join(HERE, "chudnovsky.json")
    old = json.load(open(path))["trees"] if os.path.exists(path) else []
    keep = [r for r in old if r["digits"] not in digit_list]
    dump("chudnovsky.json", {"source": "reference chudnovsky_bs(0, terms) (src/chudnovsky.cpp:64-102) "
                                       "with the NttCpu backend via oracle/_ref",
                             "trees": sorted(keep + rows, key=lambda r: r["digits"])})


def make_pi(digit_list):
    path = os.path.join(HERE, "pi_digits.json")
    old = json.load(open(path))["runs"] if os.path.exists(path) else []
    rows = [r for r in old if r["digits"] not in digit_list]
    for d in digit_list:
        t = time.time()
        s = oracle.compute_pi_ref(d)
        rows.append({"digits": d, "sha256": hashlib.sha256(s.encode()).hexdigest(),
                     "head": s[:102], "ref_s": round(time.time() - t, 2)})
        print("pi", d, f"{time.time() - t:.1f}s", flush=True)
    dump("pi_digits.json", {"source": "reference compute_pi_chudnovsky (src/chudnovsky.cpp:107-164) via "
                                      "oracle/_ref", "runs": sorted(rows, key=lambda r: r["digits"])})


if __name__ == "__main__":
    what = sys.argv[1:] or ["small"]
    if "small" in what:
        make_field()
        make_selftest()
        make_sweep(SWEEP_SMALL, "sweep_small.json")
    if "large" in what:
        make_sweep(SWEEP_LARGE, "sweep_large.json")
    if "odd" in what:
        make_sweep_parallel(SWEEP_ODD, "sweep_odd.json", 4)
    if "xl" in what:
        make_sweep_parallel(SWEEP_XL, "sweep_xl.json", 3)
    if "chudnovsky" in what:
        make_chudnovsky([1000, 100000, 1000000])
    if "chudnovsky10m" in what:
        make_chudnovsky([10000000])
    if "pi" in what:
        make_pi([1000, 3500, 10000, 100000])
    if "pi1m" in what:
        make_pi([1000, 3500, 10000, 100000, 1000000])
    if "pi3m" in what:
        make_pi([3000000])
