"""Products on 3 * 2^k-point transforms (a radix-3 step around three 2^k-point
transforms), used when 2(na + nb) <= 3 * 2^k < next_pow2(2(na + nb)).

The reference's product is the integer; these sizes are checked against the
oracle's C port of the reference's CPU NTT (oracle/gl_oracle.c) up to ~10^6
limbs, and above that through residues (mod 2^32 - 1, 2^32 + 1 and 61-bit
primes) and exact low limbs."""
import numpy as np
import pytest

import oracle
from golden_util import gen_operand

pytestmark = pytest.mark.gpu

PRIMES = [(1 << 61) - 1, (1 << 61) - 507]


def to_int(x) -> int:
    return int.from_bytes(np.ascontiguousarray(x, dtype="<u4").tobytes(), "little")


@pytest.mark.parametrize("na,nb,kind", [(20000, 20000, 0), (40000, 9000, 0), (24000, 24000, 1), (45000, 4000, 1),
                                        (32769, 16383, 0), (100000, 90000, 0), (700000, 700000, 0),
                                        (1300000, 200000, 1)])
def test_radix3_products_match_oracle(b2m_gpu, na, nb, kind):
    plan = b2m_gpu.plan_describe(na, nb)
    assert plan["three"] == 1 and plan["points"] >= 2 * (na + nb) > plan["points"] * 2 // 3
    a = gen_operand(na * 7 + 1, na, kind)
    b = gen_operand(nb * 5 + 3, nb, kind)
    assert np.array_equal(b2m_gpu.mul_ntt_cuda(a, b), oracle.mul_port(a, b))


def test_power_of_two_sizes_keep_power_of_two_transforms(b2m_gpu):
    for na, nb in [(1 << 16, 1 << 16), (60000, 60000), (1 << 20, 1 << 20)]:
        assert b2m_gpu.plan_describe(na, nb)["three"] == 0


def test_radix3_large_product_properties(b2m_gpu):
    """12M x 12M limbs: 3 * 2^24 points."""
    n = 12_000_000
    assert b2m_gpu.plan_describe(n, n)["three"] == 1
    a = gen_operand(91, n)
    b = gen_operand(92, n)
    p = b2m_gpu.mul_ntt_cuda(a, b)
    assert p.size in (2 * n, 2 * n - 1)
    assert np.array_equal(p[:64], oracle.mul_port(a[:64], b[:64])[:64])
    ia, ib, ip = to_int(a), to_int(b), to_int(p)
    for q in PRIMES + [(1 << 32) - 1, (1 << 32) + 1]:
        assert ip % q == (ia % q) * (ib % q) % q


def test_radix3_in_batches_and_autotune(b2m_gpu):
    import torch

    sizes = [(20000, 20000), (40000, 9000), (4000, 3000), (1 << 15, 1 << 15), (24000, 24000), (100, 77)]
    ops = [(gen_operand(11 + i, na), gen_operand(31 + i, nb)) for i, (na, nb) in enumerate(sizes)]
    dev = [(torch.from_numpy(a.view(np.int32)).cuda(), torch.from_numpy(b.view(np.int32)).cuda()) for a, b in ops]
    outs = [torch.zeros(na + nb, dtype=torch.int32, device="cuda") for na, nb in sizes]
    lens = torch.zeros(len(sizes), dtype=torch.int64, device="cuda")
    jobs = [(da.data_ptr(), na, db.data_ptr(), nb, o.data_ptr(), na + nb, lens.data_ptr() + 8 * i)
            for i, ((na, nb), (da, db), o) in enumerate(zip(sizes, dev, outs))]
    bt = b2m_gpu.Batch(jobs, b2m_gpu.BATCH_GRAPH | b2m_gpu.BATCH_AUTOTUNE)
    bt.launch(0)
    b2m_gpu.stream_check(0)
    bt.close()
    for i, ((a, b), o) in enumerate(zip(ops, outs)):
        n = int(lens[i].item())
        assert np.array_equal(o.cpu().numpy().view(np.uint32)[:n], oracle.mul_port(a, b)), sizes[i]
    # every candidate plan of a radix-3 size is exact too
    na, nb = 40000, 9000
    a, b = ops[1]
    cands = b2m_gpu.autotune(na, nb)
    logn = b2m_gpu.plan_describe(na, nb)["ntt_log2"]
    want = oracle.mul_port(a, b)
    try:
        for c in cands:
            b2m_gpu.set_plan(logn, c["logr"], c["logc"])
            assert np.array_equal(b2m_gpu.mul_ntt_cuda(a, b), want), c
    finally:
        best = next(c for c in cands if c["chosen"])
        b2m_gpu.set_plan(logn, best["logr"], best["logc"])
