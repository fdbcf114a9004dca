"""Every transform plan the autotuner may choose gives the reference's product.

b2m_autotune times each candidate plan (two- and three-pass splits, tiles of
2^12..2^14 elements) and keeps the fastest; b2m_set_plan fixes one. Each
candidate is run here on fixture products whose hashes come from the
reference's own mul_ntt_cpu (tests/golden/sweep_*.json), so whichever plan a
size ends up with, its products are bit-exact."""
import json
import os

import numpy as np
import pytest

from golden_util import gen_operand, sha_limbs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def fixture(name):
    for f in ("sweep_small.json", "sweep_large.json"):
        for p in json.load(open(os.path.join(GOLD, f)))["products"]:
            if p["name"] == name:
                return p
    raise KeyError(name)


@pytest.mark.parametrize("name", ["rand_2^14", "unbal_2^16", "ones_2^18", "rand_2^20", "unbal_2^20", "rand_2^22",
                                  "rand_2^24"])
def test_every_candidate_plan_is_exact(b2m_gpu, name):
    import torch

    fx = fixture(name)
    na, nb = fx["na"], fx["nb"]
    a = torch.from_numpy(gen_operand(fx["seed_a"], na, fx["kind_a"]).view(np.int32)).cuda()
    b = torch.from_numpy(gen_operand(fx["seed_b"], nb, fx["kind_b"]).view(np.int32)).cuda()
    out = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
    olen = torch.zeros(1, dtype=torch.int64, device="cuda")
    cands = b2m_gpu.autotune(na, nb)
    assert sum(c["chosen"] for c in cands) == 1
    logn = b2m_gpu.plan_describe(na, nb)["ntt_log2"]
    try:
        for c in cands:
            b2m_gpu.set_plan(logn, c["logr"], c["logc"])
            assert b2m_gpu.plan_describe(na, nb)["logr"] == c["logr"]
            out.zero_()
            b2m_gpu.mul_device(a.data_ptr(), na, b.data_ptr(), nb, out.data_ptr(), na + nb, olen.data_ptr(), 0)
            b2m_gpu.stream_check(0)
            n = int(olen.item())
            assert n == fx["len"], c
            assert sha_limbs(out.cpu().numpy().view(np.uint32)[:n]) == fx["sha256"], c
    finally:
        best = next(c for c in cands if c["chosen"])
        b2m_gpu.set_plan(logn, best["logr"], best["logc"])


def test_set_plan_rejects_unknown_plans(b2m_gpu):
    with pytest.raises(b2m_gpu.B2MError):
        b2m_gpu.set_plan(26, [13, 13], [1, 1])
