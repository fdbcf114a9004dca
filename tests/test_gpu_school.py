"""The schoolbook path of the one-CTA product kernel, and squares.

Products of at most 2^13 transform points whose na * nb is at most 128 N
limb multiply-adds are computed by schoolbook columns (96-bit
column sums, a block scan of carry functions) instead of the one-CTA NTT.
These cases sit on both sides of that choice at every one-CTA length, with
the operands that stress it most: all-0xFFFFFFFF limbs (the largest column
sums and the longest carry runs), one-limb and very unbalanced operands, and
leading zero limbs. Checked bit for bit against the oracle's port of the
reference's CPU product, through single calls and through one batch.
"""
import numpy as np
import pytest

import oracle
from golden_util import gen_operand

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 3), (5, 4), (8, 8), (13, 19), (16, 16), (32, 31), (40, 24), (64, 64), (65, 63), (96, 160),
          (128, 128), (200, 56), (255, 257), (256, 256), (300, 212), (511, 1), (512, 512), (600, 424),
          (700, 700), (1000, 24), (1024, 1024), (1100, 900), (1300, 1300), (1500, 1500), (1800, 2000),
          (2048, 2048), (4000, 96), (4095, 1), (1, 4095), (3000, 1000)]


@pytest.mark.parametrize("na,nb", SHAPES)
@pytest.mark.parametrize("kind", [0, 1])
def test_school_shapes_against_oracle(b2m_gpu, na, nb, kind):
    a = gen_operand(na * 13 + nb, na, kind)
    b = gen_operand(nb * 7 + na + 1, nb, kind)
    p = b2m_gpu.mul_ntt_cuda(a, b)
    assert np.array_equal(p, oracle.mul_port(a, b)), (na, nb, kind)


def test_school_leading_zero_limbs(b2m_gpu):
    a = np.concatenate([gen_operand(5, 300, 1), np.zeros(40, dtype=np.uint32)])
    b = np.concatenate([gen_operand(6, 77), np.zeros(3, dtype=np.uint32)])
    assert np.array_equal(b2m_gpu.mul_ntt_cuda(a, b), oracle.mul_port(a, b))


def test_school_in_one_batch(b2m_gpu):
    import torch

    rng = np.random.default_rng(2026)
    sizes = [(int(x), int(y)) for x, y in rng.integers(1, 2049, size=(300, 2))]
    sizes += [(2048, 2048), (1, 1), (4000, 60)]
    ops = [(gen_operand(3 * i + 1, na, i % 3 == 0), gen_operand(3 * i + 2, nb, i % 5 == 0))
           for i, (na, nb) in enumerate(sizes)]
    dev = [(torch.from_numpy(a.view(np.int32)).cuda(), torch.from_numpy(b.view(np.int32)).cuda()) for a, b in ops]
    outs = [torch.zeros(na + nb, dtype=torch.int32, device="cuda") for na, nb in sizes]
    lens = torch.zeros(len(sizes), dtype=torch.int64, device="cuda")
    jobs = [(da.data_ptr(), na, db.data_ptr(), nb, o.data_ptr(), na + nb, lens.data_ptr() + 8 * i)
            for i, ((na, nb), (da, db), o) in enumerate(zip(sizes, dev, outs))]
    bt = b2m_gpu.Batch(jobs, b2m_gpu.BATCH_GRAPH)
    bt.launch(0)
    b2m_gpu.stream_check(0)
    bt.close()
    for i, ((a, b), o) in enumerate(zip(ops, outs)):
        want = oracle.mul_port(a, b)
        n = int(lens[i].item())
        assert n == want.size and np.array_equal(o.cpu().numpy().view(np.uint32)[:n], want), sizes[i]


@pytest.mark.parametrize("n", [3000, 8192, 20000, 40000, 100000, 300000, 1 << 20, 1 << 23])
@pytest.mark.parametrize("kind", [0, 1])
def test_square_through_one_pointer(b2m_gpu, n, kind):
    """a * a with both operands at one device pointer takes the squaring path
    (one forward transform, its spectrum squared in the fused pass) on two-
    and three-pass and 3 * 2^k plans."""
    import torch

    a = gen_operand(n + 11, n, kind)
    d = torch.from_numpy(a.view(np.int32)).cuda()
    out = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    olen = torch.zeros(1, dtype=torch.int64, device="cuda")
    b2m_gpu.mul_device(d.data_ptr(), n, d.data_ptr(), n, out.data_ptr(), 2 * n, olen.data_ptr(), 0)
    b2m_gpu.stream_check(0)
    got = out.cpu().numpy().view(np.uint32)[: int(olen.item())]
    if n <= 100000:
        assert np.array_equal(got, oracle.mul_port(a, a))
    else:
        ia = int.from_bytes(a.tobytes(), "little")
        ip = int.from_bytes(got.tobytes(), "little")
        for q in [(1 << 61) - 1, (1 << 32) + 1, (1 << 32) - 1]:
            assert ip % q == (ia % q) * (ia % q) % q
        assert np.array_equal(got[:32], oracle.mul_port(a[:32], a[:32])[:32])


@pytest.mark.parametrize("n", [1000, 5000, 40000, 300000])
def test_square_through_the_host_call(b2m_gpu, n):
    """The reference-facing host call given one array twice (the reference's
    x * x) copies it once and squares it."""
    a = gen_operand(n + 29, n, 1 if n == 5000 else 0)
    p = b2m_gpu.mul_ntt_cuda(a, a)
    if n <= 40000:
        assert np.array_equal(p, oracle.mul_port(a, a))
    else:
        ia = int.from_bytes(a.tobytes(), "little")
        ip = int.from_bytes(p.tobytes(), "little")
        for q in [(1 << 61) - 1, (1 << 32) + 1, (1 << 32) - 1]:
            assert ip % q == (ia % q) * (ia % q) % q
