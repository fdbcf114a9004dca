"""GPU test of b2m_mul_device_noalloc, the entry point for callers that cannot
allocate device memory when they multiply (their HBM belongs to another
allocator, or cudaMalloc's synchronisation is not acceptable in their loop).

It must give the same products as b2m_mul_device and as the oracle (the
C restatement of the reference's CPU NTT), on two calls in a row (the shared
static scratch keeps the previous call's contents, so the second call checks
that nothing stale leaks through), and reject sizes beyond its fixed limit of
na + nb <= 2^19 limbs. This file is named to be collected last.
"""
import numpy as np
import pytest

import oracle
from golden_util import gen_operand

pytestmark = pytest.mark.gpu


def _product(b2m, torch, fn, a_t, na, b_t, nb):
    out = torch.full((na + nb,), -1, dtype=torch.int32, device="cuda")
    olen = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    fn(a_t.data_ptr(), na, b_t.data_ptr(), nb, out.data_ptr(), na + nb, olen.data_ptr(), s)
    b2m.stream_check(s)
    n = int(olen.item())
    return out.cpu().numpy().view(np.uint32)[:n].copy()


@pytest.mark.parametrize("na,nb,kind", [(131072, 131072, 0), (100000, 31000, 0), (65536, 65536, 1),
                                        (3000, 1234, 0)])
def test_no_alloc_matches_pool_entry_point_twice(b2m_gpu, na, nb, kind):
    torch = pytest.importorskip("torch")
    a = gen_operand(na + 11, na, kind)
    b = gen_operand(nb + 13, nb, kind)
    a_t = torch.from_numpy(a.view(np.int32)).cuda()
    b_t = torch.from_numpy(b.view(np.int32)).cuda()
    want = _product(b2m_gpu, torch, b2m_gpu.mul_device, a_t, na, b_t, nb)
    ref = oracle.mul_port(a, b)
    assert want.size == ref.size and np.array_equal(want, ref)
    for _ in range(2):
        got = _product(b2m_gpu, torch, b2m_gpu.mul_device_noalloc, a_t, na, b_t, nb)
        assert got.size == want.size and np.array_equal(got, want)


def test_no_alloc_rejects_sizes_beyond_its_limit(b2m_gpu):
    torch = pytest.importorskip("torch")
    na = nb = (1 << 18) + 1  # na + nb > 2^19 -> transform length 2^21
    a_t = torch.ones(na, dtype=torch.int32, device="cuda")
    out = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
    with pytest.raises(b2m_gpu.B2MError) as ei:
        b2m_gpu.mul_device_noalloc(a_t.data_ptr(), na, a_t.data_ptr(), nb, out.data_ptr(), na + nb)
    assert ei.value.status == b2m_gpu.TOO_LARGE
