"""GPU tests of the continuous-batching server (b2m_server_*): every product
is the same alone and in the mix (bit-exact), admission respects the HBM
budget, oversize requests are refused, caller-owned buffers work, and stop
completes queued work."""
import ctypes

import numpy as np
import pytest

from golden_util import gen_operand

pytestmark = pytest.mark.gpu


def _copy_out(torch, ptr, n):
    """Copy n u32 limbs from a raw device pointer to numpy (device-to-device
    into a torch tensor through the CUDA runtime, then to the host)."""
    if n == 0:
        return np.zeros(0, np.uint32)
    dst = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rt = _cudart(torch)
    assert rt.cudaMemcpy(ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(ptr), 4 * n, 3) == 0  # device to device
    return dst.cpu().numpy().view(np.uint32)


def _cudart(torch):
    import glob
    import os

    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            rt = ctypes.CDLL(name)
            break
        except OSError:
            rt = None
    if rt is None:
        cand = glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_runtime", "lib",
                                      "libcudart.so*"))
        rt = ctypes.CDLL(cand[0])
    rt.cudaMemcpy.restype = ctypes.c_int
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    return rt


SIZES = [(1024, 1024), (1500, 70000), (100000, 3000), (262144, 262144), (5000, 5000), (40000, 2),
         (1, 1), (65536, 65536), (300000, 200000), (2048, 4096), (17, 99999), (131072, 1000)]


def test_products_same_alone_and_in_the_mix(b2m_gpu):
    torch = pytest.importorskip("torch")
    srv = b2m_gpu.Server(hbm_budget_bytes=8 << 30, streams=4, max_batch=8)
    tickets = []
    for i, (na, nb) in enumerate(SIZES * 2):
        kind = 1 if i % 5 == 0 else 0
        tickets.append((srv.submit(na, nb, 1000 + i, 2000 + i, kind), na, nb, 1000 + i, 2000 + i, kind))
    for t, na, nb, sa, sb, kind in tickets:
        r = srv.wait(t, 120.0)
        assert r.state == b2m_gpu.DONE and r.residues_ok == 1, (na, nb, r.state, r.status)
        got = _copy_out(torch, r.out, r.out_len)
        a = gen_operand(sa, na, kind)
        b = gen_operand(sb, nb, kind)
        alone = b2m_gpu.mul_ntt_cuda(a, b)
        assert np.array_equal(got, alone), (na, nb)
        srv.release(t)
    st = srv.stats()
    assert st["completed"] == len(tickets) and st["failed"] == 0 and st["dispatches"] >= 3
    srv.stop()


def test_budget_admission_serialises_large_requests(b2m_gpu):
    # each 2^23 x 2^23 request holds ~0.64 GB (operands and output 128 MB until
    # released, 2^25-point workspace 512 MB until done): one fits in 700 MB
    srv = b2m_gpu.Server(hbm_budget_bytes=700 << 20, streams=4, max_batch=4)
    ts = [srv.submit(1 << 23, 1 << 23, 7 + i, 8 + i) for i in range(4)]
    for t in ts:
        r = srv.wait(t, 120.0)
        assert r.state == b2m_gpu.DONE and r.residues_ok == 1
        srv.release(t)
    st = srv.stats()
    assert st["peak_bytes"] <= 700 << 20 and st["dispatches"] == 4
    with pytest.raises(b2m_gpu.B2MError) as ei:
        srv.submit(1 << 24, 1 << 24, 1, 2)
    assert ei.value.status == b2m_gpu.OUT_OF_MEMORY
    srv.stop()


def test_caller_owned_buffers_and_stop_drains(b2m_gpu):
    torch = pytest.importorskip("torch")
    na, nb = 200000, 150000
    a = gen_operand(5, na)
    b = gen_operand(6, nb)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    dout = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    srv = b2m_gpu.Server(hbm_budget_bytes=4 << 30)
    t = srv.submit(na, nb, a=da.data_ptr(), b=db.data_ptr(), out=dout.data_ptr(), out_cap=na + nb)
    extra = [srv.submit(70000, 70000, 11 + i, 12 + i) for i in range(6)]
    srv.stop()  # completes everything queued
    got = dout.cpu().numpy().view(np.uint32)
    want = b2m_gpu.mul_ntt_cuda(a, b)
    assert np.array_equal(got[: want.size], want)
    del t, extra


def test_continuous_admission_while_dispatches_run(b2m_gpu):
    """Continuous batching, not a queue alone: a second wave submitted while
    the first wave's dispatches are on the GPU is admitted before the first
    wave completes, dispatches run concurrently on the server's streams, and
    every product of both waves is the same as alone."""
    import time

    torch = pytest.importorskip("torch")
    srv = b2m_gpu.Server(hbm_budget_bytes=16 << 30, streams=4, max_batch=2)
    big = 1 << 22  # each product ~1 ms of device time
    wave1 = [(srv.submit(big, big, 300 + i, 400 + i), big, big, 300 + i, 400 + i) for i in range(8)]
    # wait until the first wave is on the GPU (admitted, not yet done)
    t0 = time.time()
    while time.time() - t0 < 30:
        states = [srv.poll(t).state for t, *_ in wave1]
        if any(s >= 1 for s in states):
            break
        time.sleep(0.0002)
    assert any(s >= 1 for s in states), states
    wave2 = [(srv.submit(n, m, 500 + i, 600 + i), n, m, 500 + i, 600 + i)
             for i, (n, m) in enumerate([(1 << 20, 1 << 20), (70000, 3000), (1 << 21, 1 << 19), (4096, 4096)])]
    res1 = [srv.wait(t, 120.0) for t, *_ in wave1]
    res2 = [srv.wait(t, 120.0) for t, *_ in wave2]
    assert all(r.state == b2m_gpu.DONE and r.residues_ok == 1 for r in res1 + res2)
    last_done_1 = max(r.t_done_ns for r in res1)
    # some second-wave request was admitted to the GPU while the first wave ran
    assert min(r.t_admit_ns for r in res2) < last_done_1
    # admitted requests overlapped in time on the device (intervals [admit, done] intersect across dispatches)
    spans = sorted((r.t_admit_ns, r.t_done_ns) for r in res1 + res2)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    st = srv.stats()
    assert st["max_inflight_dispatches"] >= 2 and st["dispatches"] >= 5
    for (t, na, nb, sa, sb), r in zip(wave1 + wave2, res1 + res2):
        got = _copy_out(torch, r.out, r.out_len)
        alone = b2m_gpu.mul_ntt_cuda(gen_operand(sa, na), gen_operand(sb, nb))
        assert np.array_equal(got, alone), (na, nb)
        srv.release(t)
    srv.stop()
