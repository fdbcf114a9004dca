"""GPU tests of batched products (b2m_batch_*): mixed sizes across every
transform plan in one batch, empty and zero operands, NULL out_len, a graph
replayed twice, autotuned plans -- every product bit-exact against the oracle
or against the single-product entry point."""
import numpy as np
import pytest

import oracle
from golden_util import gen_operand

pytestmark = pytest.mark.gpu


def _pack(torch, arrays):
    """Concatenate u32 arrays into one device tensor; return (tensor, offsets)."""
    offs, tot = [], 0
    for a in arrays:
        offs.append(tot)
        tot += max(1, a.size) + 64  # keep every operand 256-byte apart
    host = np.zeros(tot, np.uint32)
    for o, a in zip(offs, arrays):
        host[o:o + a.size] = a
    return torch.from_numpy(host.view(np.int32)).cuda(), offs


def _make(torch, sizes, null_len_every=0):
    ops = []
    for i, (na, nb, kind) in enumerate(sizes):
        ops.append(gen_operand(1000 + 2 * i, na, kind))
        ops.append(gen_operand(1001 + 2 * i, nb, kind))
    dev, offs = _pack(torch, ops)
    out_sizes = [na + nb for na, nb, _ in sizes]
    out = torch.full((sum(out_sizes) + 64 * len(sizes),), -1, dtype=torch.int32, device="cuda")
    lens = torch.full((len(sizes),), -1, dtype=torch.int64, device="cuda")
    jobs, oo = [], 0
    base, obase, lbase = dev.data_ptr(), out.data_ptr(), lens.data_ptr()
    out_offs = []
    for i, (na, nb, _) in enumerate(sizes):
        olen = 0 if (null_len_every and i % null_len_every == 0) else lbase + 8 * i
        jobs.append((base + 4 * offs[2 * i], na, base + 4 * offs[2 * i + 1], nb, obase + 4 * oo, na + nb, olen))
        out_offs.append(oo)
        oo += na + nb + 64
    return ops, out, lens, jobs, out_offs


def _check(ops, out, lens, sizes, out_offs, null_len_every=0):
    host = out.cpu().numpy().view(np.uint32)
    hl = lens.cpu().numpy()
    for i, (na, nb, _) in enumerate(sizes):
        a, b = ops[2 * i], ops[2 * i + 1]
        want = oracle.mul_port(a, b) if na and nb else np.zeros(0, np.uint32)
        if not (null_len_every and i % null_len_every == 0):
            assert hl[i] == want.size, (i, na, nb)
        got = host[out_offs[i]:out_offs[i] + want.size]
        assert np.array_equal(got, want), (i, na, nb)


def _sizes(seed, n, lo=1, hi=40000):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        na, nb = (int(x) for x in np.exp(rng.uniform(np.log(lo), np.log(hi), 2)))
        out.append((na, nb, 1 if i % 17 == 0 else 0))
    out += [(0, 5, 0), (7, 0, 0), (1, 1, 0), (4096, 4096, 1), (20000, 5000, 0)]
    return out


def test_one_shot_batch_mixed_sizes(b2m_gpu):
    torch = pytest.importorskip("torch")
    sizes = _sizes(1, 300)
    ops, out, lens, jobs, oo = _make(torch, sizes, null_len_every=11)
    b2m_gpu.mul_batch(jobs, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    _check(ops, out, lens, sizes, oo, null_len_every=11)


def test_graph_batch_replayed_with_autotune(b2m_gpu):
    torch = pytest.importorskip("torch")
    sizes = _sizes(2, 200, lo=64, hi=70000)
    ops, out, lens, jobs, oo = _make(torch, sizes)
    bt = b2m_gpu.Batch(jobs, b2m_gpu.BATCH_GRAPH | b2m_gpu.BATCH_AUTOTUNE)
    s = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out.fill_(-1)
        lens.fill_(-1)
        bt.launch(s)
        b2m_gpu.stream_check(s)
        _check(ops, out, lens, sizes, oo)
    bt.close()


def test_batch_matches_single_products_on_large_jobs(b2m_gpu):
    torch = pytest.importorskip("torch")
    sizes = [(300000, 250000, 0), (1 << 20, 1 << 17, 0), (100000, 100000, 1)]
    ops, out, lens, jobs, oo = _make(torch, sizes)
    b2m_gpu.mul_batch(jobs, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    host = out.cpu().numpy().view(np.uint32)
    hl = lens.cpu().numpy()
    for i, (na, nb, _) in enumerate(sizes):
        want = b2m_gpu.mul_ntt_cuda(ops[2 * i], ops[2 * i + 1])
        assert hl[i] == want.size and np.array_equal(host[oo[i]:oo[i] + want.size], want)
