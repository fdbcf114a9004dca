"""One process per GPU: rank plumbing, sharding of independent products and
the cross-rank merge of a Chudnovsky product tree.

Every product is independent of every other, so multi-GPU work needs no
collective on the data path:

* single products run as replicas, one per rank;
* a batch of uneven products is partitioned by estimated cost, longest first
  onto the least-loaded rank (LPT), and each rank launches its share;
* a Chudnovsky tree over [0, n) is split into one contiguous term range per
  rank; each rank builds its subtree on its own GPU and the subtree roots are
  merged pairwise up a binary tree of ranks: log2(world) steps, one
  point-to-point transfer of (P, Q, T) per merge, rank 0 ends with the root.
  P, Q and T/Q of a range do not depend on where it is split
  (src/chudnovsky.cpp:64-102), so the root equals the one-GPU root.

Timings reduce as the maximum over ranks. The reference runs one process on
one GPU (src/ntt_cuda.cu:179-243); nothing here has a counterpart there. The
transport and merge logic is written against a small backend interface so
that it runs on CPU ranks (gloo, Python integers) in the tests and on GPUs
(NCCL, device-resident b2m_pqt nodes) in production.
"""
from __future__ import annotations

import datetime
import heapq
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    rank: int = 0
    world: int = 1
    local: int = 0
    dist: object = None      # torch.distributed once a process group exists
    device: object = None    # device of the tensors that collectives carry


def from_env(backend: str = "nccl", timeout_s: float = 120.0) -> Ranks:
    """RANK / WORLD_SIZE / LOCAL_RANK from the launcher (torchrun); with more
    than one rank, a process group on `backend` (nccl: one GPU per rank,
    gloo: CPU tensors) with a short timeout, so that a rank that never joins
    ends the others with an error instead of a hang."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1:
        return Ranks(rank, world, local, None, None)
    import torch
    import torch.distributed as dist

    to = datetime.timedelta(seconds=timeout_s)
    if backend == "nccl":
        torch.cuda.set_device(local)
        dev = torch.device("cuda", local)
        dist.init_process_group("nccl", timeout=to, device_id=dev)
    else:
        dev = torch.device("cpu")
        dist.init_process_group(backend, timeout=to)
    return Ranks(rank, world, local, dist, dev)


def close(r: Ranks) -> None:
    if r.dist is not None and r.dist.is_initialized():
        r.dist.destroy_process_group()


def barrier(r: Ranks) -> None:
    if r.dist is not None:
        r.dist.barrier()


def max_over_ranks(r: Ranks, *xs: float):
    """Element-wise maximum of the given floats over all ranks (every rank
    gets the result). One value in, one value out."""
    if r.dist is None:
        return xs[0] if len(xs) == 1 else list(xs)
    import torch

    t = torch.tensor(list(xs), dtype=torch.float64, device=r.device)
    r.dist.all_reduce(t, op=r.dist.ReduceOp.MAX)
    out = [float(v) for v in t.tolist()]
    return out[0] if len(out) == 1 else out


# ---- sharding of independent products ------------------------------------------------
def ntt_length(na: int, nb: int) -> int:
    """Transform length of a na x nb-limb product: the next power of two at
    or above 2(na + nb) 16-bit digits (include/ntt.h:37-50)."""
    n = 1
    while n < 2 * (na + nb):
        n <<= 1
    return n


def product_cost(na: int, nb: int) -> float:
    """Work estimate of one product: N log2 N of its transform length."""
    n = ntt_length(na, nb)
    return float(n * max(1, n.bit_length() - 1))


def lpt_shard(costs, world: int):
    """Indices of the jobs each rank runs: jobs by decreasing cost, each to
    the rank with the least work so far (ties to the lower rank, equal costs
    in index order), each rank's list in index order. Deterministic, so every
    rank computes the same partition without talking to the others."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


# ---- Chudnovsky tree across ranks ----------------------------------------------------
def term_ranges(n_terms: int, world: int):
    """One contiguous, non-empty term range per rank covering [0, n_terms),
    in rank order, sizes differing by at most one (earlier ranks larger)."""
    if n_terms < world:
        raise ValueError(f"{n_terms} terms cannot be split over {world} ranks")
    q, rem = divmod(n_terms, world)
    out, a = [], 0
    for r in range(world):
        b = a + q + (1 if r < rem else 0)
        out.append((a, b))
        a = b
    return out


def merge_schedule(world: int):
    """Steps of the pairwise reduction: step s merges rank r + 2^s into rank
    r for every r that is a multiple of 2^(s+1) (right range into left)."""
    steps, stride = [], 1
    while stride < world:
        steps.append([(r, r + stride) for r in range(0, world, 2 * stride) if r + stride < world])
        stride *= 2
    return steps


def reduce_tree(r: Ranks, node, backend):
    """Merges the ranks' subtree roots (rank i holds range i of term_ranges)
    into rank 0, following merge_schedule. Returns the root on rank 0, None
    on the others (each stops after sending its node)."""
    for step in merge_schedule(r.world):
        for dst, src in step:
            if r.rank == dst:
                node = backend.merge(node, backend.recv(r, src))
            elif r.rank == src:
                backend.send(r, node, dst)
                return None
    return node if r.rank == 0 else None


def chudnovsky_bs_ranks(r: Ranks, n_terms: int, backend):
    """(P, Q, T) of [0, n_terms) over all ranks; the root on rank 0."""
    a, b = term_ranges(n_terms, r.world)[r.rank]
    return reduce_tree(r, backend.bs(a, b), backend)


def _send_header(r: Ranks, dst: int, lengths, sign: int) -> None:
    import torch

    r.dist.send(torch.tensor(list(lengths) + [sign], dtype=torch.int64, device=r.device), dst)


def _recv_header(r: Ranks, src: int):
    import torch

    h = torch.empty(4, dtype=torch.int64, device=r.device)
    r.dist.recv(h, src)
    v = [int(x) for x in h.tolist()]
    return v[:3], v[3]


class _DeviceLimbs:
    """A device range of u32 limbs seen by torch (int32, no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}


class DeviceBackend:
    """Subtrees built on this rank's GPU (b2m_chudnovsky_bs); nodes cross
    ranks as three int32 device tensors over NCCL and are copied into a new
    device node on arrival (b2m_pqt_import); merges run on the receiving GPU
    (b2m_pqt_merge)."""

    def __init__(self, b200mul):
        self.m = b200mul

    def bs(self, a: int, b: int):
        return self.m.chudnovsky_bs(a, b)

    def merge(self, left, right):
        node = self.m.pqt_merge(left, right)
        left.free()
        right.free()
        return node

    def send(self, r: Ranks, node, dst: int) -> None:
        import torch

        _send_header(r, dst, node.lengths, node.t_sign)
        for f in range(3):
            n = node.lengths[f]
            if n:
                ptr = self.m.lib.b2m_pqt_device(node.handle, f)
                r.dist.send(torch.as_tensor(_DeviceLimbs(ptr, n), device=r.device), dst)
        torch.cuda.synchronize(r.device)
        node.free()

    def recv(self, r: Ranks, src: int):
        import torch

        lengths, sign = _recv_header(r, src)
        bufs = [torch.empty(max(1, n), dtype=torch.int32, device=r.device) for n in lengths]
        for f in range(3):
            if lengths[f]:
                r.dist.recv(bufs[f], src)
        torch.cuda.synchronize(r.device)
        return self.m.pqt_import([t.data_ptr() for t in bufs], lengths, sign)
