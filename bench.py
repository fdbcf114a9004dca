#!/usr/bin/env python
"""Benchmark of the B200 Goldilocks-NTT big-integer multiply.

Headline metric: ms per 2^24 x 2^24-limb multiply (seeded uniform random u32
limbs), device-resident operands, bit-exact product. One "step" is one full
product (repack, 3 transforms, pointwise, carry, trimmed length) per GPU.

    python bench.py [--gpus N --steps K --warmup W]
    python -m torch.distributed.run --nnodes=1 --nproc-per-node N --master-addr 127.0.0.1 \\
        --master-port P bench.py --gpus N --steps K --warmup W
    python bench.py --impl reference ...   # the reference's own CPU NTT, all host threads

Products are independent, so N GPUs run N products per step with no
collective on the data path (weak scaling); the step time is the maximum over
ranks of CUDA-event times, and `value` is that time divided by the products
all ranks completed. The JSON line also carries the end-to-end figure through
the host-buffer C-ABI call (pinned host memory, copies in the timed region),
the roofline of the dominant kernel (CUDA events around each launch), the
reference's CPU NTT timed on this host, and SM clocks sampled during timing.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cuda-pi-chudnovsky-bbp_b200")
sys.path.insert(0, PKG)

METRIC = "ms per 2^24-limb multiply"
NA = NB = 1 << 24
SEED_A, SEED_B = 24001, 24002


def algorithmic_bytes(na: int, nb: int, n: int) -> int:
    """Minimum HBM traffic of one product: u32 operands in and product out
    (8(na+nb)) plus eight N-element u64 sweeps (64N) of a two-pass schedule."""
    return 8 * (na + nb) + 64 * n


def kernel_bytes(kind: str, na: int, nb: int, n: int, operand: int) -> int:
    """Algorithmic bytes of one launch of each kernel kind (N = transform length)."""
    if kind == "fwd_first":
        return 4 * operand + 8 * n
    if kind in ("fwd_mid", "fwd_last", "inv_mid"):
        return 16 * n
    if kind == "fused_last":
        return 24 * n
    if kind == "carry":
        return 8 * n + 4 * (na + nb)
    return 8 * (na + nb)  # mul_small


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json: copy bandwidth)"
    return 6650.0, "fallback (6.65 TB/s, earlier pool measurement)"


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------- CPU
def _ref_or_port():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the checker: only the CPU-baseline leg and the reference arm use it

    if oracle.ref_available():
        return oracle, "reference", lambda a, b: oracle.mul_ref(a, b, "ntt-cpu")
    return oracle, "port", lambda a, b: oracle.mul_port(a, b)


def nlogn_scale(n_from: int, n_to: int) -> float:
    """Scale a product time from na = nb = n_from to n_to limbs by N log2 N."""
    nf, nt = 4 * n_from, 4 * n_to  # transform lengths
    return (nt * math.log2(nt)) / (nf * math.log2(nf))


def cpu_product_s(oracle_mod, fn, na: int, nb: int, seed_a: int = SEED_A, seed_b: int = SEED_B) -> float:
    """Wall time of one CPU product of the seeded operands (the same splitmix64
    operands the GPU arm multiplies, made by the oracle's C generator so that
    the product library is never loaded here)."""
    a = oracle_mod.gen_operand(seed_a, na)
    b = oracle_mod.gen_operand(seed_b, nb)
    t0 = time.perf_counter()
    p = fn(a, b)
    dt = time.perf_counter() - t0
    if p.size not in (na + nb, na + nb - 1):
        raise RuntimeError("CPU product has the wrong length")
    return dt


def cpu_baseline(sample_log: int = 24) -> dict:
    """The reference's CPU NTT (single-threaded, as the reference is) on one
    product; at the default sample_log = 24 that is the headline 2^24 x 2^24
    product itself (about a minute), measured, not scaled."""
    oracle_mod, kind, fn = _ref_or_port()
    n = 1 << sample_log
    dt = cpu_product_s(oracle_mod, fn, n, n)
    scale = nlogn_scale(n, NA)
    sample = (f"one {n}x{n}-limb product (mul_ntt_cpu, src/ntt_cpu.cpp:111-129, 1 thread) in {dt:.2f} s"
              + ("" if n == NA else f", scaled to 2^24 limbs by N log2 N (x{scale:.2f})"))
    return {"value": round(dt * 1e3 * scale, 1), "unit": "ms", "cores": 1, "kind": kind, "sample": sample,
            "measured_full_size": n == NA}


def run_reference(args) -> None:
    """The reference's own CPU implementation of the path (mul_ntt_cpu,
    src/ntt_cpu.cpp:111-129, compiled from the reference's sources into
    oracle/_ref) on this host. The reference multiplies on one thread and has
    no parallel path, so one product uses one core. `value` is one measured
    2^24 x 2^24 product, the headline workload itself. The K timed steps are
    bounded samples of the same routine (2^20 x 2^20 limbs each, about 3 s),
    so that the whole run stays within a few minutes; their N log2 N scaling
    to 2^24 limbs is reported beside the measured value, not as it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    oracle_mod, kind, fn = _ref_or_port()
    full_s = cpu_product_s(oracle_mod, fn, NA, NB)
    sl = 1 << 20
    for i in range(args.warmup):
        cpu_product_s(oracle_mod, fn, 1 << 16, 1 << 16, SEED_A + i, SEED_B + i)
    times = [cpu_product_s(oracle_mod, fn, sl, sl, SEED_A + i, SEED_B + i) for i in range(args.steps)]
    step = statistics.mean(times)
    value = full_s * 1e3
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step * 1e3, 2),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (GF(p), p=2^64-2^32+1)",
        "data": "synthetic: seeded uniform random u32 limbs (splitmix64, the GPU arm's operands)",
        "config": {"workload": "2^24 x 2^24-limb product, uniform random limbs", "na": NA, "nb": NB,
                   "threads": 1, "host_threads_available": os.cpu_count()},
        "full_size_product_ms": round(value, 1),
        "steps_sample": {"limbs": sl, "mean_ms": round(step * 1e3, 1),
                         "scaled_to_2^24_ms": round(step * 1e3 * nlogn_scale(sl, NA), 1),
                         "note": "each timed step is one 2^20 x 2^20-limb product of the same routine; "
                                 "the headline value above is the measured full-size product"},
        "cpu_baseline": {"value": round(value, 1), "unit": "ms", "cores": 1, "kind": kind,
                         "sample": f"one 2^24 x 2^24-limb product of the reference's mul_ntt_cpu "
                                   f"(src/ntt_cpu.cpp:111-129), measured in {full_s:.1f} s on one thread "
                                   f"(the reference has no multi-threaded product)"},
        "e2e": {"value": round(value, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------- ours
def run_ours(args) -> None:
    import numpy as np
    import torch

    import b200mul
    import ranks

    # Replicas: every rank multiplies its own pair (no data-path collective);
    # the step time is the maximum over ranks.
    rk = ranks.from_env("nccl", timeout_s=120)
    rank, world, local = rk.rank, rk.world, rk.local
    torch.cuda.set_device(local)
    b200mul.init(local)
    na, nb = args.na, args.nb

    def barrier():
        ranks.barrier(rk)

    def max_over_ranks(x: float) -> float:
        return ranks.max_over_ranks(rk, x)

    a_h = b200mul.gen_operand(SEED_A + 1000 * rank, na)
    b_h = b200mul.gen_operand(SEED_B + 1000 * rank, nb)
    a = torch.from_numpy(a_h.view(np.int32)).cuda()
    b = torch.from_numpy(b_h.view(np.int32)).cuda()
    out = torch.empty(na + nb, dtype=torch.int32, device="cuda")
    olen = torch.zeros(1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    # Plan choice (pass split, tile size) timed once before any measurement;
    # every later product of this transform length uses the fastest.
    tune = b200mul.autotune(na, nb, sp) if args.autotune and not args.no_autotune else []
    plan = b200mul.plan_describe(na, nb)
    n = plan["points"]

    def product():
        b200mul.mul_device(a.data_ptr(), na, b.data_ptr(), nb, out.data_ptr(), na + nb, olen.data_ptr(), sp)

    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            product()
    b200mul.stream_check(sp)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        product()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    b200mul.stream_check(sp)
    step_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)

    # Per-kernel device times (CUDA events around each launch on `stream`).
    traces = [b200mul.mul_device_traced(a.data_ptr(), na, b.data_ptr(), nb, out.data_ptr(), na + nb,
                                        olen.data_ptr(), sp) for _ in range(args.trace_steps)]
    per_kind: dict[str, list[float]] = {}
    per_launch_bytes: dict[str, int] = {}
    first_seen = 0
    for tr in traces:
        first_seen = 0
        for kind, logr, ms in tr:
            key = f"{kind}<{logr}>" if kind not in ("carry",) else kind
            operand = na if (kind == "fwd_first" and first_seen == 0) else nb
            if kind == "fwd_first":
                first_seen += 1
            per_kind.setdefault(key, []).append(ms)
            per_launch_bytes[key] = kernel_bytes(kind, na, nb, n, operand)
    kinds = {k: {"launches_per_product": len(v) // len(traces), "avg_ms": statistics.mean(v),
                 "share": sum(v) / sum(sum(x) for x in per_kind.values())} for k, v in per_kind.items()}
    dominant = max(kinds, key=lambda k: kinds[k]["avg_ms"] * kinds[k]["launches_per_product"])
    peak, peak_src = load_peaks()
    dom_ms = kinds[dominant]["avg_ms"]
    dom_bytes = per_launch_bytes[dominant]
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    prod_bytes = algorithmic_bytes(na, nb, n)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(dominant)

    # End to end through the public host-buffer call: pinned host operands,
    # H2D + product + D2H of the result inside the timed region.
    pa = torch.empty(na, dtype=torch.int32, pin_memory=True)
    pb = torch.empty(nb, dtype=torch.int32, pin_memory=True)
    po = torch.empty(na + nb, dtype=torch.int32, pin_memory=True)
    pa.numpy()[:] = a_h.view(np.int32)
    pb.numpy()[:] = b_h.view(np.int32)
    ha, hb, ho = pa.numpy().view(np.uint32), pb.numpy().view(np.uint32), po.numpy().view(np.uint32)
    for _ in range(2):
        res = b200mul.mul_ntt_cuda(ha, hb, out=ho)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        res = b200mul.mul_ntt_cuda(ha, hb, out=ho)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.e2e_steps
    barrier()
    e2e_ms = max_over_ranks(e2e_ms)
    dev = out.cpu().numpy().view(np.uint32)[: int(olen.item())]
    if not np.array_equal(dev, res):
        raise RuntimeError("device-resident and host-buffer products differ")

    # The other two workloads the metric names, on the same GPUs: the batch of
    # 4096 uneven products against one call per product, and the serving loop
    # at the configured Poisson rate (every rank takes the same steps).
    batch = serve = None
    if not args.no_extra:
        b = measure_batch(rk, args)
        batch = {"workload": b["config"]["workload"], "jobs_per_gpu": b["config"]["jobs_rank0"],
                 "glimbs_per_s": b["value"], "ms": b["ms_per_step"],
                 "one_at_a_time_glimbs_per_s": b["one_at_a_time"]["value"],
                 "one_at_a_time_ms": b["one_at_a_time"]["ms"],
                 "speedup_vs_one_at_a_time": b["speedup_vs_one_at_a_time"],
                 "bit_exact_vs_one_at_a_time": b["bit_exact_vs_one_at_a_time"]}
        def summary(v):
            return {"workload": v["config"]["workload"], "requests": v["config"]["requests"],
                    "p50_ms": v["value"], "p99_ms": v["p99_ms"], "mean_ms": v["mean_ms"],
                    "served_glimbs_per_s": v["throughput"]["glimbs_per_s"],
                    "offered_glimbs_per_s": v["throughput"]["offered_glimbs_per_s"],
                    "max_queue": v["server"]["max_queue"],
                    "max_inflight_dispatches": v["server"].get("max_inflight_dispatches"),
                    "all_products_residue_checked_ok": v["all_products_residue_checked_ok"]}

        at_cfg = summary(measure_serve(rk, args))
        serve = {"at_config_rate": at_cfg,
                 # the same size mix submitted all at once: what the server
                 # and device can complete, against the configured offer
                 "closed_loop_capacity": serve_capacity(rk, args)}
        # A sustainable rate: when the configured rate overloads the server
        # (its queue grows), 75% of the rate it actually served; otherwise the
        # configured rate itself is sustainable and is not repeated.
        ratio = at_cfg["served_glimbs_per_s"] / max(at_cfg["offered_glimbs_per_s"], 1e-9)
        if ratio < 0.97:
            sus_rate = round(0.75 * ratio * args.rate, 1)
            serve["at_sustainable_rate"] = summary(measure_serve(rk, args, rate=sus_rate))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_sample_log)

    if rank == 0:
        value = step_ms / world
        headline = na == NA and nb == NB
        metric = METRIC if headline else f"ms per {na} x {nb}-limb multiply"
        workload = ("2^24 x 2^24-limb product, uniform random limbs" if headline
                    else f"{na} x {nb}-limb product, uniform random limbs")
        wset = 4 * (na + nb) * 2 + 16 * n
        line = {
            "metric": metric, "value": round(value, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(step_ms, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 (GF(p), p=2^64-2^32+1)",
            "data": "synthetic: seeded uniform random u32 limbs (splitmix64), top limb non-zero",
            "config": {"workload": workload, "na": na, "nb": nb,
                       "ntt_length": n, "plan": plan, "products_per_step": world,
                       "autotune": (autotune_summary(tune) if tune else None),
                       "glimbs_per_s": round((na + nb) * world / (step_ms * 1e-3) / 1e9, 3),
                       "l2": f"working set {wset / 2**20:.0f} MiB per product "
                             + ("> 126 MB L2: no flush needed" if wset > 126 * 2**20
                                else "fits in the 126 MB L2: warm-cache figure")},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                         "algorithmic_bytes_per_launch": dom_bytes, "avg_launch_ms": round(dom_ms, 4),
                         "peak_source": peak_src,
                         # what the ncu captures show holds the transform kernels
                         "binding_unit": "integer ALU pipe, 79-83% of its peak in every transform kernel "
                                         "(ncu; profiles/kernels_2e23_instructions_traffic.md)",
                         "product": {"algorithmic_bytes": prod_bytes,
                                     "achieved_gbs": round(prod_bytes / (step_ms * 1e-3) / 1e9, 1),
                                     "frac": round(prod_bytes / (step_ms * 1e-3) / 1e9 / peak, 4)},
                         "kernels": {k: {"avg_ms": round(v["avg_ms"], 4), "share": round(v["share"], 4),
                                         "launches_per_product": v["launches_per_product"]}
                                     for k, v in kinds.items()}},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": 4 * (na + nb) * world,
                    "d2h_bytes_per_step": (4 * (na + nb) + 8) * world,
                    "path": "b2m_mul_host (C ABI), pinned host buffers, wall clock per call"},
            "gpu_launches": plan["launches"] * args.steps,
            "clocks": clocks,
            "batch": batch,
            "serve": serve,
        }
        print(json.dumps(line), flush=True)
    ranks.close(rk)


def autotune_summary(tune: list) -> dict:
    """Best and worst candidate, and the best of each pass count."""
    def best(c):
        t = min(c, key=lambda t: t["ms"])
        return {"logr": t["logr"], "logc": t["logc"], "ms": t["ms"]}
    out = {"candidates": len(tune), "best_ms": min(t["ms"] for t in tune), "worst_ms": max(t["ms"] for t in tune)}
    for k in (2, 3):
        c = [t for t in tune if len(t["logr"]) == k]
        if c:
            out[f"best_{k}_pass"] = best(c)
    return out


def batch_sizes(n: int, seed: int):
    """n pairs, na and nb independently log-uniform over [64, 65536] limbs:
    floor(2^(6 + 10u)) with u uniform in [0, 1)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    u = rng.random((n, 2))
    return [(int(2 ** (6 + 10 * x)), int(2 ** (6 + 10 * y))) for x, y in u]


def run_batch(args) -> None:
    """Batched uneven products: 4096 log-uniform pairs in one graph launch
    versus one b2m_mul_device call per product on the same GPU."""
    import torch

    import b200mul
    import ranks

    rk = ranks.from_env("nccl", timeout_s=300)
    torch.cuda.set_device(rk.local)
    b200mul.init(rk.local)
    line = measure_batch(rk, args)
    if rk.rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close(rk)


def measure_batch(rk, args) -> dict:
    """The batch workload's JSON object (rank 0's is complete; the step times
    are maxima over ranks)."""
    import numpy as np
    import torch

    import b200mul
    import ranks

    rank, world, local = rk.rank, rk.world, rk.local
    if args.batch_split and world > 1:
        # one batch of 4096 pairs, partitioned over the ranks by cost (LPT)
        everything = batch_sizes(args.batch_jobs, 4096)
        part = ranks.lpt_shard([ranks.product_cost(a, b) for a, b in everything], world)[rank]
        sizes = [everything[i] for i in part]
        job_limbs = sum(a + b for a, b in everything)
    else:
        # weak scaling: every rank its own 4096 pairs
        sizes = batch_sizes(args.batch_jobs, 4096 + rank)
        job_limbs = sum(a + b for a, b in sizes) * world
    total_limbs = sum(a + b for a, b in sizes)
    # Operands packed into one device tensor, outputs into two (batched, single).
    offs, tot = [], 0
    for na, nb in sizes:
        offs.append((tot, tot + na + 64))
        tot += na + nb + 128
    host = np.zeros(tot, np.uint32)
    for i, ((na, nb), (oa, ob)) in enumerate(zip(sizes, offs)):
        host[oa:oa + na] = b200mul.gen_operand(7 * i + 1, na)
        host[ob:ob + nb] = b200mul.gen_operand(7 * i + 2, nb)
    dev = torch.from_numpy(host.view(np.int32)).cuda()
    out1 = torch.zeros(tot, dtype=torch.int32, device="cuda")
    out2 = torch.zeros(tot, dtype=torch.int32, device="cuda")
    len1 = torch.zeros(len(sizes), dtype=torch.int64, device="cuda")
    len2 = torch.zeros(len(sizes), dtype=torch.int64, device="cuda")
    base = dev.data_ptr()
    jobs = [(base + 4 * oa, na, base + 4 * ob, nb, out1.data_ptr() + 4 * oa, na + nb, len1.data_ptr() + 8 * i)
            for i, ((na, nb), (oa, ob)) in enumerate(zip(sizes, offs))]
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    t0 = time.perf_counter()
    bt = b200mul.Batch(jobs, b200mul.BATCH_GRAPH | b200mul.BATCH_AUTOTUNE)
    plan_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        bt.launch(sp)
    b200mul.stream_check(sp)

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    batched_ms = timed(lambda: bt.launch(sp), args.steps)
    clocks = sampler.stop()

    def one_at_a_time():
        for i, ((na, nb), (oa, ob)) in enumerate(zip(sizes, offs)):
            b200mul.mul_device(base + 4 * oa, na, base + 4 * ob, nb, out2.data_ptr() + 4 * oa, na + nb,
                               len2.data_ptr() + 8 * i, sp)

    one_at_a_time()
    single_ms = timed(one_at_a_time, max(1, min(3, args.steps)))
    b200mul.stream_check(sp)
    same = bool(torch.equal(out1, out2) and torch.equal(len1, len2))
    bt.close()
    if not same:
        raise RuntimeError("batched and one-at-a-time products differ")
    if world > 1:
        batched_ms, single_ms = ranks.max_over_ranks(rk, batched_ms, single_ms)
    gl_b = job_limbs / (batched_ms * 1e-3) / 1e9
    gl_s = job_limbs / (single_ms * 1e-3) / 1e9
    return {
        "metric": "batched Glimbs/s (4096 log-uniform pairs, 64..65536 limbs)", "value": round(gl_b, 3),
        "unit": "Glimbs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(batched_ms, 4), "higher_is_better": True,
        "scaling": "strong" if (args.batch_split and world > 1) else "weak",
        "vs_baseline": None, "dtype": "u64 (GF(p), p=2^64-2^32+1)",
        "data": "synthetic: seeded uniform random u32 limbs; lengths floor(2^(6+10u)), u uniform",
        "config": {"workload": "4096 independent products, na and nb log-uniform in [64, 65536] limbs",
                   "parallelism": ("one batch partitioned over the ranks by cost (LPT)"
                                   if (args.batch_split and world > 1) else "one batch per rank"),
                   "jobs_rank0": len(sizes), "input_limbs_all_ranks": job_limbs,
                   "batch": "one CUDA-graph launch per step, size-bucketed, autotuned plans",
                   "plan_and_autotune_s": round(plan_s, 2)},
        "one_at_a_time": {"value": round(gl_s, 3), "unit": "Glimbs/s", "ms": round(single_ms, 3),
                          "path": "one b2m_mul_device call per product on the same stream"},
        "speedup_vs_one_at_a_time": round(single_ms / batched_ms, 2),
        "bit_exact_vs_one_at_a_time": same,
        "clocks": clocks}


def run_chudnovsky(args) -> None:
    """Chudnovsky binary splitting for `--digits` digits (default 10^7): the
    whole (P, Q, T) tree on the device, root checked against the reference."""
    import hashlib

    import numpy as np
    import torch

    import b200mul
    import ranks

    # One GPU: the whole tree. Several: one subtree per rank, roots merged
    # pairwise into rank 0 (ranks.chudnovsky_bs_ranks) -- the same tree split
    # over the GPUs, so the total work is fixed (strong scaling).
    rk = ranks.from_env("nccl", timeout_s=300)
    local, rank = rk.local, rk.rank
    torch.cuda.set_device(local)
    b200mul.init(local)
    terms = b200mul.chudnovsky_terms_for_digits(args.digits + 16)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    backend = ranks.DeviceBackend(b200mul)

    def tree():
        if rk.world == 1:
            return b200mul.chudnovsky_bs(0, terms, sp)
        return ranks.chudnovsky_bs_ranks(rk, terms, backend)

    for _ in range(args.warmup):
        t = tree()
        if t is not None:
            t.free()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    walls = []
    ranks.barrier(rk)
    torch.cuda.synchronize()
    e0.record(stream)
    r = None
    for _ in range(args.steps):
        ranks.barrier(rk)
        t0 = time.perf_counter()
        r = tree()
        torch.cuda.synchronize()
        walls.append(ranks.max_over_ranks(rk, time.perf_counter() - t0))
        if _ < args.steps - 1 and r is not None:
            r.free()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    dev_ms = e0.elapsed_time(e1) / args.steps if rk.world == 1 else statistics.median(walls) * 1e3
    if rank != 0:
        ranks.close(rk)
        return
    # end to end: tree + copy of the root's P, Q, T to host memory
    t0 = time.perf_counter()
    hq = [r.limbs(w) for w in range(3)]
    copy_s = time.perf_counter() - t0
    def sha(x):
        return hashlib.sha256(np.ascontiguousarray(x, dtype="<u4").tobytes()).hexdigest()
    fixture = os.path.join(ROOT, "tests", "golden", "chudnovsky.json")
    exact, ref_s = None, None
    if os.path.exists(fixture):
        trees = {t["terms"]: t for t in json.load(open(fixture))["trees"]}
        if terms in trees:
            tr = trees[terms]
            exact = all(sha(hq[w]) == tr[nm]["sha256"] for w, nm in enumerate("PQT")) and r.t_sign == tr["T"]["sign"]
            ref_s = tr["ref_s"]
    levels, products, lengths = r.levels, r.products, r.lengths
    r.free()
    cpu = None
    if rank == 0 and rk.world == 1 and not args.no_cpu_baseline:
        oracle_mod, kind, _ = _ref_or_port()
        sample_digits = 1000000
        st = b200mul.chudnovsky_terms_for_digits(sample_digits + 16)
        t0 = time.perf_counter()
        if kind == "reference":
            oracle_mod.bs_ref(0, st, "ntt-cpu")
        else:
            oracle_mod.bs_port(0, st)
        dt = time.perf_counter() - t0
        cpu = {"value": round(dt * 1e3, 1), "unit": "ms", "cores": 1, "kind": kind,
               "sample": f"the reference's chudnovsky_bs(0, {st}) (1,000,000 digits, NttCpu backend, 1 thread) "
                         f"timed on this host: {dt:.2f} s; its 10,000,000-digit tree took {ref_s} s on the "
                         "build container's host (tests/golden/chudnovsky.json)"}
    if rank == 0:
        print(json.dumps({
            "metric": f"ms per Chudnovsky binary-splitting tree ({args.digits} digits)",
            "value": round(statistics.median(walls) * 1e3, 2), "unit": "ms", "n_gpus": rk.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dev_ms, 2),
            "higher_is_better": False, "scaling": "strong" if rk.world > 1 else "weak",
            "vs_baseline": None, "dtype": "u32 limbs / u64 GF(p)",
            "data": "deterministic: the Chudnovsky series terms",
            "config": {"workload": f"chudnovsky_bs(0, {terms}) for {args.digits} digits, level-wise on device",
                       "parallelism": (f"{rk.world} subtrees (one per rank), roots merged pairwise into rank 0"
                                       if rk.world > 1 else "one GPU"),
                       "terms": terms, "levels": levels, "products": products,
                       "root_limbs": {"P": lengths[0], "Q": lengths[1], "T": lengths[2]}},
            "bit_exact_vs_reference_root": exact,
            "reference_cpu_tree_s": ref_s,
            "e2e": {"value": round((statistics.median(walls) + copy_s) * 1e3, 2), "unit": "ms",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 4 * sum(lengths),
                    "path": "b2m_chudnovsky_bs + copy of the root to host"},
            "cpu_baseline": cpu, "clocks": clocks}), flush=True)
    ranks.close(rk)


def run_pi(args) -> None:
    """The digit string of pi for `--digits` digits (default 10^7), every step
    on one device (b2m_compute_pi): tree, square root, division, decimal
    conversion. The leading 1,000,000 digits are checked against the
    reference's own 1,000,000-digit run (tests/golden/pi_digits.json)."""
    import hashlib

    import torch

    import b200mul

    if int(os.environ.get("RANK", "0")) != 0:
        return  # one product chain, one GPU: other ranks have nothing to do
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    b200mul.init(local)
    for _ in range(args.warmup):  # full size: pools, twiddle tables and plans exist before timing
        b200mul.compute_pi(args.digits)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    runs = []
    for _ in range(args.steps):
        t = {}
        s = b200mul.compute_pi(args.digits, t)
        runs.append(t)
    clocks = sampler.stop()
    med = sorted(runs, key=lambda t: t["total_ms"])[len(runs) // 2]
    checked = None
    fixture = os.path.join(ROOT, "tests", "golden", "pi_digits.json")
    if os.path.exists(fixture):
        ref = {r["digits"]: r for r in json.load(open(fixture))["runs"]}
        d = max([k for k in ref if k <= args.digits], default=None)
        if d:
            checked = {"digits": d, "match": hashlib.sha256(s[: 2 + d].encode()).hexdigest() == ref[d]["sha256"],
                       "reference_compute_pi_s": ref[d]["ref_s"]}
    cpu = None
    if not args.no_cpu_baseline:
        oracle_mod, kind, _ = _ref_or_port()
        sample = 100000
        t0 = time.perf_counter()
        if kind == "reference":
            oracle_mod.compute_pi_ref(sample)
        dt = time.perf_counter() - t0
        cpu = {"value": round(dt * 1e3, 1), "unit": "ms", "cores": 1, "kind": kind,
               "sample": f"the reference's compute_pi_chudnovsky({sample}) (NttCpu products, schoolbook "
                         "division and square root, 1 thread) on this host"} if kind == "reference" else None
    print(json.dumps({
        "metric": f"ms per {args.digits}-digit pi string (compute_pi_chudnovsky on the device)",
        "value": round(med["total_ms"], 1), "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(med["total_ms"], 1), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 limbs / u64 GF(p)", "data": "deterministic: the Chudnovsky series",
        "config": {"workload": f"compute_pi({args.digits}): tree, isqrt, division, decimal on device",
                   "terms": med["terms"]},
        "split_ms": {k: round(med[k], 1) for k in ("tree_ms", "sqrt_ms", "div_ms", "decimal_ms")},
        "prefix_vs_reference": checked, "cpu_baseline": cpu,
        "e2e": {"value": round(med["total_ms"], 1), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": args.digits + 2, "path": "b2m_compute_pi (C ABI), string in host memory"},
        "clocks": clocks}), flush=True)


def run_serve(args) -> None:
    """Serving: Poisson arrivals at --rate req/s for --duration s, operand
    lengths log-uniform in [2^10, 2^24] limbs, seeded operands generated on
    the device, continuous batching under an HBM budget; p50/p99 latency and
    throughput, every product residue-checked on the device."""
    import torch

    import b200mul
    import ranks

    # Several GPUs: one server per rank, each with its own arrival stream at
    # --rate (weak scaling); latencies and throughput gathered to rank 0.
    rk = ranks.from_env("nccl", timeout_s=600)
    torch.cuda.set_device(rk.local)
    b200mul.init(rk.local)
    line = measure_serve(rk, args)
    ranks.close(rk)
    if rk.rank == 0:
        print(json.dumps(line), flush=True)


def serve_capacity(rk, args, n_req: int = 600) -> dict:
    """Closed-loop capacity of the server on the serving size mix: n_req
    requests (lengths log-uniform in [2^10, 2^24] limbs) submitted at once,
    time to complete them all (max over ranks)."""
    import numpy as np

    import b200mul
    import ranks

    rng = np.random.default_rng(3000 + rk.rank)
    lens = (2.0 ** rng.uniform(10, 24, (n_req, 2))).astype(np.int64)
    srv = b200mul.Server(hbm_budget_bytes=args.serve_budget_gb << 30, streams=args.serve_streams,
                         max_batch=args.serve_batch)
    warm = [srv.submit(1 << k, 1 << k, 99 + k, 199 + k) for k in range(10, 25)]
    for t in warm:
        srv.wait(t, 120.0)
        srv.release(t)
    t0 = time.perf_counter()
    ts = [srv.submit(int(a), int(b), 11 * i + 3, 11 * i + 4) for i, (a, b) in enumerate(lens)]
    bad = 0
    for t in ts:
        r = srv.wait(t, 300.0)
        bad += int(r.state != b200mul.DONE or r.residues_ok != 1)
        srv.release(t)
    wall = time.perf_counter() - t0
    srv.stop()
    wall = ranks.max_over_ranks(rk, wall)
    limbs = int(lens.sum()) * rk.world
    return {"requests": n_req * rk.world, "wall_s": round(wall, 3),
            "glimbs_per_s": round(limbs / wall / 1e9, 3), "req_per_s": round(n_req * rk.world / wall, 1),
            "mean_limbs_per_request": int(lens.sum()) // n_req, "all_ok": bad == 0}


def measure_serve(rk, args, rate: float | None = None) -> dict:
    """The serving workload's JSON object at `rate` req/s (default --rate)."""
    import numpy as np

    import b200mul

    rank, local = rk.rank, rk.local
    rate = args.rate if rate is None else rate
    rng = np.random.default_rng(2000 + rank)
    n_req = int(rate * args.duration)
    gaps = rng.exponential(1.0 / rate, n_req)
    arrivals = np.cumsum(gaps)
    lens = (2.0 ** rng.uniform(10, 24, (n_req, 2))).astype(np.int64)
    srv = b200mul.Server(hbm_budget_bytes=args.serve_budget_gb << 30, streams=args.serve_streams,
                         max_batch=args.serve_batch)
    # warm-up: a few requests of every octave so pools and kernels are ready
    warm = [srv.submit(1 << k, 1 << k, 99 + k, 199 + k) for k in range(10, 25, 2)]
    for t in warm:
        srv.wait(t, 120.0)
        srv.release(t)
    sampler = ClockSampler(local)
    sampler.start()
    outstanding = []
    lat, done_t, bad, limbs_done = [], [], 0, 0
    t0 = time.perf_counter()
    i = 0

    def reap(block: bool):
        nonlocal bad, limbs_done
        while outstanding:
            t, na, nb = outstanding[0]
            r = srv.poll(t) if not block else srv.wait(t, 300.0)
            if r.state < b200mul.DONE:
                return
            outstanding.pop(0)
            if r.state != b200mul.DONE or r.residues_ok != 1:
                bad += 1
            lat.append((r.t_done_ns - r.t_submit_ns) * 1e-6)
            done_t.append(r.t_done_ns)
            limbs_done += na + nb
            srv.release(t)

    while i < n_req:
        now = time.perf_counter() - t0
        while i < n_req and arrivals[i] <= now:
            na, nb = int(lens[i, 0]), int(lens[i, 1])
            outstanding.append((srv.submit(na, nb, 7 * i + 1, 7 * i + 2), na, nb))
            i += 1
        reap(False)
        nxt = arrivals[i] if i < n_req else now
        time.sleep(max(0.0, min(0.0005, nxt - (time.perf_counter() - t0))))
    submit_end = time.perf_counter() - t0
    reap(True)
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    st = srv.stats()
    srv.stop()
    offered_limbs = int(lens.sum())
    if rk.world > 1:
        mine = {"lat": lat, "bad": bad, "limbs": limbs_done, "offered": offered_limbs, "wall": wall, "n": n_req}
        every = [None] * rk.world
        rk.dist.all_gather_object(every, mine)
        lat = [x for e in every for x in e["lat"]]
        bad = sum(e["bad"] for e in every)
        limbs_done = sum(e["limbs"] for e in every)
        offered_limbs = sum(e["offered"] for e in every)
        wall = max(e["wall"] for e in every)
        n_req = sum(e["n"] for e in every)
    lat = np.array(lat)
    return {
        "metric": "serve p50/p99 latency ms (Poisson arrivals, log-uniform 2^10..2^24 limbs)",
        "value": round(float(np.percentile(lat, 50)), 2), "unit": "ms",
        "p99_ms": round(float(np.percentile(lat, 99)), 2), "mean_ms": round(float(lat.mean()), 2),
        "n_gpus": rk.world, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64 (GF(p), p=2^64-2^32+1)",
        "data": "synthetic: seeded random limbs generated on the device per request",
        "config": {"workload": f"{rate} req/s Poisson for {args.duration} s per GPU", "requests": n_req,
                   "hbm_budget_gb": args.serve_budget_gb, "streams": args.serve_streams,
                   "max_batch": args.serve_batch, "submit_window_s": round(submit_end, 2)},
        "throughput": {"req_per_s": round(n_req / wall, 1), "glimbs_per_s": round(limbs_done / wall / 1e9, 3),
                       "offered_glimbs_per_s": round(offered_limbs / args.duration / 1e9, 3),
                       "wall_s": round(wall, 2)},
        "all_products_residue_checked_ok": bad == 0, "failed_or_mismatched": bad,
        "server": st, "clocks": clocks}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["single", "batch", "chudnovsky", "pi", "serve"], default="single",
                    help="single: the 2^24-limb product (headline); batch: 4096 log-uniform pairs; "
                         "chudnovsky: the binary-splitting tree; pi: the whole digit string on the device; "
                         "serve: Poisson request stream")
    ap.add_argument("--digits", type=int, default=10000000)
    ap.add_argument("--rate", type=float, default=2000.0, help="serve: Poisson arrival rate (req/s)")
    ap.add_argument("--duration", type=float, default=10.0, help="serve: seconds of arrivals")
    ap.add_argument("--serve-budget-gb", type=int, default=120)
    ap.add_argument("--serve-streams", type=int, default=4)
    ap.add_argument("--serve-batch", type=int, default=8,
                    help="requests per dispatch (8: lowest latency on the log-uniform mix, measured)")
    ap.add_argument("--batch-jobs", type=int, default=4096)
    ap.add_argument("--batch-split", action="store_true",
                    help="batch, several GPUs: partition one batch over the ranks (LPT) instead of one per rank")
    ap.add_argument("--na", type=int, default=NA)
    ap.add_argument("--nb", type=int, default=NB)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--trace-steps", type=int, default=10)
    ap.add_argument("--cpu-sample-log", type=int, default=24,
                    help="log2 limbs of the CPU-baseline product (24: the headline product itself)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="single: skip the batch and serving measurements that the default line carries")
    ap.add_argument("--autotune", action="store_true",
                    help="single: time every candidate plan first and keep the fastest (the default plan of each "
                         "length is already the measured fastest; candidates within noise of it may win)")
    ap.add_argument("--no-autotune", action="store_true", help="single: keep the default plan (the default)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "chudnovsky":
        run_chudnovsky(args)
    elif args.workload == "pi":
        run_pi(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
