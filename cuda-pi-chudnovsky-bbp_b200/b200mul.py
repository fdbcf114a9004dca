"""Python host mirror of the B200 multiply backend (ctypes over libb2m.so).

Mirrors the reference's multiply-backend interface for the ``ntt-cuda`` path
(include/bignum.h:180-205): ``mul_ntt_cuda(a, b)`` takes and returns
little-endian u32 limb arrays (numpy), ``cuda_available()`` reports whether the
backend initialised. Unlike the reference (src/ntt_cuda.cu:182,239-241) there
is no CPU fallback: every failure raises :class:`B2MError` carrying the C
status code.

The library is loaded from this directory; importing this module on a machine
where ``libb2m.so`` has not been built raises immediately.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb2m.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "b2m.h")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"libb2m.so not built ({LIB_PATH}); run `make -C {HERE}`")

lib = ctypes.CDLL(LIB_PATH)

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_u64 = ctypes.c_uint64

STATUS = {
    0: "B2M_OK", 1: "B2M_ERR_INVALID_ARGUMENT", 2: "B2M_ERR_NO_DEVICE", 3: "B2M_ERR_NOT_INITIALIZED",
    4: "B2M_ERR_CUDA", 5: "B2M_ERR_OUT_OF_MEMORY", 6: "B2M_ERR_TOO_LARGE", 7: "B2M_ERR_OUTPUT_TOO_SMALL",
    8: "B2M_ERR_DEVICE_TIMEOUT", 9: "B2M_ERR_QUEUE_FULL", 10: "B2M_ERR_NOT_FOUND", 11: "B2M_ERR_SHUTDOWN", 12: "B2M_ERR_INTERNAL",
}
OK, INVALID_ARGUMENT, NO_DEVICE, NOT_INITIALIZED = 0, 1, 2, 3
CUDA, OUT_OF_MEMORY, TOO_LARGE, OUTPUT_TOO_SMALL, DEVICE_TIMEOUT = 4, 5, 6, 7, 8


class B2MError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        detail = lib.b2m_last_error().decode()
        super().__init__(f"{where}: {STATUS.get(status, status)} ({lib.b2m_strerror(status).decode()})"
                         + (f": {detail}" if detail else ""))


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


_sig("b2m_init", ctypes.c_int, [ctypes.c_int, _u64])
_sig("b2m_shutdown", ctypes.c_int, [])
_sig("b2m_cuda_available", ctypes.c_int, [])
_sig("b2m_strerror", ctypes.c_char_p, [ctypes.c_int])
_sig("b2m_last_error", ctypes.c_char_p, [])
_sig("b2m_ntt_length", _u64, [_u64, _u64])
_sig("b2m_workspace_bytes", _u64, [_u64, _u64])
_sig("b2m_mul_host", ctypes.c_int, [_u32p, _u64, _u32p, _u64, _u32p, _u64, _u64p])
_sig("b2m_mul_device", ctypes.c_int,
     [ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, ctypes.c_void_p, ctypes.c_void_p])
_sig("b2m_stream_check", ctypes.c_int, [ctypes.c_void_p])
_sig("b2m_mul_device_noalloc", ctypes.c_int,
     [ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, ctypes.c_void_p, ctypes.c_void_p])


class PlanDesc(ctypes.Structure):
    _fields_ = [("ntt_log2", ctypes.c_uint32), ("npass", ctypes.c_uint32), ("logr", ctypes.c_uint32 * 3),
                ("logc", ctypes.c_uint32 * 3), ("launches", ctypes.c_uint32), ("three", ctypes.c_uint32)]


class KernelTime(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("logr", ctypes.c_uint32), ("ms", ctypes.c_float)]


KERNEL_KINDS = {1: "fwd_first", 2: "fwd_mid", 3: "fwd_last", 4: "fused_last", 5: "inv_mid", 6: "carry",
                7: "mul_small", 8: "r3_fwd", 9: "r3_inv"}

_sig("b2m_plan_describe", ctypes.c_int, [_u64, _u64, ctypes.POINTER(PlanDesc)])
_sig("b2m_mul_device_traced", ctypes.c_int,
     [ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.POINTER(KernelTime), ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)])


def check(status: int, where: str) -> None:
    if status != OK:
        raise B2MError(status, where)


def header_symbols(path: str = HEADER) -> list[str]:
    """Every function name declared in include/b2m.h (for export checks)."""
    text = open(path).read()
    return sorted(set(re.findall(r"\b(b2m_[a-z0-9_]+)\s*\(", text)))


def init(device: int = 0, hbm_budget_bytes: int = 0) -> None:
    check(lib.b2m_init(device, hbm_budget_bytes), "b2m_init")


def shutdown() -> None:
    check(lib.b2m_shutdown(), "b2m_shutdown")


def cuda_available() -> bool:
    """Reference: pidigits::cuda_available() (src/ntt_cuda.cu:165-173)."""
    return bool(lib.b2m_cuda_available())


def ntt_length(na: int, nb: int) -> int:
    """Reference: ntt_length (include/ntt.h:47-50)."""
    return int(lib.b2m_ntt_length(na, nb))


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def mul_ntt_cuda(a, b, out: np.ndarray | None = None) -> np.ndarray:
    """Reference: pidigits::mul_ntt_cuda (src/ntt_cuda.cu:179-243).

    Host arrays in, trimmed product out, synchronous. ``out`` (u32, at least
    len(a) + len(b) limbs, ideally page-locked) may be supplied to avoid an
    allocation; the returned array is then a view of it.
    """
    a, b = _u32(a), _u32(b)
    if a.size == 0 or b.size == 0:
        return np.zeros(0, np.uint32)
    if out is None:
        out = np.empty(a.size + b.size, np.uint32)
    n = _u64(0)
    check(lib.b2m_mul_host(a.ctypes.data_as(_u32p), a.size, b.ctypes.data_as(_u32p), b.size,
                           out.ctypes.data_as(_u32p), out.size, ctypes.byref(n)), "b2m_mul_host")
    return out[: n.value]


def mul_device(a_ptr: int, na: int, b_ptr: int, nb: int, out_ptr: int, out_cap: int,
               out_len_ptr: int = 0, stream: int = 0) -> None:
    """Device-pointer product ordered on `stream` (raw CUDA handles as ints)."""
    check(lib.b2m_mul_device(a_ptr, na, b_ptr, nb, out_ptr, out_cap, out_len_ptr or None, stream or None),
          "b2m_mul_device")


def mul_device_noalloc(a_ptr: int, na: int, b_ptr: int, nb: int, out_ptr: int, out_cap: int,
                       out_len_ptr: int = 0, stream: int = 0) -> None:
    """The product without any device allocation, for callers that cannot
    allocate at call time: scratch is the library's fixed static device array,
    so na + nb <= 2^19 limbs, and calls that overlap on the GPU race."""
    check(lib.b2m_mul_device_noalloc(a_ptr, na, b_ptr, nb, out_ptr, out_cap, out_len_ptr or None,
                                     stream or None), "b2m_mul_device_noalloc")


def stream_check(stream: int = 0) -> None:
    check(lib.b2m_stream_check(stream or None), "b2m_stream_check")


# ---- seeded operands -----------------------------------------------------------
# limb i of (seed, n) = high 32 bits of splitmix64's output function applied to
# seed + (i + 1) * 0x9E3779B97F4A7C15; the top limb is forced non-zero.
# kind 0 = uniform random limbs, 1 = all 0xFFFFFFFF (worst-case carries).
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


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


def plan_describe(na: int, nb: int) -> dict:
    d = PlanDesc()
    check(lib.b2m_plan_describe(na, nb, ctypes.byref(d)), "b2m_plan_describe")
    return {"ntt_log2": d.ntt_log2, "npass": d.npass, "logr": list(d.logr)[: max(d.npass, 1)],
            "logc": list(d.logc)[: max(d.npass, 1)], "launches": d.launches, "three": d.three,
            "points": (3 if d.three else 1) << d.ntt_log2}


class TuneEntry(ctypes.Structure):
    _fields_ = [("plan", PlanDesc), ("ms", ctypes.c_float), ("chosen", ctypes.c_uint32)]


_sig("b2m_autotune", ctypes.c_int, [_u64, _u64, ctypes.c_void_p, ctypes.POINTER(TuneEntry), ctypes.c_uint32,
                                    ctypes.POINTER(ctypes.c_uint32)])


def autotune(na: int, nb: int, stream: int = 0) -> list[dict]:
    """Times every candidate plan for an na x nb product and keeps the
    fastest for that transform length (b2m_autotune). Returns the timings."""
    out = (TuneEntry * 512)()
    n = ctypes.c_uint32(0)
    check(lib.b2m_autotune(na, nb, stream or None, out, 512, ctypes.byref(n)), "b2m_autotune")
    res = []
    for e in out[: n.value]:
        k = max(e.plan.npass, 1)
        res.append({"logr": list(e.plan.logr)[:k], "logc": list(e.plan.logc)[:k], "ms": round(e.ms, 4),
                    "chosen": bool(e.chosen)})
    return res


_sig("b2m_selftest_wait_timeout", ctypes.c_int, [ctypes.c_void_p])


def selftest_wait_timeout(stream: int = 0) -> int:
    """Status of b2m_selftest_wait_timeout (8, B2M_ERR_DEVICE_TIMEOUT, when the
    bounded device-side wait fires as designed)."""
    return int(lib.b2m_selftest_wait_timeout(stream or None))


_sig("b2m_field_eval_host", ctypes.c_int, [ctypes.c_int, _u64p, _u64p, _u64p, ctypes.c_uint64])
FIELD_OPS = {"add": 0, "sub": 1, "mul": 2, "shl": 3, "pow": 4, "inv": 5, "dft8": 6, "idft8": 7, "shl_rt": 8, "shl_160": 9, "shl_rt2": 10}


def field_eval(op: str, a, b=None) -> np.ndarray:
    """The device field arithmetic of the kernels, element-wise
    (b2m_field_eval_host): op in FIELD_OPS, a and b u64 arrays."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64))
    b = np.zeros_like(a) if b is None else np.ascontiguousarray(np.asarray(b, dtype=np.uint64))
    out = np.zeros_like(a)
    check(lib.b2m_field_eval_host(FIELD_OPS[op], a.ctypes.data_as(_u64p), b.ctypes.data_as(_u64p),
                                  out.ctypes.data_as(_u64p), a.size), "b2m_field_eval_host")
    return out


_sig("b2m_set_plan", ctypes.c_int, [ctypes.POINTER(PlanDesc)])


def set_plan(ntt_log2: int, logr, logc) -> None:
    """Fixes the plan of one transform length (b2m_set_plan)."""
    d = PlanDesc()
    d.ntt_log2, d.npass = ntt_log2, len(logr) if ntt_log2 > 13 else 0
    for k, (r, c) in enumerate(zip(logr, logc)):
        d.logr[k], d.logc[k] = r, c
    check(lib.b2m_set_plan(ctypes.byref(d)), "b2m_set_plan")


def mul_device_traced(a_ptr: int, na: int, b_ptr: int, nb: int, out_ptr: int, out_cap: int,
                      out_len_ptr: int = 0, stream: int = 0) -> list[tuple[str, int, float]]:
    """Device product with per-launch CUDA-event times: [(kind, logr, ms), ...]."""
    times = (KernelTime * 16)()
    n = ctypes.c_uint32(0)
    check(lib.b2m_mul_device_traced(a_ptr, na, b_ptr, nb, out_ptr, out_cap, out_len_ptr or None, stream or None,
                                    times, 16, ctypes.byref(n)), "b2m_mul_device_traced")
    return [(KERNEL_KINDS[times[i].kind], times[i].logr, times[i].ms) for i in range(n.value)]


# ---- batched products ----------------------------------------------------------------
class Job(ctypes.Structure):
    """b2m_job: device pointers of one product of a batch."""
    _fields_ = [("a", ctypes.c_void_p), ("na", _u64), ("b", ctypes.c_void_p), ("nb", _u64),
                ("out", ctypes.c_void_p), ("out_cap", _u64), ("out_len", ctypes.c_void_p)]


BATCH_GRAPH, BATCH_AUTOTUNE = 1, 2
_sig("b2m_batch_create", ctypes.c_int, [ctypes.POINTER(Job), _u64, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)])
_sig("b2m_batch_launch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p])
_sig("b2m_batch_destroy", ctypes.c_int, [ctypes.c_void_p])
_sig("b2m_mul_batch", ctypes.c_int, [ctypes.POINTER(Job), _u64, ctypes.c_void_p])


def _jobs(jobs):
    arr = (Job * max(1, len(jobs)))()
    for i, (a, na, b, nb, out, cap, olen) in enumerate(jobs):
        arr[i] = Job(a or None, na, b or None, nb, out or None, cap, olen or None)
    return arr


class Batch:
    """A planned batch of independent products (device pointers); launch() it
    any number of times. jobs: [(a_ptr, na, b_ptr, nb, out_ptr, out_cap, out_len_ptr)]."""

    def __init__(self, jobs, flags: int = BATCH_GRAPH):
        self._arr = _jobs(jobs)
        self.handle = ctypes.c_void_p()
        check(lib.b2m_batch_create(self._arr, len(jobs), flags, ctypes.byref(self.handle)), "b2m_batch_create")

    def launch(self, stream: int = 0) -> None:
        check(lib.b2m_batch_launch(self.handle, stream or None), "b2m_batch_launch")

    def close(self) -> None:
        if self.handle:
            check(lib.b2m_batch_destroy(self.handle), "b2m_batch_destroy")
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mul_batch(jobs, stream: int = 0) -> None:
    """One-shot batch (no graph), synchronous on `stream`."""
    arr = _jobs(jobs)
    check(lib.b2m_mul_batch(arr, len(jobs), stream or None), "b2m_mul_batch")


# ---- Chudnovsky binary splitting ---------------------------------------------------
_sig("b2m_chudnovsky_bs", ctypes.c_int, [_u64, _u64, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)])
_sig("b2m_pqt_info", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_u64), ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(_u64)])
_sig("b2m_pqt_device", ctypes.c_void_p, [ctypes.c_void_p, ctypes.c_int])
_sig("b2m_pqt_copy", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _u32p, _u64])
_sig("b2m_pqt_free", ctypes.c_int, [ctypes.c_void_p])
_sig("b2m_pqt_merge", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)])
_sig("b2m_pqt_import", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(_u64), ctypes.c_int32,
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)])


class PQT:
    """Device-resident (P, Q, T) of a Chudnovsky term range (b2m_pqt)."""

    def __init__(self, handle):
        self.handle = handle
        ln = (_u64 * 3)()
        sg = ctypes.c_int32()
        lv = ctypes.c_uint32()
        pr = _u64()
        check(lib.b2m_pqt_info(handle, ln, ctypes.byref(sg), ctypes.byref(lv), ctypes.byref(pr)), "b2m_pqt_info")
        self.lengths = [int(x) for x in ln]
        self.t_sign = int(sg.value)
        self.levels = int(lv.value)
        self.products = int(pr.value)

    def limbs(self, which: int) -> np.ndarray:
        out = np.zeros(max(1, self.lengths[which]), np.uint32)
        check(lib.b2m_pqt_copy(self.handle, which, out.ctypes.data_as(_u32p), out.size), "b2m_pqt_copy")
        return out[: self.lengths[which]]

    def signed(self):
        """[(sign, magnitude)] for P, Q, T, as the reference's BigInt holds them."""
        return [(1 if self.lengths[0] else 0, self.limbs(0)), (1 if self.lengths[1] else 0, self.limbs(1)),
                (self.t_sign, self.limbs(2))]

    def free(self) -> None:
        if self.handle:
            check(lib.b2m_pqt_free(self.handle), "b2m_pqt_free")
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def chudnovsky_bs(a: int, b: int, stream: int = 0) -> PQT:
    """Reference: chudnovsky_bs(a, b) (src/chudnovsky.cpp:64-102), on the device."""
    h = ctypes.c_void_p()
    check(lib.b2m_chudnovsky_bs(a, b, stream or None, ctypes.byref(h)), "b2m_chudnovsky_bs")
    return PQT(h)


def pqt_merge(left: PQT, right: PQT, stream: int = 0) -> PQT:
    """(P, Q, T) of the union of two adjacent term ranges, left first
    (reference: the merge step of chudnovsky_bs, src/chudnovsky.cpp:96-100)."""
    h = ctypes.c_void_p()
    check(lib.b2m_pqt_merge(left.handle, right.handle, stream or None, ctypes.byref(h)), "b2m_pqt_merge")
    return PQT(h)


def pqt_import(ptrs, lengths, t_sign: int, stream: int = 0) -> PQT:
    """A node copied from device limbs: ptrs/lengths of P, Q, |T| and T's sign."""
    p = (ctypes.c_void_p * 3)(*[int(x) if x else None for x in ptrs])
    ln = (_u64 * 3)(*[int(x) for x in lengths])
    h = ctypes.c_void_p()
    check(lib.b2m_pqt_import(p, ln, int(t_sign), stream or None, ctypes.byref(h)), "b2m_pqt_import")
    return PQT(h)


_sig("b2m_divmod_device", ctypes.c_int, [ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, ctypes.c_void_p, _u64,
                                         ctypes.POINTER(_u64), ctypes.c_void_p, _u64, ctypes.POINTER(_u64),
                                         ctypes.c_void_p])
_sig("b2m_isqrt_device", ctypes.c_int, [ctypes.c_void_p, _u64, ctypes.c_void_p, _u64, ctypes.POINTER(_u64),
                                        ctypes.c_void_p])


def divmod_device(d_a: int, na: int, d_b: int, nb: int, d_q: int, q_cap: int, d_r: int, r_cap: int,
                  stream: int = 0):
    """Reference: divmod_knuth / div_fast (src/bignum_div.cpp:162-178), on the
    device. Returns the trimmed lengths (q_len, r_len)."""
    ql, rl = _u64(0), _u64(0)
    check(lib.b2m_divmod_device(d_a or None, na, d_b, nb, d_q or None, q_cap, ctypes.byref(ql), d_r or None,
                                r_cap, ctypes.byref(rl), stream or None), "b2m_divmod_device")
    return int(ql.value), int(rl.value)


def isqrt_device(d_a: int, na: int, d_out: int, cap: int, stream: int = 0) -> int:
    """Reference: isqrt (src/bignum_div.cpp:189-204), on the device. Returns
    the trimmed length of floor(sqrt(a))."""
    n = _u64(0)
    check(lib.b2m_isqrt_device(d_a or None, na, d_out, cap, ctypes.byref(n), stream or None), "b2m_isqrt_device")
    return int(n.value)


DIGITS_PER_TERM = 14.181647462725477  # src/chudnovsky.cpp:46


def chudnovsky_terms_for_digits(digits: int) -> int:
    """Reference: chudnovsky_terms_for_digits (src/chudnovsky.cpp:54-59)."""
    n = int(float(digits) / DIGITS_PER_TERM) + 2
    return max(n, 2)


def _to_int(limbs: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(limbs, dtype="<u4").tobytes(), "little")


class PiTimings(ctypes.Structure):
    _fields_ = [("tree_ms", ctypes.c_double), ("sqrt_ms", ctypes.c_double), ("div_ms", ctypes.c_double),
                ("decimal_ms", ctypes.c_double), ("total_ms", ctypes.c_double), ("terms", _u64)]


_sig("b2m_to_decimal_device", ctypes.c_int, [ctypes.c_void_p, _u64, ctypes.c_char_p, _u64, ctypes.POINTER(_u64),
                                             ctypes.c_void_p])
_sig("b2m_compute_pi", ctypes.c_int, [_u64, ctypes.c_char_p, _u64, ctypes.POINTER(_u64), ctypes.POINTER(PiTimings)])


_sig("b2m_divmod_host", ctypes.c_int, [_u32p, _u64, _u32p, _u64, _u32p, _u64, ctypes.POINTER(_u64), _u32p, _u64,
                                       ctypes.POINTER(_u64)])
_sig("b2m_isqrt_host", ctypes.c_int, [_u32p, _u64, _u32p, _u64, ctypes.POINTER(_u64)])
_sig("b2m_to_decimal_host", ctypes.c_int, [_u32p, _u64, ctypes.c_char_p, _u64, ctypes.POINTER(_u64)])


def _u32_arr(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.uint32)


def divmod_host(a, b):
    """Host-limb floor division (b2m_divmod_host): (q, r) as u32 arrays."""
    a, b = _u32_arr(a), _u32_arr(b)
    q = np.zeros(max(1, a.size - b.size + 1), np.uint32)
    r = np.zeros(max(1, b.size), np.uint32)
    ql, rl = _u64(0), _u64(0)
    check(lib.b2m_divmod_host(a.ctypes.data_as(_u32p), a.size, b.ctypes.data_as(_u32p), b.size,
                              q.ctypes.data_as(_u32p), q.size, ctypes.byref(ql), r.ctypes.data_as(_u32p), r.size,
                              ctypes.byref(rl)), "b2m_divmod_host")
    return q[: ql.value], r[: rl.value]


def isqrt_host(a):
    a = _u32_arr(a)
    s = np.zeros((a.size + 1) // 2 + 1, np.uint32)
    n = _u64(0)
    check(lib.b2m_isqrt_host(a.ctypes.data_as(_u32p), a.size, s.ctypes.data_as(_u32p), s.size, ctypes.byref(n)),
          "b2m_isqrt_host")
    return s[: n.value]


def to_decimal_host(a) -> str:
    a = _u32_arr(a)
    cap = int(a.size * 9.64) + 16
    buf = ctypes.create_string_buffer(cap)
    n = _u64(0)
    check(lib.b2m_to_decimal_host(a.ctypes.data_as(_u32p), a.size, buf, cap, ctypes.byref(n)), "b2m_to_decimal_host")
    return buf.raw[: n.value].decode()


def to_decimal_device(d_a: int, na: int, stream: int = 0) -> str:
    """Reference: BigInt::to_decimal (src/bignum_div.cpp:239-267), on the device."""
    cap = int(na * 32 * 0.30103) + 16
    buf = ctypes.create_string_buffer(cap)
    n = _u64(0)
    check(lib.b2m_to_decimal_device(d_a or None, na, buf, cap, ctypes.byref(n), stream or None),
          "b2m_to_decimal_device")
    return buf.raw[: n.value].decode()


def compute_pi(digits: int, timings: dict | None = None) -> str:
    """Reference: compute_pi_chudnovsky (src/chudnovsky.cpp:107-164), every
    step on the device (b2m_compute_pi): tree, square root, division and
    decimal conversion. Returns "3." and `digits` digits."""
    buf = ctypes.create_string_buffer(digits + 8)
    n = _u64(0)
    t = PiTimings()
    check(lib.b2m_compute_pi(digits, buf, len(buf), ctypes.byref(n), ctypes.byref(t)), "b2m_compute_pi")
    if timings is not None:
        timings.update({"terms": int(t.terms), "tree_ms": t.tree_ms, "sqrt_ms": t.sqrt_ms, "div_ms": t.div_ms,
                        "decimal_ms": t.decimal_ms, "total_ms": t.total_ms})
    return buf.raw[: n.value].decode()


# ---- serving ------------------------------------------------------------------------
class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", _u64), ("streams", ctypes.c_uint32), ("max_batch", ctypes.c_uint32),
                ("max_pending", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class Request(ctypes.Structure):
    _fields_ = [("a", ctypes.c_void_p), ("na", _u64), ("b", ctypes.c_void_p), ("nb", _u64), ("seed_a", _u64),
                ("seed_b", _u64), ("kind", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("out", ctypes.c_void_p), ("out_cap", _u64)]


class Result(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("status", ctypes.c_int), ("out", ctypes.c_void_p), ("out_len", _u64),
                ("t_submit_ns", _u64), ("t_admit_ns", _u64), ("t_done_ns", _u64), ("residues_ok", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, _u64) for n in ("submitted", "completed", "failed", "dispatches", "inflight_dispatches",
                                    "queued", "max_queue", "bytes_in_use", "peak_bytes",
                                    "max_inflight_dispatches", "host_dispatch_ns", "slot_busy_ns")]


_sig("b2m_server_start", ctypes.c_int, [ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)])
_sig("b2m_server_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Request), ctypes.POINTER(_u64)])
_sig("b2m_server_poll", ctypes.c_int, [ctypes.c_void_p, _u64, ctypes.POINTER(Result)])
_sig("b2m_server_wait", ctypes.c_int, [ctypes.c_void_p, _u64, ctypes.c_double, ctypes.POINTER(Result)])
_sig("b2m_server_release", ctypes.c_int, [ctypes.c_void_p, _u64])
_sig("b2m_server_get_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)])
_sig("b2m_server_stop", ctypes.c_int, [ctypes.c_void_p])
_sig("b2m_gen_operand", ctypes.c_int, [_u64, _u64, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p])

QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3


def gen_operand_device(seed: int, n: int, kind: int, ptr: int, stream: int = 0) -> None:
    """Device copy of gen_operand (b2m_gen_operand)."""
    check(lib.b2m_gen_operand(seed, n, kind, ptr, stream or None), "b2m_gen_operand")


class Server:
    """Continuous-batching multiply server (b2m_server_*)."""

    def __init__(self, hbm_budget_bytes: int = 0, streams: int = 0, max_batch: int = 0, max_pending: int = 0):
        cfg = ServerConfig(hbm_budget_bytes, streams, max_batch, max_pending, 0)
        self.handle = ctypes.c_void_p()
        check(lib.b2m_server_start(ctypes.byref(cfg), ctypes.byref(self.handle)), "b2m_server_start")

    def submit(self, na: int, nb: int, seed_a: int = 0, seed_b: int = 0, kind: int = 0, a: int = 0, b: int = 0,
               out: int = 0, out_cap: int = 0) -> int:
        req = Request(a or None, na, b or None, nb, seed_a, seed_b, kind, 0, out or None, out_cap)
        t = _u64()
        check(lib.b2m_server_submit(self.handle, ctypes.byref(req), ctypes.byref(t)), "b2m_server_submit")
        return t.value

    def poll(self, ticket: int) -> Result:
        r = Result()
        check(lib.b2m_server_poll(self.handle, ticket, ctypes.byref(r)), "b2m_server_poll")
        return r

    def wait(self, ticket: int, timeout_s: float = 60.0) -> Result:
        r = Result()
        st = lib.b2m_server_wait(self.handle, ticket, timeout_s, ctypes.byref(r))
        if st not in (OK, DEVICE_TIMEOUT):
            check(st, "b2m_server_wait")
        return r

    def release(self, ticket: int) -> None:
        check(lib.b2m_server_release(self.handle, ticket), "b2m_server_release")

    def stats(self) -> dict:
        s = ServerStats()
        check(lib.b2m_server_get_stats(self.handle, ctypes.byref(s)), "b2m_server_get_stats")
        return {n: int(getattr(s, n)) for n, _ in ServerStats._fields_}

    def stop(self) -> None:
        if self.handle:
            check(lib.b2m_server_stop(self.handle), "b2m_server_stop")
            self.handle = ctypes.c_void_p()

