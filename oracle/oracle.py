"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracles.

Two libraries are loaded from this directory:

* ``liboracle.so`` -- our plain-C restatement of the reference's CPU path
  (``gl_oracle.c``; every function there cites the reference line it follows).
* ``_ref/libpidigits_ref.so`` -- the reference's own CPU sources compiled
  unmodified (``Makefile`` target ``ref``): ``mul_schoolbook``,
  ``mul_karatsuba``, ``mul_ntt_cpu`` (src/bignum.cpp:125-195,
  src/ntt_cpu.cpp:111-129), the Goldilocks field (include/goldilocks.h) and
  ``chudnovsky_bs`` / ``compute_pi_chudnovsky`` (src/chudnovsky.cpp).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker. The product never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libpidigits_ref.so")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64 = ctypes.c_uint64
_sz = ctypes.c_size_t

_port = None
_ref = None


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def port_lib():
    """Load (building on first use if absent) our C restatement."""
    global _port
    if _port is None:
        if not os.path.exists(PORT_PATH):
            import subprocess

            subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
        lib = ctypes.CDLL(PORT_PATH)
        for name in ("orc_gl_add", "orc_gl_sub", "orc_gl_mul", "orc_gl_mul_def", "orc_gl_pow",
                     "orc_gl_reduce128"):
            getattr(lib, name).restype = _u64
            getattr(lib, name).argtypes = [_u64, _u64]
        for name in ("orc_gl_inv", "orc_gl_root_of_unity"):
            getattr(lib, name).restype = _u64
            getattr(lib, name).argtypes = [_u64]
        lib.orc_ntt_length.restype = _u64
        lib.orc_ntt_length.argtypes = [_u64, _u64]
        for name in ("orc_mul_ntt", "orc_mul_schoolbook"):
            getattr(lib, name).restype = _u64
            getattr(lib, name).argtypes = [_u32p, _u64, _u32p, _u64, _u32p]
        lib.orc_carry_propagate.restype = _u64
        lib.orc_carry_propagate.argtypes = [ctypes.POINTER(ctypes.c_uint64), _u64, _u32p, _u64]
        lib.orc_gen_operand.restype = None
        lib.orc_gen_operand.argtypes = [_u64, _u64, ctypes.c_int, _u32p]
        lib.orc_bs_run.restype = ctypes.c_void_p
        lib.orc_bs_run.argtypes = [_u64, _u64]
        lib.orc_bs_len.restype = _u64
        lib.orc_bs_len.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.orc_bs_sign.restype = ctypes.c_int
        lib.orc_bs_sign.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.orc_bs_copy.restype = None
        lib.orc_bs_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, _u32p]
        lib.orc_bs_free.restype = None
        lib.orc_bs_free.argtypes = [ctypes.c_void_p]
        _port = lib
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref_lib():
    """Load the reference's own compiled CPU code (oracle/_ref)."""
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_PATH)
        lib.ref_mul.restype = ctypes.c_int
        lib.ref_mul.argtypes = [ctypes.c_int, _u32p, _sz, _u32p, _sz, _u32p, _sz,
                                ctypes.POINTER(_sz)]
        for name in ("ref_gl_add", "ref_gl_sub", "ref_gl_mul", "ref_gl_pow", "ref_gl_reduce128",
                     "ref_ntt_length"):
            getattr(lib, name).restype = _u64
            getattr(lib, name).argtypes = [_u64, _u64]
        for name in ("ref_gl_inv", "ref_gl_root_of_unity", "ref_chudnovsky_terms_for_digits"):
            getattr(lib, name).restype = _u64
            getattr(lib, name).argtypes = [_u64]
        lib.ref_bs_run.restype = ctypes.c_void_p
        lib.ref_bs_run.argtypes = [_u64, _u64, ctypes.c_int]
        lib.ref_bs_len.restype = _sz
        lib.ref_bs_len.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.ref_bs_sign.restype = ctypes.c_int
        lib.ref_bs_sign.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.ref_bs_copy.restype = None
        lib.ref_bs_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, _u32p]
        lib.ref_bs_free.restype = None
        lib.ref_bs_free.argtypes = [ctypes.c_void_p]
        lib.ref_compute_pi.restype = _sz
        lib.ref_compute_pi.argtypes = [_u64, ctypes.c_char_p, _sz, ctypes.POINTER(_u64)]
        _ref = lib
    return _ref


# ---- multiply ----------------------------------------------------------------

def _as_u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def mul_port(a, b, schoolbook: bool = False) -> np.ndarray:
    """Our C restatement: the reference's CPU NTT (or schoolbook) multiply."""
    a, b = _as_u32(a), _as_u32(b)
    if a.size == 0 or b.size == 0:
        return np.zeros(0, np.uint32)
    out = np.zeros(a.size + b.size, np.uint32)
    fn = port_lib().orc_mul_schoolbook if schoolbook else port_lib().orc_mul_ntt
    n = fn(_ptr(a), a.size, _ptr(b), b.size, _ptr(out))
    return out[:n]


BACKENDS = {"schoolbook": 0, "karatsuba": 1, "ntt-cpu": 2, "auto": 3}


def mul_ref(a, b, backend: str = "ntt-cpu") -> np.ndarray:
    """The reference's own compiled multiply (schoolbook/karatsuba/ntt-cpu/auto)."""
    a, b = _as_u32(a), _as_u32(b)
    out = np.zeros(max(1, a.size + b.size), np.uint32)
    n = _sz(0)
    rc = ref_lib().ref_mul(BACKENDS[backend], _ptr(a), a.size, _ptr(b), b.size, _ptr(out),
                           out.size, ctypes.byref(n))
    if rc != 0:
        raise RuntimeError("ref_mul: output buffer too small")
    return out[: n.value]


def gen_operand(seed: int, n: int, kind: int = 0) -> np.ndarray:
    """The C copy of the seeded operand generator (cross-checks the numpy one)."""
    out = np.zeros(n, np.uint32)
    if n:
        port_lib().orc_gen_operand(seed, n, kind, _ptr(out))
    return out


# ---- binary splitting -----------------------------------------------------------

def _read_pqt(lib, h, prefix):
    res = []
    for w in range(3):
        n = getattr(lib, prefix + "_len")(h, w)
        v = np.zeros(n, np.uint32)
        if n:
            getattr(lib, prefix + "_copy")(h, w, _ptr(v))
        res.append((getattr(lib, prefix + "_sign")(h, w), v))
    getattr(lib, prefix + "_free")(h)
    return res


def bs_port(a: int, b: int):
    """Our restatement of chudnovsky_bs(a, b): [(sign, mag) for P, Q, T]."""
    lib = port_lib()
    return _read_pqt(lib, lib.orc_bs_run(a, b), "orc_bs")


def bs_ref(a: int, b: int, backend: str = "auto"):
    """The reference's chudnovsky_bs(a, b) with the given CPU backend forced."""
    lib = ref_lib()
    return _read_pqt(lib, lib.ref_bs_run(a, b, BACKENDS[backend]), "ref_bs")


def compute_pi_ref(digits: int) -> str:
    """The reference's compute_pi_chudnovsky(digits) on the CPU."""
    buf = ctypes.create_string_buffer(digits + 64)
    terms = _u64(0)
    n = ref_lib().ref_compute_pi(digits, buf, len(buf), ctypes.byref(terms))
    if n == 0:
        raise RuntimeError("ref_compute_pi: buffer too small")
    return buf.value.decode()
