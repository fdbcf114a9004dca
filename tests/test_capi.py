"""CPU tests of the C ABI boundary: the library loads, exports every symbol the
header declares, and its host logic (sizes, statuses, argument checks) behaves
without touching a GPU."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import b200mul
import oracle

PKG = os.path.dirname(b200mul.LIB_PATH)


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def test_every_declared_symbol_is_exported():
    syms = b200mul.header_symbols()
    assert "b2m_mul_host" in syms and "b2m_init" in syms
    for s in syms:
        assert hasattr(b200mul.lib, s), f"libb2m.so does not export {s}"


def test_shim_exports_reference_signatures():
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(PKG, "libb2m_shim.so")],
                         capture_output=True, text=True, check=True).stdout
    demangled = subprocess.run(["c++filt"], input=out, capture_output=True, text=True, check=True).stdout
    # include/bignum.h:200-205
    assert "pidigits::mul_ntt_cuda(std::vector<unsigned int, std::allocator<unsigned int> > const&, " \
           "std::vector<unsigned int, std::allocator<unsigned int> > const&)" in demangled
    assert "pidigits::cuda_available()" in demangled


def test_ntt_length_matches_reference_rule():
    lib = oracle.port_lib()
    for na, nb in [(1, 1), (1, 2), (3, 5), (60000, 60000), (1 << 24, 1 << 24), (1 << 24, 1 << 21), (12345, 1)]:
        assert b200mul.ntt_length(na, nb) == lib.orc_ntt_length(na, nb)


def test_workspace_accounting():
    lib = b200mul.lib
    assert lib.b2m_workspace_bytes(0, 5) == 0
    small = lib.b2m_workspace_bytes(100, 100)
    assert 0 < small < 4096
    big = lib.b2m_workspace_bytes(1 << 24, 1 << 24)
    assert big >= 2 * 8 * (1 << 26)  # two N-element u64 transform arrays


def test_status_strings_cover_all_codes():
    for code in b200mul.STATUS:
        s = b200mul.lib.b2m_strerror(code)
        assert s and s != b"unknown status"
    assert b200mul.lib.b2m_strerror(999) == b"unknown status"


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device behaviour")
def test_without_gpu_every_entry_point_reports_instead_of_falling_back():
    assert b200mul.lib.b2m_init(0, 0) == b200mul.NO_DEVICE
    assert not b200mul.cuda_available()
    a = np.ones(4, np.uint32)
    with pytest.raises(b200mul.B2MError) as ei:
        b200mul.mul_ntt_cuda(a, a)
    assert ei.value.status == b200mul.NOT_INITIALIZED
    assert b200mul.lib.b2m_mul_device(None, 1, None, 1, None, 2, None, None) == b200mul.NOT_INITIALIZED
    assert b200mul.lib.b2m_stream_check(None) == b200mul.NOT_INITIALIZED


def test_empty_operand_is_empty_product_without_device():
    # reference: mul_ntt_cuda returns {} for an empty input (src/ntt_cuda.cu:181)
    a = np.ones(3, np.uint32)
    assert b200mul.mul_ntt_cuda(a, np.zeros(0, np.uint32)).size == 0


def test_default_plans_without_device():
    """Default plans (no context, no GPU): the measured power-of-two plan of
    the 2^26-point headline, the radix-3 sub-transform plans where they
    differ from it, and the power-of-two plan where no radix-3 entry exists."""
    d = b200mul.plan_describe(1 << 24, 1 << 24)
    assert (d["three"], d["ntt_log2"], d["logr"]) == (0, 26, [9, 9, 8])
    d = b200mul.plan_describe(3 << 21, 3 << 21)  # 3 * 2^23 points
    assert (d["three"], d["ntt_log2"], d["logr"], d["logc"]) == (1, 23, [9, 6, 8], [3, 6, 4])
    d = b200mul.plan_describe(3 << 19, 3 << 19)  # 3 * 2^21 points
    assert (d["three"], d["ntt_log2"], d["logr"]) == (1, 21, [9, 6, 6])
    d3 = b200mul.plan_describe(3 << 20, 3 << 20)  # 3 * 2^22 points: no radix-3 entry
    d2 = b200mul.plan_describe(1 << 20, 1 << 20)  # 2^22 points
    assert d3["three"] == 1 and d3["ntt_log2"] == d2["ntt_log2"] == 22 and d3["logr"] == d2["logr"]
