"""GPU tests of the drop-in: the reference's own front-ends, built from the
reference sources with the B200 shim linked in place of src/ntt_cuda.cu
(oracle/Makefile target `dropin`), run unchanged on this backend.

* pi_selftest_b200 is the reference's tests/self_test.cu: field algebra, the
  120 multiply pairs (mul_ntt_cuda == schoolbook), division/sqrt/decimal,
  Chudnovsky digits with Auto and with NttCuda forced (:103-122), BBP.
* pi_b200 is the reference's CLI (src/main.cpp) with `--backend ntt-cuda`:
  every multiply of the binary-splitting tree goes through the shim; its
  digits must equal the reference's CPU run (tests/golden/pi_digits.json).
"""
import hashlib
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
SELFTEST = os.path.join(REF, "pi_selftest_b200")
CLI = os.path.join(REF, "pi_b200")


@pytest.mark.skipif(not os.path.exists(SELFTEST), reason="drop-in build needs the reference tree")
def test_reference_selftest_runs_on_b200_backend():
    r = subprocess.run([SELFTEST], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "cuda_available = yes" in r.stdout
    assert " 0 failed" in r.stdout and "ALL TESTS PASSED" in r.stdout


@pytest.mark.skipif(not os.path.exists(CLI), reason="drop-in build needs the reference tree")
@pytest.mark.parametrize("digits", [10000, 100000])
def test_reference_cli_digits_with_ntt_cuda_backend(tmp_path, digits):
    runs = json.load(open(os.path.join(ROOT, "tests", "golden", "pi_digits.json")))["runs"]
    want = [r for r in runs if r["digits"] == digits][0]
    out = tmp_path / "pi.txt"
    r = subprocess.run([CLI, "--backend", "ntt-cuda", "--digits", str(digits), "--out", str(out), "--quiet"],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    got = out.read_text().rstrip("\n")
    assert got[:102] == want["head"]
    assert hashlib.sha256(got.encode()).hexdigest() == want["sha256"]


def test_bounded_device_wait_reports_timeout_and_context_survives(b2m_gpu):
    """Failure detection without a fault: a carry block waits on a predecessor
    that never publishes; the bounded wait gives up, the call reports
    B2M_ERR_DEVICE_TIMEOUT, and the next product on the same context is exact."""
    import time

    import numpy as np

    import oracle

    t0 = time.perf_counter()
    assert b2m_gpu.selftest_wait_timeout() == 8  # B2M_ERR_DEVICE_TIMEOUT
    assert time.perf_counter() - t0 < 30
    b2m_gpu.stream_check(0)  # the error word was read and cleared
    a = np.arange(1, 5001, dtype=np.uint32)
    b = np.arange(7, 3007, dtype=np.uint32)
    assert np.array_equal(b2m_gpu.mul_ntt_cuda(a, b), oracle.mul_port(a, b))
