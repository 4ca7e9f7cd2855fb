"""Failure detection without a GPU fault.

* A device-side wait on a barrier that nothing arrives on (the staging
  pipelines' bounded mbarrier wait) runs out after its poll limit, reports
  through the library's flag, and the context stays usable: an FBP right
  after it gives the same image as before.
* Injected allocation refusals: the call that meets one raises through the
  Python layer (the reference would exit the process), the next call
  succeeds with the right result; a refusal inside a multi-GPU split
  (same device twice) is reported as well."""
import numpy as np
import pytest

from helpers import fbp_params, sino_case

pytestmark = pytest.mark.gpu


def _fbp(sino, ang, gpus=(0,)):
    from sscRaft.rafttypes import libraft, check_error
    B, A, N = sino.shape
    pf, pi = fbp_params(N, A, B, pad=2, ftype=5)
    obj = np.zeros((B, N, N), np.float32)
    g = np.array(gpus, np.intc)
    libraft.getFBPMultiGPU(g.ctypes.data, len(g), obj.ctypes.data, sino.ctypes.data, ang.ctypes.data,
                           pf.ctypes.data, pi.ctypes.data)
    check_error("fbp")
    return obj


def test_bounded_wait_runs_out_and_context_survives():
    from sscRaft.rafttypes import libraft
    sino, ang = sino_case(64, 60, 2, seed=61)
    before = _fbp(sino, ang)
    assert libraft.raft_selftest_bounded_wait(0, 1, 1 << 10) == 0     # arrived: the wait completes
    assert libraft.raft_selftest_bounded_wait(0, 0, 1 << 12) == 1     # never arrived: runs out, reported
    after = _fbp(sino, ang)
    assert np.array_equal(before, after)


def test_injected_allocation_failure_raises_then_recovers():
    from sscRaft.rafttypes import libraft
    sino, ang = sino_case(72, 50, 3, seed=62)
    ref = _fbp(sino, ang)
    big, bang = sino_case(112, 70, 3, seed=63)
    libraft.raft_inject_alloc_failures(1)
    try:
        with pytest.raises(RuntimeError, match="refused"):
            _fbp(big, bang)
    finally:
        libraft.raft_inject_alloc_failures(0)
    out = _fbp(big, bang)                     # recovers
    assert np.abs(out).max() > 0
    assert np.array_equal(_fbp(sino, ang), ref)
    libraft.raft_inject_alloc_failures(1)
    try:
        bigger, bgang = sino_case(136, 40, 5, seed=64)
        with pytest.raises(RuntimeError, match="refused"):
            _fbp(bigger, bgang, gpus=(0, 0))
    finally:
        libraft.raft_inject_alloc_failures(0)
    assert np.abs(_fbp(bigger, bgang, gpus=(0, 0))).max() > 0
