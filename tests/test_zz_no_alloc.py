"""GPU test of raft_fbp_device_noalloc, the FBP entry point that allocates no
device memory (for callers that cannot allocate while reconstructing: a scan
pipeline that reserved the GPU's memory up front, or a host application whose
own allocator owns the device memory).

Two calls of the new entry point in a row, with different sizes and
operators, each must give exactly the image of the existing entry point
(raft_fbp_device) on the same inputs: every launch shape and row layout of
the backprojector sums a pixel's angles in the same order, so the results
are bit-identical.  Both calls run while the library refuses every
device-buffer request (raft_inject_alloc_failures), and a repeat of them
leaves the device's free memory unchanged.  An over-sized request is refused
with a clear message before any work is issued.  This file is collected last
on purpose."""
import ctypes

import numpy as np
import pytest

from helpers import fbp_params, sino_case

pytestmark = pytest.mark.gpu


def _run(fn, d_sino, ang, pf, pi, geometry, store, out=None):
    import torch
    from sscRaft.rafttypes import _ptr, check_error
    B, A, N = d_sino.shape
    No = int(pi[3])
    if out is None:
        out = torch.full((B, No, No), float("nan"), dtype=torch.float32, device="cuda")
    rc = fn(0, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(d_sino.data_ptr()), _ptr(ang), _ptr(pf),
            _ptr(pi), geometry, store, None)
    if rc:
        check_error("fbp")
    torch.cuda.synchronize()
    return out.cpu().numpy()


CASES = [
    # N, A, B, pad, filter, offset, geometry, store
    (256, 180, 3, 2, 5, 1.5, 0, 0),     # nearest (reference rule), Hann, axis offset
    (200, 150, 2, 1, 7, 0.0, 1, 1),     # linear, FP32 pairs, ramp
]


def test_noalloc_matches_existing_entry_point_on_two_calls_in_a_row():
    import torch
    from sscRaft.rafttypes import libraft
    inputs = []
    for N, A, B, pad, ftype, offset, g, s in CASES:
        sino, ang = sino_case(N, A, B, seed=N + A)
        pf, pi = fbp_params(N, A, B, pad=pad, ftype=ftype, offset=offset)
        inputs.append((torch.from_numpy(sino).cuda(), np.ascontiguousarray(ang), pf, pi, g, s))
    # the new entry point, twice in a row, while every device-buffer request
    # of the library is refused
    libraft.raft_inject_alloc_failures(1 << 20)
    try:
        new = [_run(libraft.raft_fbp_device_noalloc, *x) for x in inputs]
    finally:
        libraft.raft_inject_alloc_failures(0)
    # the existing entry point on the same inputs
    old = [_run(libraft.raft_fbp_device, *x) for x in inputs]
    for a, b in zip(new, old):
        assert np.all(np.isfinite(a))
        np.testing.assert_array_equal(a, b)
    # the same two calls again into outputs made beforehand: the device's
    # free memory does not move
    outs = [torch.full((int(x[3][2]), int(x[3][3]), int(x[3][3])), float("nan"), device="cuda") for x in inputs]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for x, o in zip(inputs, outs):
        _run(libraft.raft_fbp_device_noalloc, *x, out=o)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    for o, b in zip(outs, old):
        np.testing.assert_array_equal(o.cpu().numpy(), b)


def test_noalloc_refuses_oversized_requests():
    import torch
    from sscRaft.rafttypes import libraft, _ptr
    N, A, B = 2048, 3600, 1            # linear FP32 rows of one slice alone exceed 64 MiB
    pf, pi = fbp_params(N, A, B)
    d = torch.zeros((1, 1), dtype=torch.float32, device="cuda")
    ang = np.zeros(A, np.float32)
    rc = libraft.raft_fbp_device_noalloc(0, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                         _ptr(ang), _ptr(pf), _ptr(pi), 1, 1, None)
    assert rc == 1
    buf = ctypes.create_string_buffer(512)
    assert libraft.raft_last_error(buf, 512) == 1
    assert b"64 MiB" in buf.value
