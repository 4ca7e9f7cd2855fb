"""GPU tests of the flat/dark correction (getBackgroundCorrectionMultiGPU and
raft_background_device).

Tolerances: vs the reference library's own outputs (golden fixtures) and vs
the FP64 oracle, rel-L2 <= 1e-6 (float rounding and the fast division / log
intrinsics both the reference build and this kernel use).  Host and device entry points, single- and multi-chunk pipelines and
pinned / pageable buffers give bit-identical results."""
import ctypes
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu


def _raw(B, A, N, nflats, seed):
    rng = np.random.default_rng(seed)
    flat = rng.uniform(800.0, 1200.0, (B, nflats, N)).astype(np.float32)
    dark = rng.uniform(50.0, 150.0, (B, N)).astype(np.float32)
    frames = (dark[:, None, :] + rng.uniform(-30.0, 1.3, (B, A, N)) * (flat[:, :1, :] - dark[:, None, :]))
    return frames.astype(np.float32), flat, dark


def test_background_vs_reference_fixtures():
    import sscRaft
    files = sorted(glob.glob(os.path.join(GOLDEN, "ref_bg_*.npz")))
    assert files, "flat/dark fixtures missing"
    for f in files:
        d = np.load(f)
        out = sscRaft.correct_background(d["frames"].copy(), d["flat"], d["dark"], gpus=[0],
                                         is_log=bool(int(d["is_log"])))
        assert rel_l2(out, d["out"]) <= 1e-6, (os.path.basename(f), rel_l2(out, d["out"]))


@pytest.mark.parametrize("N,nflats,is_log", [(128, 1, 1), (130, 2, 1), (64, 3, 0), (37, 2, 0)])
def test_background_vs_oracle(oracle, N, nflats, is_log):
    import sscRaft
    frames, flat, dark = _raw(3, 41, N, nflats, seed=N + nflats)
    out = sscRaft.correct_background(frames.copy(), flat, dark, gpus=[0], is_log=bool(is_log))
    ref = oracle.background(frames, flat, dark, is_log)
    assert rel_l2(out, ref) <= 1e-6, rel_l2(out, ref)
    # clamps: frames below the dark give max(T, 0.5) / Q
    low = frames - dark[:, None, :] < 0.5
    assert low.any()


def test_background_pipeline_and_device_entry_agree():
    import torch
    import sscRaft
    from sscRaft.rafttypes import libraft
    B, A, N, nf = 9, 30, 96, 2
    frames, flat, dark = _raw(B, A, N, nf, seed=3)
    whole = sscRaft.correct_background(frames.copy(), flat, dark, gpus=[0], is_log=True)
    chunked = sscRaft.correct_background(frames.copy(), flat, dark, gpus=[0], is_log=True, blocksize=2)
    pinned = torch.from_numpy(frames.copy()).pin_memory()
    sscRaft.correct_background(pinned.numpy(), flat, dark, gpus=[0], is_log=True, blocksize=4)
    assert np.array_equal(whole, chunked) and np.array_equal(whole, pinned.numpy())
    d = torch.from_numpy(frames).cuda()
    d_flat, d_dark = torch.from_numpy(flat).cuda(), torch.from_numpy(dark).cuda()   # held: pointers are passed
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = libraft.raft_background_device(0, p(d), p(d_flat), p(d_dark), N, A, B, nf, 1, None)
    assert rc == 0
    assert np.array_equal(d.cpu().numpy(), whole)
    # two-dimensional frames (one slice)
    one = sscRaft.correct_background(frames[0].copy(), flat[:1], dark[:1], gpus=[0], is_log=True)
    assert np.array_equal(one, whole[0])


def test_background_invalid_arguments_raise():
    from sscRaft.rafttypes import libraft, check_error
    g = np.array([0], np.intc)
    x = np.zeros((1, 2, 4), np.float32)
    libraft.getBackgroundCorrectionMultiGPU(g.ctypes.data, 1, x.ctypes.data, x.ctypes.data, x.ctypes.data,
                                            4, 2, 1, 0, 1, 0)      # zero flats
    with pytest.raises(RuntimeError):
        check_error("background")
