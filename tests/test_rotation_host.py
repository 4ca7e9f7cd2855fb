"""CPU tests of the rotation-axis host helpers (no GPU): correctRotationAxis
(the integer shift in the C ABI) and the numpy helpers of
sscRaft.processing.alignments.rotationaxis, against direct numpy statements
of the reference's behaviour (rotationaxis.py:82-400 of cnpem/ssc-raft)."""
import numpy as np


def test_correct_rotation_axis_host_shift():
    from sscRaft.processing import c_correct_rotation_axis
    rng = np.random.default_rng(0)
    d = rng.random((2, 3, 10)).astype(np.float32)
    for dev in (3, -4, 0, 12, -12):
        out = c_correct_rotation_axis(d, dev)
        ref = np.zeros_like(d)
        if dev > 0:
            ref[..., dev:] = d[..., :max(0, 10 - dev)] if dev < 10 else 0
        elif dev < 0:
            ref[..., :10 + dev] = d[..., -dev:] if -dev < 10 else 0
        else:
            ref = out                      # the reference leaves the output untouched for 0
        assert np.array_equal(out, ref), dev
    inplace = d.copy()
    c_correct_rotation_axis(inplace, 2, out=inplace)
    assert np.array_equal(inplace[..., 2:], d[..., :-2]) and not inplace[..., :2].any()


def test_numpy_helpers():
    from sscRaft.processing import (correct_rotation_axis_cropped, correct_rotation_axis_int,
                                    correct_rotation_axis360, find_rotation_axis_360)
    d = np.arange(2 * 3 * 8, dtype=np.float64).reshape(2, 3, 8)
    c = correct_rotation_axis_cropped(d.copy(), 2)
    assert np.array_equal(c[..., 2:], d[..., :-2]) and not c[..., :2].any()
    w = correct_rotation_axis_int(d, 3)        # -3 after the sign fix: data placed at the right
    assert w.shape == (2, 3, 14) and np.array_equal(w[..., 6:], d)
    # a symmetric 360-degree sinogram whose axis sits 3 rays right of the middle
    nth, nz, nx = 40, 4, 64
    x = np.arange(nx)
    axis = nx // 2 + 3
    rows = np.exp(-((x - axis - 6.0) ** 2) / 20.0)[None, :] * np.linspace(1, 2, nth // 2)[:, None]
    mirrored = np.array([np.interp(2 * axis - x, x, r) for r in rows])
    tomo = np.zeros((nth, nz, nx))
    tomo[:nth // 2] = rows[:, None, :]
    tomo[nth // 2:] = mirrored[:, None, :]
    dev = find_rotation_axis_360(tomo, nx_search=8, nx_window=12, nsinos=1)
    assert abs(dev - 3) <= 1
    proj, shift = correct_rotation_axis360(np.swapaxes(tomo, 0, 1), {"shift": (False, 3),
                                                                     "findRotationAxis": (8, 12, 1)})
    assert shift == 3 and proj.shape == (nz, nth, nx + 6)
