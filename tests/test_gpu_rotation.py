"""GPU tests of the rotation-axis finders and correction.

findcentersino / findcentersino16: the reference's integer result exactly
(its own outputs in the fixtures, and the FP64 oracle on further frame
pairs); findcentersino_subpixel: within one step (0.005 rays of result) of
the reference's; getRotAxisCorrectionMultiGPU: rel-L2 <= 1e-5 against the
reference's output and the oracle."""
import ctypes
import glob
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(GOLDEN)))


def _fixtures(kind):
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "ref_rot*.npz"))):
        d = np.load(f)
        if str(d["kind"]) == kind:
            out.append((os.path.basename(f), d))
    return out


def test_centersino_vs_reference_fixtures():
    from sscRaft.processing import Centersino, Centersino16, Centersino_subpixel
    cases = _fixtures("centersino")
    assert cases
    for name, d in cases:
        f0, f1, dk, ft = d["frame0"], d["frame180"], d["dark"], d["flat"]
        assert Centersino(f0, f1, ft, dk) == int(d["out"]), name
        assert Centersino16(f0.astype(np.uint16), f1.astype(np.uint16), ft.astype(np.uint16),
                            dk.astype(np.uint16)) == int(d["out16"]), name
        assert abs(Centersino_subpixel(f0, f1, ft, dk) - float(d["out_subpixel"])) <= 0.0051, name


@pytest.mark.parametrize("sizex,sizey,axis", [(320, 128, 150.0), (200, 50, 104.5), (128, 128, 60.0)])
def test_centersino_vs_oracle(oracle, sizex, sizey, axis):
    from sscRaft.processing import Centersino
    from golden.make_golden import frame_pair
    f0, f1, dk, ft = frame_pair(sizex, sizey, axis, seed=sizex + sizey)
    assert Centersino(f0, f1, ft, dk) == oracle.centersino(f0, f1, dk, ft)


def test_centersino_device_entry_matches_host():
    import torch
    from sscRaft.processing import Centersino
    from sscRaft.rafttypes import libraft
    from golden.make_golden import frame_pair
    arrs = frame_pair(256, 64, 120.0, seed=5)
    d = [torch.from_numpy(a).cuda() for a in arrs]
    res = ctypes.c_double(0)
    rc = libraft.raft_centersino_device(0, *[ctypes.c_void_p(t.data_ptr()) for t in d], 256, 64, 0,
                                        ctypes.byref(res), None)
    assert rc == 0 and int(res.value) == Centersino(arrs[0], arrs[1], arrs[3], arrs[2])


def test_rotaxis_correction_vs_reference_and_oracle(oracle):
    from sscRaft.processing import correct_rotation_axis
    cases = _fixtures("rotaxis")
    assert cases
    for name, d in cases:
        for off, key in zip(d["offsets"], ("out_a", "out_b")):
            out = correct_rotation_axis(d["tomo"].copy(), float(off))
            assert rel_l2(out, d[key]) <= 1e-5, (name, off, rel_l2(out, d[key]))
            assert rel_l2(out, oracle.rotaxis(d["tomo"], float(off))) <= 1e-5


@pytest.mark.parametrize("sizex,sizey,axis", [(176, 44, 80.0), (143, 64, 70.5)])
def test_centersino_prime_factor_sizes_vs_oracle(oracle, sizex, sizey, axis):
    # 176 = 16 x 11, 44 = 4 x 11, 143 = 11 x 13: Bluestein transforms
    from sscRaft.processing import Centersino
    from golden.make_golden import frame_pair
    f0, f1, dk, ft = frame_pair(sizex, sizey, axis, seed=sizex + sizey)
    assert Centersino(f0, f1, ft, dk) == oracle.centersino(f0, f1, dk, ft)


def test_centersino_too_long_size_raises():
    from sscRaft.processing import Centersino
    z = np.ones((10, 7919), np.float32)      # 7919 is prime: its transform would not fit shared memory
    with pytest.raises(RuntimeError):
        Centersino(z, z, z, z)
