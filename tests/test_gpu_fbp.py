"""GPU parity tests of the FBP path (filter + backprojector) through the C ABI.

Tolerances:
  * nearest-sample operator vs the FP64 oracle given the GPU fast-intrinsic
    sin/cos values (the values the reference's index rule uses): rel-L2 <= 2e-5;
  * vs the reference library's own outputs (golden fixtures): rel-L2 <= 1e-4;
  * linear operator FP32 vs FP64 oracle: rel-L2 <= 1e-5;
  * linear operator BF16 storage vs FP64 oracle: rel-L2 <= 4e-3.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2
from helpers import fbp_params, sino_case

pytestmark = pytest.mark.gpu


def gpu_fbp(sino, angles, pf, pi, operator="nearest", precision="float32"):
    import sscRaft
    from sscRaft.rafttypes import CNICE, _ptr, check_error, libraft, GEOMETRY, STORE
    B, A, N = sino.shape
    No = int(pi[3])
    obj = np.zeros((B, No, No), np.float32)
    s = CNICE(sino.copy())
    g = np.array([0], np.intc)
    ang = CNICE(np.asarray(angles))
    if operator == "nearest":
        libraft.getFBPMultiGPU(_ptr(g), 1, _ptr(obj), _ptr(s), _ptr(ang), _ptr(pf), _ptr(pi))
    else:
        libraft.raft_fbp_ext(_ptr(g), 1, _ptr(obj), _ptr(s), _ptr(ang), _ptr(pf), _ptr(pi),
                             GEOMETRY[operator], STORE[precision])
    check_error("fbp")
    np.testing.assert_array_equal(s, sino)   # input is read-only
    return obj


CASES = [
    # N, A, B, pad, ftype, pixel, offset
    (64, 90, 2, 2, 7, 1.0, 0.0),
    (96, 120, 1, 2, 5, 1.0, 3.5),
    (50, 64, 1, 2, 6, 0.5, 1.25),
    (80, 100, 1, 1, 7, 1.0, 0.0),
    (63, 37, 1, 0, 7, 1.0, 0.0),      # odd N, no padding, A not a multiple of 32
    (130, 33, 1, 2, 3, 1.0, -2.0),    # N not a multiple of the tile
    (61, 20, 1, 2, 7, 1.0, 0.0),      # Np = 183 = 3 * 61: direct-convolution filter
    (256, 180, 1, 2, 7, 1.0, 0.0),
]


@pytest.mark.parametrize("case", CASES)
def test_fbp_nearest_vs_oracle(case, oracle):
    N, A, B, pad, ftype, pixel, offset = case
    sino, ang = sino_case(N, A, B, seed=N + A, pixel=pixel)
    pf, pi = fbp_params(N, A, B, pad=pad, ftype=ftype, pixel=pixel, offset=offset)
    out = gpu_fbp(sino, ang, pf, pi)
    from sscRaft.rafttypes import fast_sincos
    ref = oracle.fbp(sino, ang, oracle.MODE_REF, ftype, pad, offset=offset, pixel=pixel,
                     trig=fast_sincos(ang, 0))
    assert np.all(np.isfinite(out))
    assert rel_l2(out, ref) <= 2e-5, rel_l2(out, ref)


@pytest.mark.parametrize("case", CASES[:6])
@pytest.mark.parametrize("ftype", [7, 5, 9])
def test_fbp_linear_fp32_vs_oracle(case, ftype, oracle):
    N, A, B, pad, _, pixel, offset = case
    sino, ang = sino_case(N, A, B, seed=N + 2 * A, pixel=pixel)
    pf, pi = fbp_params(N, A, B, pad=pad, ftype=ftype, pixel=pixel, offset=offset)
    out = gpu_fbp(sino, ang, pf, pi, operator="linear")
    ref = oracle.fbp(sino, ang, oracle.MODE_LIN, ftype, pad, offset=offset, pixel=pixel)
    assert rel_l2(out, ref) <= 1e-5, rel_l2(out, ref)


@pytest.mark.parametrize("case", CASES[:4])
def test_fbp_linear_bf16_vs_oracle(case, oracle):
    N, A, B, pad, ftype, pixel, offset = case
    sino, ang = sino_case(N, A, B, seed=N + 3 * A, pixel=pixel)
    pf, pi = fbp_params(N, A, B, pad=pad, ftype=ftype, pixel=pixel, offset=offset)
    out = gpu_fbp(sino, ang, pf, pi, operator="linear", precision="bfloat16")
    ref = oracle.fbp(sino, ang, oracle.MODE_LIN, ftype, pad, offset=offset, pixel=pixel)
    assert rel_l2(out, ref) <= 4e-3, rel_l2(out, ref)


def _golden(kind):
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz"))):
        d = np.load(f)
        if str(d["kind"]) == kind:
            out.append((os.path.basename(f), d))
    return out


def test_fbp_vs_reference_library_fixtures():
    cases = _golden("fbp")
    if not cases:
        pytest.skip("no golden fixtures")
    for name, d in cases:
        out = gpu_fbp(d["sino"], d["angles"], d["paramf"], d["parami"])
        err = rel_l2(out, d["out"])
        assert err <= 1e-4, (name, err)


def test_nearest_index_rule_bit_exact():
    """The reference's own outputs on index-encoded sinograms: every pixel's
    chosen detector bin must be identical."""
    cases = _golden("index_probe")
    if not cases:
        pytest.skip("no golden fixtures")
    for name, d in cases:
        N, pad, pixel = int(d["N"]), int(d["pad"]), float(d["pixel"])
        off = (pad * N) // 2
        for t, th in enumerate(d["thetas"]):
            ang = np.array([th, th + 2.0 ** -10], np.float32)
            sino = np.zeros((1, 2, N), np.float32)
            sino[0, 0, :] = np.arange(N, dtype=np.float32) + off
            pf, pi = fbp_params(N, 2, 1, pad=pad, ftype=0, pixel=pixel)
            out = gpu_fbp(sino, ang, pf, pi)[0]
            mism = int(np.count_nonzero(out != d["out"][t]))
            assert mism == 0, (name, float(th), mism)


def test_fbp_multi_chunk_and_determinism():
    N, A, B = 96, 60, 7
    sino, ang = sino_case(N, A, B, seed=5)
    pf, pi = fbp_params(N, A, B, blocksize=3)
    a = gpu_fbp(sino, ang, pf, pi)
    pf2, pi2 = fbp_params(N, A, B, blocksize=0)
    b = gpu_fbp(sino, ang, pf2, pi2)
    np.testing.assert_array_equal(a, b)
    # slice-by-slice equals batched (slices are independent)
    for k in (0, 6):
        pf1, pi1 = fbp_params(N, A, 1)
        c = gpu_fbp(sino[k:k + 1], ang, pf1, pi1)
        np.testing.assert_array_equal(c[0], a[k])


def test_fbp_empty_and_errors():
    import sscRaft
    sino = np.zeros((0, 10, 16), np.float32)
    pf, pi = fbp_params(16, 10, 0)
    out = gpu_fbp(sino, np.linspace(0, np.pi, 10, endpoint=False).astype(np.float32), pf, pi)
    assert out.shape == (0, 16, 16)
    with pytest.raises(RuntimeError):
        sscRaft.fbp(np.zeros((1, 10, 16), np.float32),
                    dic={"gpu": [99], "angles[rad]": np.zeros(10, np.float32)})


def test_lowpass_vs_oracle_and_reference(oracle):
    import sscRaft
    sino, ang = sino_case(64, 30, 2, seed=300)
    t = sino.copy()
    out = sscRaft.lowpass(t, dic={"gpu": [0], "filter": "hann", "padding": 2})
    assert out is t                          # in place, as the reference
    ref = oracle.lowpass(sino, oracle.MODE_REF, 5, 2)
    assert rel_l2(out, ref) <= 1e-5, rel_l2(out, ref)
    for name, d in _golden("lowpass"):
        t = d["sino"].copy()
        pf, pi = d["paramf"], d["parami"]
        from sscRaft.rafttypes import _ptr, check_error, libraft
        g = np.array([0], np.intc)
        libraft.getFilterLowPassMultiGPU(_ptr(g), 1, _ptr(t), _ptr(pf), _ptr(pi))
        check_error("lowpass")
        assert rel_l2(t, d["out"]) <= 1e-4, (name, rel_l2(t, d["out"]))


def test_public_fbp_api(oracle):
    import sscRaft
    sino, ang = sino_case(64, 90, 1, seed=11)
    out = sscRaft.fbp(sino.copy(), dic={"gpu": [0], "angles[rad]": ang, "filter": "hann",
                                        "rotation axis offset": 1.5})
    from sscRaft.rafttypes import fast_sincos
    ref = oracle.fbp(sino, ang, oracle.MODE_REF, 5, 2, offset=1.5, trig=fast_sincos(ang, 0))
    assert rel_l2(out, ref) <= 2e-5
    lin = sscRaft.fbp(sino.copy(), dic={"gpu": [0], "angles[rad]": ang, "filter": "shepp-logan",
                                        "operator": "linear", "precision": "bfloat16"})
    ref = oracle.fbp(sino, ang, oracle.MODE_LIN, 9, 2)
    assert rel_l2(lin, ref) <= 4e-3
