"""CPU tests of the Python drop-in layer (sscRaft): the packed parameter
arrays it hands to the C ABI match the reference wrappers
(sscRaft/geometries/parallel/fbp_methods.py:86-95, em_methods.py:55-65,136-145,
radon_methods.py:42-58, processing/filters.py:75-87,
processing/background_correction.py:6-106 of cnpem/ssc-raft).
The library is replaced by a recording fake; no GPU is touched."""
import ctypes

import numpy as np
import pytest


class Fake:
    def __init__(self, real):
        self.real = real
        self.calls = []

    def __getattr__(self, name):
        if name.startswith("raft_last_error") or name.startswith("raft_clear"):
            return getattr(self.real, name)

        def rec(*args):
            self.calls.append((name, args))
            if name == "getRadonRTMultiGPU":       # write ones into the output
                nr, na, ns = args[7], args[8], args[9]
                out = np.ctypeslib.as_array(ctypes.cast(args[2], ctypes.POINTER(ctypes.c_float)),
                                            shape=(ns * na * nr,))
                out[:] = 1.0
            return 0
        return rec


def arr(p, n, ct):
    return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ct)), shape=(n,)).copy()


@pytest.fixture
def fake(monkeypatch):
    import sscRaft
    from sscRaft.geometries.parallel import fbp_methods, em_methods, radon_methods
    from sscRaft.processing import filters, background_correction
    f = Fake(sscRaft.rafttypes.libraft)
    for m in (fbp_methods, em_methods, radon_methods, filters, background_correction):
        monkeypatch.setattr(m, "libraft", f)
    sscRaft.rafttypes.libraft.raft_clear_error()
    return f


def test_fbp_packing(fake):
    import sscRaft
    t = np.zeros((3, 10, 16), np.float32)
    ang = np.linspace(0, np.pi, 10, endpoint=False)
    out = sscRaft.fbp(t, dic={"gpu": [1], "angles[rad]": ang, "filter": "hann", "rotation axis offset": 3.5,
                              "beta/delta": 0.5, "z2[m]": 2.0, "energy[eV]": 100.0, "detectorPixel[m]": 1e-6})
    name, a = fake.calls[-1]
    assert name == "getFBPMultiGPU"
    assert out.shape == (3, 16, 16) and out.dtype == np.float32
    pi = arr(a[6], 10, ctypes.c_int32)
    pf = arr(a[5], 7, ctypes.c_float)
    assert list(pi) == [16, 10, 3, 16, 2, 0, 0, 5, 0, 0]
    np.testing.assert_allclose(pf, [2.0, 0.0, 100.0, 2.0, 1e-6, 1e-6, 3.5], rtol=1e-6)
    assert arr(a[0], 1, ctypes.c_int32)[0] == 1 and a[1] == 1


def test_fbp_defaults_and_filter_names(fake):
    import sscRaft
    from sscRaft.rafttypes import FilterNumber
    assert [FilterNumber(n) for n in ("none", "gaussian", "lorentz", "cosine", "rectangle", "hann",
                                      "hamming", "ramp", "bogus", "Shepp-Logan")] == [0, 1, 2, 3, 4, 5, 6, 7, 6, 9]
    t = np.zeros((10, 16), np.float64)            # 2-D input, non-float32
    sscRaft.fbp(t, dic={"gpu": [0], "angles[rad]": np.zeros(10)})
    name, a = fake.calls[-1]
    pi = arr(a[6], 10, ctypes.c_int32)
    pf = arr(a[5], 7, ctypes.c_float)
    assert list(pi) == [16, 10, 1, 16, 2, 0, 0, 7, 0, 0]      # ramp, padding 2
    np.testing.assert_allclose(pf, [0, 0, 1, 0, 1, 1, 0])      # beta/delta 0 -> z2 0, energy 1
    with pytest.raises(ValueError):
        sscRaft.fbp(t, dic={"angles[rad]": np.zeros(10)})     # 'gpu' is required
    # BST: the reference packing (bstGPU, fbp_methods.py:152-201), offset truncated to an integer
    sscRaft.fbp(np.zeros((2, 10, 16), np.float32), dic={"gpu": [0], "method": "BST", "filter": "hann",
                                                         "rotation axis offset": 2.7, "padding": 1})
    name, a = fake.calls[-1]
    assert name == "getBSTMultiGPU" and a[7] == 0
    assert list(arr(a[6], 10, ctypes.c_int32)) == [16, 10, 2, 16, 1, 0, 0, 5, 0, 0]
    np.testing.assert_allclose(arr(a[5], 7, ctypes.c_float), [0, 0, 1, 0, 1, 1, 2.0])
    np.testing.assert_allclose(arr(a[4], 10, ctypes.c_float), np.linspace(0, np.pi, 10, endpoint=False), rtol=1e-6)


def test_fbp_extension_keys(fake):
    import sscRaft
    t = np.zeros((2, 10, 16), np.float32)
    sscRaft.fbp(t, dic={"gpu": [0], "angles[rad]": np.zeros(10), "operator": "linear", "precision": "bfloat16",
                        "filter": "shepp-logan"})
    name, a = fake.calls[-1]
    assert name == "raft_fbp_ext" and a[7] == 1 and a[8] == 2
    with pytest.raises(ValueError):
        sscRaft.fbp(t, dic={"gpu": [0], "angles[rad]": np.zeros(10), "precision": "bfloat16"})


def test_tem_packing_and_inplace_counts(fake):
    import sscRaft
    data = np.full((2, 6, 8), 0.5, np.float32)
    ang = np.linspace(0, np.pi, 6, endpoint=False)
    obj = sscRaft.em(data, angles=ang, dic={"gpu": [0], "method": "tEMRT", "iterations": 7, "blocksize": 3})
    name, a = fake.calls[-1]
    assert name == "get_tEM_RT_MultiGPU"
    np.testing.assert_allclose(data, np.exp(-0.5), rtol=1e-6)     # overwritten, as em_methods.py:109
    pi = arr(a[7], 10, ctypes.c_int32)
    assert list(pi) == [8, 6, 2, 8, 0, 0, 0, 2, 7, 3]
    assert obj.shape == (2, 8, 8) and np.all(obj == 1)
    flat = arr(a[4], 16, ctypes.c_float)
    assert np.all(flat == 1)


def test_temfq_packing(fake):
    # tEMFQ_GPU_ packing (em_methods.py:154-232 of the reference): parami of 11,
    # paramf [pixel x, pixel y, 0 (total variation off)], padding from the dictionary
    import sscRaft
    data = np.full((2, 6, 8), 100.0, np.float32)
    obj = sscRaft.em(data, angles=np.linspace(0, np.pi, 6, endpoint=False),
                     dic={"gpu": [0], "method": "tEMFQ", "iterations": 5, "padding": 1,
                          "interpolation": "nearest", "detectorPixel[m]": 2e-6})
    name, a = fake.calls[-1]
    assert name == "get_tEM_FQ_MultiGPU"
    assert list(arr(a[7], 11, ctypes.c_int32)) == [8, 6, 2, 8, 1, 0, 0, 1, 5, 0, 0]   # nflats 1 for a 2-D flat
    np.testing.assert_allclose(arr(a[6], 3, ctypes.c_float), [2e-6, 2e-6, 0.0])
    assert np.all(arr(a[5], 16, ctypes.c_float) == 1)                 # default flat: ones per slice
    assert np.all(arr(a[2], 96, ctypes.c_float) == 100)                # counts as given (no -log)
    assert obj.shape == (2, 8, 8) and np.all(obj == 1)                 # default initial guess: ones
    sscRaft.em(data, flat=np.full(8, 7.0), angles=np.zeros(6), dic={"gpu": [0], "method": "tEMFQ"})
    name, a = fake.calls[-1]
    assert np.all(arr(a[5], 16, ctypes.c_float) == 7)                 # one flat row serves both slices
    assert list(arr(a[7], 11, ctypes.c_int32))[4] == 2                 # default padding 2, bilinear
    assert list(arr(a[7], 11, ctypes.c_int32))[9] == 1
    with pytest.raises(ValueError):
        sscRaft.em(data, flat=np.ones((3, 8)), angles=np.zeros(6), dic={"gpu": [0], "method": "tEMFQ"})


def test_eem_packing(fake):
    import sscRaft
    data = np.ones((6, 8), np.float32)
    guess = np.full((1, 8, 8), 2.0, np.float32)
    obj = sscRaft.em(data, angles=np.zeros(6), obj=guess, dic={"gpu": [0], "method": "eEMRT"})
    name, a = fake.calls[-1]
    assert name == "get_eEM_RT_MultiGPU"
    assert list(arr(a[6], 10, ctypes.c_int32)) == [8, 6, 1, 8, 0, 0, 0, 1, 10, 0]   # default 10 iterations
    assert obj is guess                                                                # in/out initial guess
    with pytest.raises(ValueError):
        sscRaft.em(data, angles=np.zeros(6), dic={"gpu": [0], "method": "nope"})


def test_radon_scaling(fake):
    import sscRaft
    out = sscRaft.radon_RT(np.zeros((2, 12, 12), np.float32), np.zeros(5), [0], pixel=0.25)
    name, a = fake.calls[-1]
    assert name == "getRadonRTMultiGPU" and a[5:10] == (12, 12, 12, 5, 2)
    np.testing.assert_allclose(out, 12 * 0.25 / 2)


def test_lowpass_inplace(fake):
    import sscRaft
    t = np.zeros((2, 5, 16), np.float32)
    out = sscRaft.lowpass(t, dic={"gpu": [0], "filter": "hamming", "padding": 1})
    name, a = fake.calls[-1]
    assert out is t and name == "getFilterLowPassMultiGPU"
    assert list(arr(a[4], 10, ctypes.c_int32)) == [16, 5, 2, 16, 1, 0, 0, 6, 0, 0]
    assert arr(a[3], 7, ctypes.c_float)[6] == 0.0      # axis offset forced to 0


def test_background_packing_and_layouts(fake):
    import sscRaft
    fr = np.zeros((3, 7, 16), np.float32)
    fl = np.ones((3, 2, 16), np.float32)
    dk = np.zeros((3, 1, 16), np.float32)               # [slices, 1, rays] is accepted
    out = sscRaft.correct_background(fr, fl, dk, gpus=[0], is_log=True, blocksize=4)
    name, a = fake.calls[-1]
    assert out is fr and name == "getBackgroundCorrectionMultiGPU"
    assert a[5:] == (16, 7, 3, 2, 1, 4)
    # correct_projections takes [angles, slices, rays] and returns [slices, angles, rays]
    raw = np.zeros((7, 3, 16), np.float32)
    out = sscRaft.correct_projections(raw, np.ones((1, 3, 16), np.float32), np.zeros((1, 3, 16), np.float32),
                                      {"gpu": [0], "uselog": False})
    name, a = fake.calls[-1]
    assert out.shape == (3, 7, 16) and a[5:] == (16, 7, 3, 1, 0, 0)


def test_background_shape_errors(fake):
    import sscRaft
    fr = np.zeros((3, 7, 16), np.float32)
    with pytest.raises(ValueError):
        sscRaft.correct_background(fr, np.ones((2, 1, 16), np.float32), np.zeros((3, 16), np.float32))
    with pytest.raises(ValueError):
        sscRaft.correct_background(fr, np.ones((3, 1, 16), np.float32), np.zeros((3, 15), np.float32))
    with pytest.raises(ValueError):
        sscRaft.correct_background(np.zeros((1, 3, 7, 16), np.float32), np.ones((3, 1, 16), np.float32),
                                   np.zeros((3, 16), np.float32))
    assert not [c for c in fake.calls if c[0] == "getBackgroundCorrectionMultiGPU"]
