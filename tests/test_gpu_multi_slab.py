"""The multi-GPU slab split of every drop-in entry point, exercised on one
device: a GPU list that names the same device two or three times runs one
host thread per entry on its own contiguous z-slab (uneven: 5 slices over 2
or 3 entries), and the result must be bit-identical to the one-entry call --
the per-slice independence the reference's split relies on (fbp.cu:267-301)."""
import numpy as np
import pytest

from helpers import fbp_params, phantom_case, sino_case, temfq_counts

pytestmark = pytest.mark.gpu

LISTS = ([0], [0, 0], [0, 0, 0])


def _g(lst):
    return np.array(lst, np.intc)


def _run_all(fn):
    outs = [fn(_g(lst)) for lst in LISTS]
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    return outs[0]


def test_fbp_lowpass_bst_split():
    from sscRaft.rafttypes import libraft, check_error
    N, A, B = 64, 64, 5
    ang = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    sino, _ = sino_case(N, A, B, seed=41, angles=ang)
    pf, pi = fbp_params(N, A, B, pad=2, ftype=5, offset=1.5)

    def fbp(g):
        obj = np.zeros((B, N, N), np.float32)
        libraft.getFBPMultiGPU(g.ctypes.data, len(g), obj.ctypes.data, sino.ctypes.data, ang.ctypes.data,
                               pf.ctypes.data, pi.ctypes.data)
        check_error("fbp")
        return obj

    def lowpass(g):
        t = sino.copy()
        libraft.getFilterLowPassMultiGPU(g.ctypes.data, len(g), t.ctypes.data, pf.ctypes.data, pi.ctypes.data)
        check_error("lowpass")
        return t

    pfb, pib = fbp_params(N, A, B, pad=2, ftype=5, offset=1.0)

    def bst(g):
        obj = np.zeros((B, N, N), np.float32)
        libraft.getBSTMultiGPU(g.ctypes.data, len(g), obj.ctypes.data, sino.ctypes.data, ang.ctypes.data,
                               pfb.ctypes.data, pib.ctypes.data, 0)
        check_error("bst")
        return obj

    for fn in (fbp, lowpass, bst):
        assert np.abs(_run_all(fn)).max() > 0


def test_radon_em_split():
    from sscRaft.rafttypes import libraft, check_error
    N, A, B = 48, 40, 5
    img = phantom_case(N, B, seed=43, scale=0.02)
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)

    def radon(g):
        out = np.zeros((B, A, N), np.float32)
        libraft.getRadonRTMultiGPU(g.ctypes.data, len(g), out.ctypes.data, img.ctypes.data, ang.ctypes.data,
                                   N, N, N, A, B, 1.0, 1.0)
        check_error("radon")
        return out

    proj = _run_all(radon)
    counts = np.exp(-proj * N / 2).astype(np.float32)
    flat = np.ones((B, N), np.float32)
    pf = np.array([0], np.float32)
    pi = np.array([N, A, B, N, 0, 0, 0, B, 3, 0], np.int32)

    def tem(g):
        obj = np.ones((B, N, N), np.float32)
        c = counts.copy()
        libraft.get_tEM_RT_MultiGPU(g.ctypes.data, len(g), obj.ctypes.data, c.ctypes.data, flat.ctypes.data,
                                    ang.ctypes.data, pf.ctypes.data, pi.ctypes.data)
        check_error("tem")
        return obj

    def eem(g):
        obj = np.ones((B, N, N), np.float32)
        t = proj.copy()
        libraft.get_eEM_RT_MultiGPU(g.ctypes.data, len(g), obj.ctypes.data, t.ctypes.data, ang.ctypes.data,
                                    pf.ctypes.data, pi.ctypes.data)
        check_error("eem")
        return obj

    for fn in (tem, eem):
        assert np.abs(_run_all(fn)).max() > 0


def test_background_axis_temfq_split():
    import sscRaft.processing.alignments.rotationaxis  # noqa: F401  (declares the axis-correction prototype)
    from sscRaft.rafttypes import libraft, check_error
    N, A, B = 64, 64, 5
    rng = np.random.default_rng(45)
    frames = rng.uniform(200, 1000, (B, A, N)).astype(np.float32)
    flat = rng.uniform(1000, 1100, (B, 2, N)).astype(np.float32)
    dark = rng.uniform(50, 100, (B, N)).astype(np.float32)

    def background(g):
        t = frames.copy()
        libraft.getBackgroundCorrectionMultiGPU(g.ctypes.data, len(g), t.ctypes.data, flat.ctypes.data,
                                                dark.ctypes.data, N, A, B, 2, 1, 0)
        check_error("background")
        return t

    sino = _run_all(background)

    def axis(g):
        t = sino.copy()
        libraft.getRotAxisCorrectionMultiGPU(g.ctypes.data, len(g), t.ctypes.data, 1.7, N, A, B, 0)
        check_error("axis")
        return t

    _run_all(axis)
    counts, fl, ang = temfq_counts(N, A, B, 0.02, seed=47)
    pi = np.array([N, A, B, N, 1, 0, 0, B, 2, 1, 0], np.int32)
    pf = np.array([0.02, 0.02, 0.0], np.float32)

    def temfq(g):
        obj = np.ones((B, N, N), np.float32)
        libraft.get_tEM_FQ_MultiGPU(g.ctypes.data, len(g), counts.ctypes.data, obj.ctypes.data, ang.ctypes.data,
                                    fl.ctypes.data, pf.ctypes.data, pi.ctypes.data)
        check_error("temfq")
        return obj

    assert np.abs(_run_all(temfq)).max() > 0
