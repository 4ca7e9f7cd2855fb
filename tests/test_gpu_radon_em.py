"""GPU parity tests of the Radon projector and the EM iterations.

Tolerances: vs the reference library's own outputs (golden fixtures)
rel-L2 <= 1e-4.  Vs the FP64 oracle given the GPU fast-intrinsic sin/cos
values (the values the reference's index rules use): Radon rel-L2 <= 2e-5;
tEM <= 1e-3 and eEM <= 2e-2, where the EM grid puts many samples exactly on
pixel boundaries and the (reference's and this library's) fast division
decides the bin, which the oracle does not restate.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2
from helpers import phantom_case

pytestmark = pytest.mark.gpu


def _golden(kind):
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz"))):
        d = np.load(f)
        if str(d["kind"]) == kind:
            out.append((os.path.basename(f), d))
    return out


def F(ang):
    from sscRaft.rafttypes import fast_sincos
    return fast_sincos(ang, 0)


def B(ang):
    from sscRaft.rafttypes import fast_sincos
    return fast_sincos(ang, 1)


def test_radon_vs_oracle(oracle):
    import sscRaft
    img = phantom_case(64, 2, seed=3)
    ang = (np.arange(90) * (np.pi / 90)).astype(np.float32)
    out = sscRaft.radon_RT(img, ang, [0], pixel=1.0)
    ref = oracle.radon_rt(img, ang, trig=F(ang)) * 64 / 2
    assert rel_l2(out, ref) <= 2e-5, rel_l2(out, ref)
    img = phantom_case(100, 1, seed=4)
    ang = (np.arange(45) * (np.pi / 45)).astype(np.float32)
    out = sscRaft.radon_RT(img, ang, [0], pixel=0.5)
    ref = oracle.radon_rt(img, ang, trig=F(ang)) * 100 * 0.5 / 2
    assert rel_l2(out, ref) <= 2e-5, rel_l2(out, ref)


def test_radon_vs_reference_fixture():
    import sscRaft
    for name, d in _golden("radon"):
        out = sscRaft.radon_RT(d["img"], d["angles"], [0]) / (d["img"].shape[2] / 2)
        assert rel_l2(out, d["out"]) <= 1e-4, (name, rel_l2(out, d["out"]))


def _transmission(N, A, B, seed, oracle):
    img = phantom_case(N, B, seed=seed, scale=0.02)
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    p = oracle.em_forward(img.astype(np.float64), ang, N)
    return p.astype(np.float32), ang


def test_tem_vs_oracle(oracle):
    import sscRaft
    data, ang = _transmission(48, 36, 2, 21, oracle)
    flat = np.ones((2, 48), np.float32)
    out = sscRaft.em(data.copy(), flat=flat, angles=ang,
                     dic={"gpu": [0], "method": "tEMRT", "iterations": 3})
    ref = oracle.tem(np.exp(-data).astype(np.float32), flat, ang, 3, fwd_trig=F(ang), bp_trig=B(ang))
    assert rel_l2(out, ref) <= 1e-3, rel_l2(out, ref)


def test_eem_vs_oracle(oracle):
    import sscRaft
    img = phantom_case(48, 2, seed=31)
    ang = (np.arange(40) * (np.pi / 40)).astype(np.float32)
    tomo = oracle.em_forward(img.astype(np.float64), ang, 48).astype(np.float32)
    out = sscRaft.em(tomo.copy(), angles=ang, dic={"gpu": [0], "method": "eEMRT", "iterations": 4})
    ref = oracle.eem(tomo, ang, 4, fwd_trig=F(ang), bp_trig=B(ang))
    assert rel_l2(out, ref) <= 2e-2, rel_l2(out, ref)


def test_em_vs_reference_fixtures():
    import sscRaft
    from sscRaft.geometries.parallel.em_methods import em_with_metrics
    for name, d in _golden("tem"):
        obj, _ = em_with_metrics("tEM", d["counts"], d["angles"], int(d["iterations"]), flat=d["flat"])
        assert rel_l2(obj, d["out"]) <= 1e-4, (name, rel_l2(obj, d["out"]))
    for name, d in _golden("eem"):
        obj = sscRaft.em(d["tomo"].copy(), angles=d["angles"],
                         dic={"gpu": [0], "method": "eEMRT", "iterations": int(d["iterations"])})
        assert rel_l2(obj, d["out"]) <= 1e-4, (name, rel_l2(obj, d["out"]))


def test_em_graph_equals_stream_and_metrics(oracle):
    from sscRaft.geometries.parallel.em_methods import em_with_metrics
    data, ang = _transmission(40, 30, 2, 41, oracle)
    counts = np.exp(-data).astype(np.float32)
    a, ma = em_with_metrics("tEM", counts, ang, 5, use_graph=True)
    b, mb = em_with_metrics("tEM", counts, ang, 5, use_graph=False)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(ma, mb, rtol=1e-12)
    # metrics of the iterate entering iteration k vs the oracle's restatement
    x = np.ones((2, 40, 40))
    flat = np.ones((2, 40), np.float32)
    for k in range(3):
        res, nll = oracle.tem_metrics(counts, flat, ang, x, fwd_trig=F(ang))
        got_res = np.sqrt(ma[k, :, 0]) / np.sqrt(ma[k, :, 1])
        np.testing.assert_allclose(got_res, res, rtol=2e-3)
        np.testing.assert_allclose(ma[k, :, 2], nll, rtol=1e-5)
        x = oracle.tem(counts, flat, ang, 1, obj=x, fwd_trig=F(ang), bp_trig=B(ang))


@pytest.fixture
def pj_order(request):
    old = os.environ.get("RAFT_PJ_SEQUENTIAL")
    if request.param:
        os.environ["RAFT_PJ_SEQUENTIAL"] = "1"
    else:
        os.environ.pop("RAFT_PJ_SEQUENTIAL", None)
    yield request.param
    if old is None:
        os.environ.pop("RAFT_PJ_SEQUENTIAL", None)
    else:
        os.environ["RAFT_PJ_SEQUENTIAL"] = old


@pytest.mark.parametrize("pj_order", [False, True], indirect=True, ids=["phases", "sequential"])
def test_interleaved_projector_bit_identical(pj_order):
    """8 or more slices run the projector on slice-interleaved copies (groups of
    8, a partial last group zero-filled); fewer run it on planar images.  The
    samples and their summation order are the same (four sample phases per ray
    by default, one sequential sum with RAFT_PJ_SEQUENTIAL=1), so 11 slices at
    once must equal 4 + 7 slices bit for bit: Radon, tEM (with metrics) and eEM."""
    import ctypes
    import torch
    from sscRaft import synthetic as S
    from sscRaft.rafttypes import _ptr, libraft
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    N, A, n = 200, 150, 11
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    img = torch.stack([S.phantom_image(S.ellipse_params(700 + k, 8), N, xp=torch, device="cuda")
                       for k in range(n)]).contiguous()
    full = torch.empty((n, A, N), device="cuda")
    assert libraft.raft_radon_device(0, p(full), p(img), _ptr(ang), N, N, N, A, n, 1.0, 1.0, None) == 0
    parts = torch.empty_like(full)
    for a, b in ((0, 4), (4, 11)):
        assert libraft.raft_radon_device(0, p(parts[a:b]), p(img[a:b]), _ptr(ang), N, N, N, A, b - a, 1.0, 1.0,
                                         None) == 0
    torch.cuda.synchronize()
    assert torch.equal(full, parts)
    trans = torch.exp(-full * (2.5 / full.amax())).contiguous()
    flat = torch.ones((n, N), device="cuda")
    for kind, data in ((0, trans), (1, full * (2.0 / (N - 1)))):
        data = data.contiguous()
        o_full = torch.ones((n, N, N), device="cuda")
        m_full = torch.zeros((3, n, 3), dtype=torch.float64, device="cuda")
        assert libraft.raft_em_device(kind, 0, p(o_full), p(data), p(flat), _ptr(ang), N, A, n, 3, p(m_full), 1,
                                      None) == 0
        o_part = torch.ones_like(o_full)
        m_part = torch.zeros_like(m_full)
        for a, b in ((0, 4), (4, 11)):
            m = torch.zeros((3, b - a, 3), dtype=torch.float64, device="cuda")
            assert libraft.raft_em_device(kind, 0, p(o_part[a:b]), p(data[a:b]), p(flat[a:b]), _ptr(ang), N, A,
                                          b - a, 3, p(m), 1, None) == 0
            m_part[:, a:b] = m
        torch.cuda.synchronize()
        assert torch.equal(o_full, o_part), kind
        assert torch.allclose(m_full, m_part, rtol=1e-12, atol=0), kind


def test_projector_phases_agree_with_sequential_sums():
    """Each ray's samples summed over four lane phases and combined by a fixed
    butterfly (the default) against one sequential sum per ray (the
    reference's order, RAFT_PJ_SEQUENTIAL=1): rounding only.  Two FP32 orders
    of a 300-term sum differ by about sqrt(300) x 6e-8 = 1e-6 (measured 1.2e-6),
    so rel-L2 <= 5e-6 for the Radon transform of 9 slices (interleaved) and of
    1 slice (planar); a misplaced sample shows as 1e-3 or more."""
    import ctypes
    import torch
    from sscRaft import synthetic as S
    from sscRaft.rafttypes import _ptr, libraft
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    N, A = 300, 200
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    img = torch.stack([S.phantom_image(S.ellipse_params(900 + k, 8), N, xp=torch, device="cuda")
                       for k in range(9)]).contiguous()
    old = os.environ.get("RAFT_PJ_SEQUENTIAL")
    try:
        outs = {}
        for seq in (False, True):
            if seq:
                os.environ["RAFT_PJ_SEQUENTIAL"] = "1"
            else:
                os.environ.pop("RAFT_PJ_SEQUENTIAL", None)
            for n in (9, 1):
                o = torch.empty((n, A, N), device="cuda")
                assert libraft.raft_radon_device(0, p(o), p(img[:n].contiguous()), _ptr(ang), N, N, N, A, n, 1.0, 1.0,
                                                 None) == 0
                outs[(seq, n)] = o
        torch.cuda.synchronize()
    finally:
        if old is None:
            os.environ.pop("RAFT_PJ_SEQUENTIAL", None)
        else:
            os.environ["RAFT_PJ_SEQUENTIAL"] = old
    for n in (9, 1):
        a, b = outs[(False, n)].double(), outs[(True, n)].double()
        err = float((a - b).norm() / b.norm())
        print(f"Radon {n} slices, phases vs sequential: rel-L2 {err:.2e}")
        assert err <= 5e-6, (n, err)
