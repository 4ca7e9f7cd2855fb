"""GPU test of the ragged batch: FBP and eEM requests of different sizes and
angle counts in one batch; every output must equal the single-request entry
point's output (same operators, same summation order) -- bit for bit."""
import ctypes

import numpy as np
import pytest

from helpers import fbp_params, phantom_case, sino_case

pytestmark = pytest.mark.gpu


def test_ragged_batch_matches_single_requests(oracle):
    import torch
    from sscRaft.geometries.parallel.batch_methods import reconstruct_ragged
    from sscRaft.geometries.parallel.em_methods import em_with_metrics
    from sscRaft.rafttypes import libraft, _ptr, check_error
    reqs, refs = [], []
    for N, A, filt, off in ((64, 45, 7, 0.0), (130, 90, 5, 1.5), (100, 180, 7, 0.0), (257, 60, 6, -2.0)):
        sino, ang = sino_case(N, A, 1, seed=N + A)
        d = torch.from_numpy(sino[0]).cuda()
        out = torch.zeros((N, N), dtype=torch.float32, device="cuda")
        reqs.append({"kind": "fbp", "data": d, "out": out, "angles": ang,
                     "filter": {7: "ramp", 5: "hann", 6: "hamming"}[filt], "offset": off})
        ref = torch.zeros((1, N, N), dtype=torch.float32, device="cuda")
        pf, pi = fbp_params(N, A, 1, ftype=filt, offset=off)
        rc = libraft.raft_fbp_device(0, ctypes.c_void_p(ref.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                     _ptr(np.ascontiguousarray(ang)), _ptr(pf), _ptr(pi), 0, 0, None)
        if rc:
            check_error("fbp")
        refs.append(ref[0])
    for N, A in ((48, 40), (64, 72)):
        img = phantom_case(N, 1, seed=N)
        ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
        tomo = oracle.em_forward(img.astype(np.float64), ang, N).astype(np.float32)[0]
        out = torch.ones((N, N), dtype=torch.float32, device="cuda")
        reqs.append({"kind": "eem", "data": torch.from_numpy(tomo).cuda(), "out": out, "angles": ang,
                     "iterations": 3})
        obj, _ = em_with_metrics("eEM", tomo[None], ang, 3)
        refs.append(torch.from_numpy(obj[0]).cuda())
    lat, total = reconstruct_ragged(reqs)
    torch.cuda.synchronize()
    for r, ref in zip(reqs, refs):
        got = r["out"].cpu().numpy()
        want = ref.cpu().numpy()
        assert np.array_equal(got, want), (r["kind"], got.shape, float(np.abs(got - want).max()))
    assert np.all(lat > 0) and np.all(lat <= total + 1e-9)
