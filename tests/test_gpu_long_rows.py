"""GPU parity of padded rows too long for one CTA's shared memory.

Up to N*(1+pad) = 14080 bins the row filter transforms a row pair inside one
CTA; longer rows are filtered by a cluster of C CTAs (distributed shared
memory, four-step transform, C = the smallest of 2..8 that fits).  Vs the
FP64 oracle: FBP nearest (given the GPU fast-intrinsic sin/cos values)
rel-L2 <= 2e-5 (also with the 'none' filter, which only pads), linear FP32
<= 1e-5, lowpass <= 1e-5; lowpass with 'none' leaves its input unchanged
(the reference returns early).  Rows whose length has a prime factor above
7 are transformed by Bluestein's algorithm, or, when its buffers do not fit,
filtered by direct circular convolution: <= 2e-5 against the oracle.
"""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import fbp_params, sino_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,pad", [(4096, 2), (4096, 1)])
def test_fbp_largest_compiled_lengths_vs_oracle(N, pad, oracle):
    """4096^2 images with 12288- and 8192-point rows (the largest filter
    lengths compiled for their length), 2 slices, Hann, axis offset 1.5:
    nearest vs the FP64 oracle given the fast-intrinsic sin/cos <= 2e-5,
    linear FP32 rows <= 1e-5, linear BF16 rows <= 4e-3."""
    from sscRaft.rafttypes import fast_sincos
    A, B, ftype, offset = 64, 2, 5, 1.5
    sino, ang = sino_case(N, A, B, seed=N + pad, n_ell=12)
    pf, pi = fbp_params(N, A, B, pad=pad, ftype=ftype, offset=offset)
    out = _fbp(sino, ang, pf, pi)
    ref = oracle.fbp(sino, ang, oracle.MODE_REF, ftype, pad, offset=offset, trig=fast_sincos(ang, 0))
    err = rel_l2(out, ref)
    print(f"N={N} pad={pad} nearest vs oracle: {err:.3e}")
    assert err <= 2e-5, err
    ref = oracle.fbp(sino, ang, oracle.MODE_LIN, ftype, pad, offset=offset)
    err32 = rel_l2(_fbp(sino, ang, pf, pi, 1, 1), ref)
    err16 = rel_l2(_fbp(sino, ang, pf, pi, 1, 2), ref)
    print(f"N={N} pad={pad} linear vs oracle: FP32 {err32:.3e}, BF16 {err16:.3e}")
    assert err32 <= 1e-5, err32
    assert err16 <= 4e-3, err16


def _fbp(sino, ang, pf, pi, geometry=0, store=0):
    from sscRaft.rafttypes import _ptr, check_error, libraft
    No = int(pi[3])
    obj = np.zeros((sino.shape[0], No, No), np.float32)
    g = np.array([0], np.intc)
    rc = libraft.raft_fbp_ext(_ptr(g), 1, _ptr(obj), _ptr(sino), _ptr(ang), _ptr(pf), _ptr(pi), geometry, store)
    check_error("fbp")
    assert rc == 0
    return obj


@pytest.mark.parametrize("N,A,ftype,offset", [
    (4800, 48, 5, 2.5),     # Np = 14400 = 2 x 7200: cluster of 2
    (4725, 32, 7, 0.0),     # Np = 14175 = 3 x 4725 (odd): cluster of 3
    (4800, 16, 0, 0.0),     # 'none': pad and copy only, by the cluster kernel
])
def test_fbp_long_rows_vs_oracle(N, A, ftype, offset, oracle):
    from sscRaft.rafttypes import fast_sincos
    sino, ang = sino_case(N, A, 1, seed=N, n_ell=6)
    pf, pi = fbp_params(N, A, 1, pad=2, ftype=ftype, offset=offset)
    out = _fbp(sino, ang, pf, pi)
    ref = oracle.fbp(sino, ang, oracle.MODE_REF, ftype, 2, offset=offset, trig=fast_sincos(ang, 0))
    err = rel_l2(out, ref)
    print(f"N={N} nearest vs oracle: {err:.3e}")
    assert err <= 2e-5, err
    if N == 4800:
        lin = _fbp(sino, ang, pf, pi, geometry=1, store=1)
        ref = oracle.fbp(sino, ang, oracle.MODE_LIN, ftype, 2, offset=offset)
        err = rel_l2(lin, ref)
        print(f"N={N} linear FP32 vs oracle: {err:.3e}")
        assert err <= 1e-5, err


@pytest.mark.parametrize("N,A", [
    (61, 20),       # Np = 183 = 3 x 61: Bluestein transforms (M = 375)
    (2447, 8),      # Np = 7341 = 3 x 2447: Bluestein would not fit, direct circular convolution
])
def test_fbp_prime_factor_rows_vs_oracle(N, A, oracle):
    from sscRaft.rafttypes import fast_sincos
    sino, ang = sino_case(N, A, 1, seed=N + 1, n_ell=6)
    pf, pi = fbp_params(N, A, 1, pad=2, ftype=5, offset=1.5)
    out = _fbp(sino, ang, pf, pi)
    ref = oracle.fbp(sino, ang, oracle.MODE_REF, 5, 2, offset=1.5, trig=fast_sincos(ang, 0))
    err = rel_l2(out, ref)
    print(f"N={N} (Np={3 * N}) nearest vs oracle: {err:.3e}")
    assert err <= 2e-5, err


def test_lowpass_long_rows_vs_oracle(oracle):
    import sscRaft
    # Np = 32768: two or three CTAs cannot hold it, a cluster of 4 does
    N, A = 16384, 6
    rng = np.random.default_rng(7)
    x = np.linspace(-1, 1, N)
    sino = np.stack([np.exp(-((x - rng.uniform(-0.5, 0.5)) / 0.2) ** 2) + 0.01 * rng.standard_normal(N)
                     for _ in range(A)]).astype(np.float32)[None]
    t = sino.copy()
    out = sscRaft.lowpass(t, dic={"gpu": [0], "filter": "hann", "padding": 1})
    ref = oracle.lowpass(sino, oracle.MODE_REF, 5, 1)
    err = rel_l2(out, ref)
    print(f"lowpass N={N} pad 1 vs oracle: {err:.3e}")
    assert err <= 1e-5, err
    # the 'none' filter pads and crops only: the input comes back unchanged
    t = sino.copy()
    out = sscRaft.lowpass(t, dic={"gpu": [0], "filter": "none", "padding": 1})
    np.testing.assert_array_equal(out, sino)
