"""Shared input builders for the tests (seeded, small)."""
import ctypes
import os

import numpy as np

from sscRaft import synthetic as S


def sino_case(N, A, nslices=1, seed=0, n_ell=8, pixel=1.0, pad=2, angles=None, noise=0.0):
    ang = S.uniform_angles(A) if angles is None else np.asarray(angles, np.float32)
    sinos = []
    for k in range(nslices):
        prm = S.ellipse_params(seed + k, n_ell)
        s = S.ellipse_sinogram(prm, ang, N, pixel=pixel, pad=pad)
        if noise:
            rng = np.random.default_rng(seed + 1000 + k)
            s = s + noise * rng.standard_normal(s.shape)
        sinos.append(s)
    return np.ascontiguousarray(np.stack(sinos).astype(np.float32)), ang


def phantom_case(N, nslices=1, seed=0, n_ell=8, scale=1.0):
    imgs = [S.phantom_image(S.ellipse_params(seed + k, n_ell), N) * scale for k in range(nslices)]
    return np.ascontiguousarray(np.stack(imgs).astype(np.float32))


def fbp_params(N, A, nslices, pad=2, ftype=7, pixel=1.0, offset=0.0, reg=0.0, beta_delta=0.0,
               blocksize=0, objsize=None):
    objsize = N if objsize is None else objsize
    pi = np.array([N, A, nslices, objsize, pad, 0, 0, ftype, 0, blocksize], np.int32)
    pf = np.array([beta_delta, reg, 1.0, 0.0, pixel, pixel, offset], np.float32)
    return pf, pi


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def temfq_counts(N, A, B, dx, seed):
    """Seeded transmission counts [B][A][N] of a phantom (attenuation in units
    of 1/dx per pixel, projections of about 1) with Poisson noise, a flat
    [B][N] of about 1e4 varying along the rays, and angles k pi / A."""
    import oracle as O  # only to make the transmission data from a forward projection
    rng = np.random.default_rng(seed)
    ang = (np.arange(A) * (np.pi / A)).astype(np.float32)
    img = phantom_case(N, B, seed=seed)
    p = O.em_forward(img.astype(np.float64), ang, N) * (N / 2) * dx
    x = np.arange(N)
    flat = np.stack([1e4 * (1 + 0.05 * np.cos(2 * np.pi * (x / N + rng.uniform()))) for _ in range(B)])
    counts = rng.poisson(flat[:, None, :] * np.exp(-p)).astype(np.float32)
    return counts, flat.astype(np.float32), ang
