"""Seeded synthetic tomography inputs: random-ellipse phantoms and their exact
parallel-beam projections.

The reference ships no datasets for this path, so every benchmark and test
input is generated here.  Geometry follows the FBP convention of
ssc-raft (cuda/src/geometries/parallel/reconstruction_methods/fbp.cu:38-67):
pixel column ``i`` sits at ``x = (i + off - Np/2) * pixel`` with
``off = pad*N//2``, ``Np = N*(1+pad)`` (which is ``(i - N/2) * pixel`` whenever
``pad*N`` is even), rows likewise in ``y``, detector bin ``c`` at the same
coordinate ``t``, and projection lines ``x*cos(theta) - y*sin(theta) = t``.

Ellipse parameters are in units of the half-width ``R = N/2`` pixels, so the
same phantom description rasterises / projects at any size.  Projections are
analytic line integrals (chord length times density) in physical length units
(``pixel`` per pixel), the unit the FBP filter expects.

All functions take an array namespace ``xp`` (numpy by default; torch works
for the large benchmark inputs, evaluated on the GPU).
"""
import math

import numpy as np


def ellipse_params(seed, n_ellipses, semi=(0.05, 0.4), intensity=(0.0, 1.0)):
    """Random ellipses: centre uniform in the unit disc, semi-axes U[semi],
    orientation U[0, pi), density U[intensity].  Returns float64 [n, 6]
    rows (x0, y0, a, b, phi, rho)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    r = np.sqrt(rng.uniform(0.0, 1.0, n_ellipses))
    ang = rng.uniform(0.0, 2 * math.pi, n_ellipses)
    a = rng.uniform(semi[0], semi[1], n_ellipses)
    b = rng.uniform(semi[0], semi[1], n_ellipses)
    phi = rng.uniform(0.0, math.pi, n_ellipses)
    rho = rng.uniform(intensity[0], intensity[1], n_ellipses)
    # keep every ellipse inside the unit disc so the object fits the field of view
    rr = np.minimum(r, np.maximum(0.0, 0.98 - np.maximum(a, b)))
    return np.stack([rr * np.cos(ang), rr * np.sin(ang), a, b, phi, rho], axis=1)


def uniform_angles(nangles, xp=np):
    """theta_a = a*pi/A, a < A (endpoint excluded)."""
    return (xp.arange(nangles, dtype=xp.float64) * (math.pi / nangles)).astype(xp.float32) \
        if xp is np else (xp.arange(nangles, dtype=xp.float64) * (math.pi / nangles)).float()


def _coord_offset(N, pad):
    Np = N * (1 + pad)
    return (pad * N) // 2 - Np / 2.0


def phantom_image(params, N, pad=2, xp=np, device=None):
    """Rasterise ellipses (pixel centres) on the N x N FBP grid, float32."""
    R = N / 2.0
    c0 = _coord_offset(N, pad)
    kw = {} if xp is np else {"device": device}
    idx = xp.arange(N, dtype=xp.float64, **kw)
    X = (idx + c0)[None, :] / R
    Y = (idx + c0)[:, None] / R
    img = xp.zeros((N, N), dtype=xp.float64, **kw)
    for x0, y0, a, b, phi, rho in np.asarray(params, dtype=np.float64):
        cp, sp = math.cos(phi), math.sin(phi)
        u = (X - x0) * cp + (Y - y0) * sp
        v = -(X - x0) * sp + (Y - y0) * cp
        img = img + rho * (((u / a) ** 2 + (v / b) ** 2) <= 1.0)
    return img.astype(xp.float32) if xp is np else img.float()


def ellipse_sinogram(params, angles, N, pixel=1.0, pad=2, nrays=None, xp=np, device=None):
    """Exact line integrals of the ellipse phantom, [A, nrays] float64,
    detector bins on the same centred grid as the image."""
    nrays = N if nrays is None else nrays
    R = N / 2.0
    c0 = _coord_offset(N, pad)
    kw = {} if xp is np else {"device": device}
    if xp is np:
        th = np.asarray(angles, dtype=np.float64)[:, None]
    else:
        th = xp.as_tensor(np.asarray(angles, dtype=np.float64), device=device)[:, None]
    t = ((xp.arange(nrays, dtype=xp.float64, **kw) + c0) / R)[None, :]
    cth, sth = xp.cos(th), xp.sin(th)
    out = xp.zeros((th.shape[0], nrays), dtype=xp.float64, **kw)
    for x0, y0, a, b, phi, rho in np.asarray(params, dtype=np.float64):
        cphi, sphi = math.cos(phi), math.sin(phi)
        c = cth * cphi - sth * sphi          # cos(theta + phi)
        s = sth * cphi + cth * sphi          # sin(theta + phi)
        s2 = (a * c) ** 2 + (b * s) ** 2
        tau = t - (x0 * cth - y0 * sth)
        d = s2 - tau * tau
        d = xp.clip(d, 0.0, None) if xp is np else xp.clamp(d, min=0.0)
        out = out + rho * 2.0 * a * b * xp.sqrt(d) / s2
    return out * (R * pixel)


def poisson_log_sinogram(p, I0, seed, scale_to=3.0, xp=np, generator=None):
    """Transmission data: counts ~ Poisson(I0*exp(-p*s)) with s such that
    max(p*s) = scale_to, returned as -log(max(counts,1)/I0) (float32) and s."""
    pmax = float(p.max())
    s = scale_to / pmax if pmax > 0 else 1.0
    lam = I0 * xp.exp(-p * s)
    if xp is np:
        rng = np.random.Generator(np.random.PCG64(seed))
        counts = rng.poisson(lam).astype(np.float64)
        return (-np.log(np.maximum(counts, 1.0) / I0)).astype(np.float32), s
    counts = xp.poisson(lam, generator=generator)
    return (-xp.log(xp.clamp(counts, min=1.0) / I0)).float(), s
