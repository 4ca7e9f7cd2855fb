"""CPU check of the backprojector's shared-memory window bounds.

For each configuration the layout comes from the library's own planner
(raft_plan_window); the per-tile, per-angle window start restates the
kernel's rule (backproject.cu angle_param: min index over the tile's four
corners, minus one bin, aligned down).  Every pixel of every tile must then
index inside its staged window [0, W), and every window inside the stored
row [0, Wg) -- so the kernel's safety clamps never change a result."""
import numpy as np
import pytest

TX, TY = 64, 32
f32 = np.float32


def plan(pf, pi, geometry, store):
    from sscRaft.rafttypes import libraft, _ptr, check_error
    out = np.zeros(4, np.int32)
    if libraft.raft_plan_window(_ptr(pf), _ptr(pi), geometry, store, _ptr(out)):
        check_error("plan_window")
    return [int(v) for v in out]


def floor_to(v, a):
    return v - ((v % a) + a) % a


def check_fbp_ref(N, pad, pixel, angles):
    pf = np.array([0, 0, 1, 0, pixel, pixel, 0], np.float32)
    pi = np.array([N, len(angles), 1, N, pad, 0, 0, 7, 0, 0], np.int32)
    wlo, Wg, W, align = plan(pf, pi, 0, 0)
    Np = N * (1 + pad)
    xmin = f32(-f32(pixel) * f32(Np) / f32(2.0))
    tmin = xmin
    off = (pad * N) // 2
    Xe = -(-N // TX) * TX
    Ye = -(-N // TY) * TY
    ii = np.arange(Xe)
    jj = np.arange(Ye)
    x = (xmin + (ii + off).astype(f32) * f32(pixel)).astype(f32)
    y = (xmin + (jj + off).astype(f32) * f32(pixel)).astype(f32)
    for th in angles:
        c, s = np.cos(f32(th), dtype=f32), np.sin(f32(th), dtype=f32)
        t = (x[None, :] * c - y[:, None] * s).astype(f32)
        ti = np.trunc(((t - tmin) / f32(pixel)).astype(f32)).astype(np.int64)
        for ty in range(Ye // TY):
            for tx in range(Xe // TX):
                blk = ti[ty * TY:(ty + 1) * TY, tx * TX:(tx + 1) * TX]
                corners = [blk[0, 0], blk[0, -1], blk[-1, 0], blk[-1, -1]]
                b = floor_to(min(corners) - 1 - wlo, align)
                assert 0 <= b <= Wg - W, (N, pad, th, b, Wg, W)
                k = blk - (wlo + b)
                assert k.min() >= 0 and k.max() < W, (N, pad, th, k.min(), k.max(), W)


def check_fbp_lin(N, pad, pixel, angles, store):
    pf = np.array([0, 0, 1, 0, pixel, pixel, 0], np.float32)
    pi = np.array([N, len(angles), 1, N, pad, 0, 0, 7, 0, 0], np.int32)
    wlo, Wg, W, align = plan(pf, pi, 1, store)
    Np, off = N * (1 + pad), (pad * N) // 2
    c0 = off - 0.5 * Np
    u0 = 0.5 * Np - wlo - 0.5
    Xe = -(-N // TX) * TX
    Ye = -(-N // TY) * TY
    for th in angles:
        cd, sd = np.cos(float(f32(th))), -np.sin(float(f32(th)))
        for ty in range(Ye // TY):
            for tx in range(Xe // TX):
                x0, y0 = tx * TX, ty * TY
                v00 = (x0 + c0) * cd + (y0 + c0) * sd + u0
                vmin = v00 + min(0.0, (TX - 1) * cd) + min(0.0, (TY - 1) * sd)
                b = floor_to(int(np.floor(vmin)) - 1, align)
                assert 0 <= b <= Wg - W
                va = f32(v00 - b)
                li = np.arange(TX, dtype=f32)
                lj = np.arange(TY, dtype=f32)
                v = (va + lj[:, None] * f32(sd) + li[None, :] * f32(cd)).astype(f32)
                k = np.rint(v)        # round half to even, as the magic-number add
                assert k.min() >= 0 and k.max() <= W - 1, (k.min(), k.max(), W)


@pytest.mark.parametrize("N,pad,pixel", [(64, 2, 1.0), (50, 2, 0.5), (63, 0, 1.0), (130, 1, 0.7),
                                         (257, 2, 1e-6), (40, 3, 2.0)])
def test_fbp_windows_in_bounds(N, pad, pixel):
    rng = np.random.default_rng(N + pad)
    angles = np.concatenate([[0.0, np.pi / 4, np.pi / 2, np.pi, 3 * np.pi / 2],
                             rng.uniform(0, 2 * np.pi, 12)]).astype(np.float32)
    check_fbp_ref(N, pad, pixel, angles)
    check_fbp_lin(N, pad, pixel, angles, 1)
    check_fbp_lin(N, pad, pixel, angles, 2)


@pytest.mark.parametrize("N", [16, 48, 100, 129])
def test_em_windows_in_bounds(N):
    pi = np.array([N, 20, 1, N, 0, 0, 0, 1, 1, 0], np.int32)
    pf = np.zeros(1, np.float32)
    wlo, Wg, W, align = plan(pf, pi, 2, 0)
    dxy = f32(2.0 / (N - 1))
    dt = f32(2.0 / (N - 1))
    Xe = -(-N // TX) * TX
    Ye = -(-N // TY) * TY
    x = (f32(-1.0) + np.arange(Xe).astype(f32) * dxy).astype(f32)
    y = (f32(-1.0) + np.arange(Ye).astype(f32) * dxy).astype(f32)
    rng = np.random.default_rng(N)
    for th in np.concatenate([[0, np.pi / 3, np.pi], rng.uniform(0, np.pi, 8)]).astype(np.float32):
        c, s = np.cos(th, dtype=f32), np.sin(th, dtype=f32)
        t = (x[None, :] * c + y[:, None] * s).astype(f32)
        T = np.trunc(((t - f32(-1.0)) / dt).astype(f32)).astype(np.int64)
        for ty in range(Ye // TY):
            for tx in range(Xe // TX):
                blk = T[ty * TY:(ty + 1) * TY, tx * TX:(tx + 1) * TX]
                corners = [blk[0, 0], blk[0, -1], blk[-1, 0], blk[-1, -1]]
                b = floor_to(min(corners) - 1 - wlo, align)
                assert 0 <= b <= Wg - W
                k = blk - (wlo + b)
                assert k.min() >= 0 and k.max() < W
        # the projector writes bins [0, N) at element (bin - wlo): inside the row
        assert -wlo >= 0 and N - 1 - wlo < Wg


def _tiles(a, ty, tx):
    """[Ye, Xe] -> [tiles_y, tiles_x, TY, TX]."""
    return a.reshape(ty, TY, tx, TX).transpose(0, 2, 1, 3)


def check_fbp_ref_vectorised(N, pad, pixel, angles):
    """check_fbp_ref for large N: one angle's whole image at a time."""
    pf = np.array([0, 0, 1, 0, pixel, pixel, 0], np.float32)
    pi = np.array([N, len(angles), 1, N, pad, 0, 0, 5, 0, 0], np.int32)
    wlo, Wg, W, align = plan(pf, pi, 0, 0)
    Np, off = N * (1 + pad), (pad * N) // 2
    xmin = f32(-f32(pixel) * f32(Np) / f32(2.0))
    Xe, Ye = -(-N // TX) * TX, -(-N // TY) * TY
    x = (xmin + (np.arange(Xe) + off).astype(f32) * f32(pixel)).astype(f32)
    y = (xmin + (np.arange(Ye) + off).astype(f32) * f32(pixel)).astype(f32)
    for th in angles:
        c, s = np.cos(f32(th), dtype=f32), np.sin(f32(th), dtype=f32)
        t = (x[None, :] * c - y[:, None] * s).astype(f32)
        ti = _tiles(np.trunc(((t - xmin) / f32(pixel)).astype(f32)).astype(np.int64), Ye // TY, Xe // TX)
        corners = np.minimum(np.minimum(ti[:, :, 0, 0], ti[:, :, 0, -1]), np.minimum(ti[:, :, -1, 0], ti[:, :, -1, -1]))
        b = corners - 1 - wlo
        b = b - ((b % align) + align) % align
        assert b.min() >= 0 and b.max() <= Wg - W, (N, th, int(b.min()), int(b.max()), Wg, W)
        k = ti - (wlo + b)[:, :, None, None]
        # no pixel reaches the kernel's clamp at W - 1 from beyond the window
        assert k.min() >= 0 and k.max() < W, (N, th, int(k.min()), int(k.max()), W)


def check_fbp_lin_vectorised(N, pad, pixel, angles, store):
    pf = np.array([0, 0, 1, 0, pixel, pixel, 0], np.float32)
    pi = np.array([N, len(angles), 1, N, pad, 0, 0, 5, 0, 0], np.int32)
    wlo, Wg, W, align = plan(pf, pi, 1, store)
    Np, off = N * (1 + pad), (pad * N) // 2
    c0 = off - 0.5 * Np
    u0 = 0.5 * Np - wlo - 0.5
    Xe, Ye = -(-N // TX) * TX, -(-N // TY) * TY
    tx0 = (np.arange(Xe // TX) * TX)[None, :]
    ty0 = (np.arange(Ye // TY) * TY)[:, None]
    li = np.arange(TX, dtype=f32)
    lj = np.arange(TY, dtype=f32)
    for th in angles:
        cd, sd = np.cos(float(f32(th))), -np.sin(float(f32(th)))
        v00 = (tx0 + c0) * cd + (ty0 + c0) * sd + u0
        vmin = v00 + min(0.0, (TX - 1) * cd) + min(0.0, (TY - 1) * sd)
        b = np.floor(vmin).astype(np.int64) - 1
        b = b - ((b % align) + align) % align
        assert b.min() >= 0 and b.max() <= Wg - W
        va = (v00 - b).astype(f32)
        v = (va[:, :, None, None] + lj[None, None, :, None] * f32(sd) + li[None, None, None, :] * f32(cd)).astype(f32)
        k = np.rint(v)
        assert k.min() >= 0 and k.max() <= W - 1, (N, th, float(k.min()), float(k.max()), W)


def test_fbp_windows_in_bounds_at_the_benchmark_size():
    """2048^2 images, 1800 angles over [0, pi), padding 2 (the batched FBP
    workload): every 15th angle plus the axis-aligned and diagonal ones."""
    ang = (np.arange(1800) * (np.pi / 1800)).astype(np.float32)
    pick = np.concatenate([ang[::15], np.array([np.pi / 4, np.pi / 2, 3 * np.pi / 4], np.float32)])
    check_fbp_ref_vectorised(2048, 2, 1.0, pick)
    check_fbp_lin_vectorised(2048, 2, 1.0, pick[::2], 1)
    check_fbp_lin_vectorised(2048, 2, 1.0, pick[::2], 2)
