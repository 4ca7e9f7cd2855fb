"""GPU tests of the U-Net's 3x3 convolution on the tcgen05 tensor cores
(TMA-staged operands, TMEM accumulators): against the FP64 oracle on
BF16-rounded inputs (rel-L2 <= 1e-2: BF16 outputs) and against the mma.sync
kernel on the same inputs, over the tile shapes the kernel takes -- 128-pixel
tiles along a row (W >= 128, W not a multiple of 128), several whole rows per
tile (W = 64, 32, with H not a multiple of the rows per tile), 32- and
64-channel k-blocks, a concatenated second input, output-channel tiles of 32 to
256 and several tiles per pixel block (Cout = 384), the split output of the
data gradient; no pipeline wait runs out.  The weight gradient on tcgen05
against the oracle and the mma.sync kernel."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _bf(t):
    import torch
    return t.to(torch.bfloat16).contiguous()


def _f64(t):
    return t.float().cpu().numpy().astype(np.float64)


def _conv(x0, x1, w, b, N, H, W, C0, C1, Co, relu=1, path=2, split=0):
    import torch
    from sscRaft import warmstart as ws
    from sscRaft.rafttypes import libraft
    assert libraft.raft_unet_set_conv_path(path) == 0      # 2: tcgen05 kernel only, 1: mma.sync only
    try:
        if split:
            y = torch.empty(N, H, W, split, dtype=torch.bfloat16, device="cuda")
            y1 = torch.empty(N, H, W, Co - split, dtype=torch.bfloat16, device="cuda")
        else:
            y = torch.empty(N, H, W, Co, dtype=torch.bfloat16, device="cuda")
            y1 = None
        assert libraft.raft_unet_conv_fwd(ws._p(x0), C0, ws._p(x1), C1, ws._p(w), ws._p(b), ws._p(y), ws._p(y1),
                                          split, N, H, W, Co, relu, None) == 0
        torch.cuda.synchronize()
        assert libraft.raft_unet_conv_error() == 0
    finally:
        libraft.raft_unet_set_conv_path(0)
    return y if not split else torch.cat([y, y1], dim=-1)


@pytest.mark.parametrize("N,H,W,C0,C1,Co", [
    (1, 3, 128, 32, 0, 32),        # one tile per row, KC 32, BN 32
    (2, 3, 130, 64, 0, 64),        # a second, mostly out-of-image x block; KC 64
    (1, 5, 64, 64, 32, 64),        # two rows per tile, H odd; concatenated input with KC 32
    (1, 6, 32, 128, 0, 256),       # four rows per tile; BN 256
    (1, 2, 256, 128, 64, 128),     # concatenation with KC 64; BN 128
    (1, 2, 128, 64, 0, 384),       # three output-channel tiles of 128
])
def test_tc_conv_vs_oracle_and_mma_sync(oracle, N, H, W, C0, C1, Co):
    import torch
    torch.manual_seed(N * 1000 + H * 100 + W + C0 + C1 + Co)
    x0 = _bf(torch.randn(N, H, W, C0, device="cuda"))
    x1 = _bf(torch.randn(N, H, W, C1, device="cuda")) if C1 else None
    w = _bf(torch.randn(Co, 3, 3, C0 + C1, device="cuda") * 0.1)
    b = torch.randn(Co, device="cuda")
    y_tc = _conv(x0, x1, w, b, N, H, W, C0, C1, Co)
    y_ms = _conv(x0, x1, w, b, N, H, W, C0, C1, Co, path=1)
    xc = _f64(x0) if x1 is None else np.concatenate([_f64(x0), _f64(x1)], axis=-1)
    ref = oracle.conv3x3(xc, _f64(w), _f64(b), relu=True)
    assert rel_l2(_f64(y_tc), ref) <= 1e-2, rel_l2(_f64(y_tc), ref)
    assert rel_l2(_f64(y_tc), _f64(y_ms)) <= 1e-2, rel_l2(_f64(y_tc), _f64(y_ms))


def test_tc_conv_split_output_no_bias(oracle):
    # the data-gradient form: no bias, no ReLU, output channels split into two tensors
    import torch
    torch.manual_seed(5)
    N, H, W, C0, Co, split = 1, 4, 128, 64, 96, 64
    x0 = _bf(torch.randn(N, H, W, C0, device="cuda"))
    w = _bf(torch.randn(Co, 3, 3, C0, device="cuda") * 0.1)
    y = _conv(x0, None, w, None, N, H, W, C0, 0, Co, relu=0, split=split)
    ref = oracle.conv3x3(_f64(x0), _f64(w), None, relu=False)
    assert rel_l2(_f64(y), ref) <= 1e-2, rel_l2(_f64(y), ref)


def test_tc_only_path_rejects_other_widths():
    import torch
    from sscRaft import warmstart as ws
    from sscRaft.rafttypes import libraft
    x = _bf(torch.randn(1, 2, 70, 32, device="cuda"))
    w = _bf(torch.randn(32, 3, 3, 32, device="cuda"))
    y = torch.empty(1, 2, 70, 32, dtype=torch.bfloat16, device="cuda")
    libraft.raft_unet_set_conv_path(2)
    try:
        assert libraft.raft_unet_conv_fwd(ws._p(x), 32, None, 0, ws._p(w), None, ws._p(y), None, 0,
                                          1, 2, 70, 32, 0, None) == 1
    finally:
        libraft.raft_unet_set_conv_path(0)
    # the default path takes the mma.sync kernel for this width
    assert libraft.raft_unet_conv_fwd(ws._p(x), 32, None, 0, ws._p(w), None, ws._p(y), None, 0,
                                      1, 2, 70, 32, 0, None) == 0


@pytest.mark.parametrize("N,H,W,C0,C1", [(1, 5, 128, 32, 0), (2, 3, 130, 32, 0), (1, 6, 256, 64, 32), (1, 4, 512, 32, 0)])
def test_tc_conv_halo_tiles(oracle, N, H, W, C0, C1):
    # 32 -> 32 channel layers use halo tiles (one input box per 32-channel chunk serves
    # all nine taps); same results as the per-tap tiles and the oracle
    import torch
    from sscRaft.rafttypes import libraft
    torch.manual_seed(7 + H + W + C0 + C1)
    x0 = _bf(torch.randn(N, H, W, C0, device="cuda"))
    x1 = _bf(torch.randn(N, H, W, C1, device="cuda")) if C1 else None
    w = _bf(torch.randn(32, 3, 3, C0 + C1, device="cuda") * 0.1)
    b = torch.randn(32, device="cuda")
    y_halo = _conv(x0, x1, w, b, N, H, W, C0, C1, 32)
    libraft.raft_unet_set_conv_halo(0)
    try:
        y_tap = _conv(x0, x1, w, b, N, H, W, C0, C1, 32)
    finally:
        libraft.raft_unet_set_conv_halo(1)
    xc = _f64(x0) if x1 is None else np.concatenate([_f64(x0), _f64(x1)], axis=-1)
    ref = oracle.conv3x3(xc, _f64(w), _f64(b), relu=True)
    assert rel_l2(_f64(y_halo), ref) <= 1e-2, rel_l2(_f64(y_halo), ref)
    assert rel_l2(_f64(y_halo), _f64(y_tap)) <= 2e-3, rel_l2(_f64(y_halo), _f64(y_tap))


def _wgrad(dy, x0, x1, N, H, W, C0, C1, Co, path):
    import torch
    from sscRaft import warmstart as ws
    from sscRaft.rafttypes import libraft
    dw = torch.full((Co, 3, 3, C0 + C1), 0.25, device="cuda")      # the gradient accumulates into dw
    db = torch.full((Co,), -0.5, device="cuda")
    assert libraft.raft_unet_set_conv_path(path) == 0
    try:
        assert libraft.raft_unet_conv_wgrad(ws._p(dy), ws._p(x0), C0, ws._p(x1), C1, ws._p(dw), ws._p(db),
                                            N, H, W, Co, None) == 0
        torch.cuda.synchronize()
        assert libraft.raft_unet_conv_error() == 0
    finally:
        libraft.raft_unet_set_conv_path(0)
    return _f64(dw) - 0.25, _f64(db) + 0.5


@pytest.mark.parametrize("N,H,W,C0,C1,Co", [
    (2, 5, 64, 32, 0, 32),        # level-0 shape: 9 row blocks of 32 in three 128-row tiles
    (1, 4, 128, 32, 32, 64),      # concatenated input
    (1, 3, 192, 96, 0, 32),       # 27 row blocks: a partly filled last tile
    (2, 3, 64, 64, 64, 128),
    (1, 2, 64, 256, 256, 256),    # 144 row blocks, 256 output channels
])
def test_tc_wgrad_vs_oracle_and_mma_sync(oracle, N, H, W, C0, C1, Co):
    """Weight and bias gradients on tcgen05 (operands transposed in shared
    memory, split over the pixels, partials summed in a fixed order; both CTA
    shapes: all nine taps of a 32-channel chunk, and 128-row blocks) vs the
    FP64 oracle on the BF16 inputs (rel-L2 <= 1e-4, FP32 accumulation of exact
    BF16 products) and vs the mma.sync kernel (<= 1e-5)."""
    import torch
    torch.manual_seed(11 + H + W + C0 + C1 + Co)
    x0 = _bf(torch.randn(N, H, W, C0, device="cuda"))
    x1 = _bf(torch.randn(N, H, W, C1, device="cuda")) if C1 else None
    dy = _bf(torch.randn(N, H, W, Co, device="cuda"))
    from sscRaft.rafttypes import libraft
    dw_tc, db_tc = _wgrad(dy, x0, x1, N, H, W, C0, C1, Co, 2)
    dw_ms, db_ms = _wgrad(dy, x0, x1, N, H, W, C0, C1, Co, 1)
    libraft.raft_unet_set_wgrad_nine(0)          # 128-row blocks of (tap, channel) instead of nine-tap CTAs
    try:
        dw_rb, _ = _wgrad(dy, x0, x1, N, H, W, C0, C1, Co, 2)
    finally:
        libraft.raft_unet_set_wgrad_nine(1)
    xc = _f64(x0) if x1 is None else np.concatenate([_f64(x0), _f64(x1)], axis=-1)
    ref = oracle.conv3x3_wgrad(_f64(dy), xc)
    assert rel_l2(dw_rb, ref) <= 1e-4, rel_l2(dw_rb, ref)
    assert rel_l2(dw_tc, ref) <= 1e-4, rel_l2(dw_tc, ref)
    assert rel_l2(dw_tc, dw_ms) <= 1e-5, rel_l2(dw_tc, dw_ms)
    ref_db = _f64(dy).sum(axis=(0, 1, 2))
    assert rel_l2(db_tc, ref_db) <= 1e-4, rel_l2(db_tc, ref_db)
