"""GPU tests of the learned warm start (tensor-core U-Net kernels).

* conv3x3 forward (with a concatenated second input, bias, ReLU), weight
  gradient and data gradient vs the FP64 CPU oracle on BF16-rounded inputs:
  rel-L2 <= 1e-2 for BF16 outputs, <= 1e-4 for the FP32 weight gradient;
* the whole network's parameter gradients vs PyTorch FP32 autograd on the
  same weights and inputs: rel-L2 <= 5e-2 per tensor (BF16 activations);
* training lowers the loss by a quarter or more, the trained network's output
  on held-out pairs is closer to the EM label than its FBP input (MSE below
  0.8x), and its warm start reaches the plain-EM target residual in fewer
  iterations than plain EM."""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _bf(t):
    import torch
    return t.to(torch.bfloat16).contiguous()


def _f64(t):
    return t.float().cpu().numpy().astype(np.float64)


def test_conv_kernels_vs_oracle(oracle):
    import torch
    from sscRaft import warmstart as ws
    from sscRaft.rafttypes import libraft
    torch.manual_seed(0)
    N, H, W, C0, C1, Co = 2, 8, 70, 32, 32, 64
    x0 = _bf(torch.randn(N, H, W, C0, device="cuda"))
    x1 = _bf(torch.randn(N, H, W, C1, device="cuda"))
    w = _bf(torch.randn(Co, 3, 3, C0 + C1, device="cuda") * 0.1)
    b = torch.randn(Co, device="cuda")
    y = torch.empty(N, H, W, Co, dtype=torch.bfloat16, device="cuda")
    assert libraft.raft_unet_conv_fwd(ws._p(x0), C0, ws._p(x1), C1, ws._p(w), ws._p(b), ws._p(y), None, 0,
                                      N, H, W, Co, 1, None) == 0
    xc = np.concatenate([_f64(x0), _f64(x1)], axis=-1)
    ref = oracle.conv3x3(xc, _f64(w), _f64(b), relu=True)
    assert rel_l2(_f64(y), ref) <= 1e-2, rel_l2(_f64(y), ref)
    # weight gradient (and bias gradient)
    dy = _bf(torch.randn(N, H, W, Co, device="cuda"))
    dw = torch.zeros(Co, 3, 3, C0 + C1, device="cuda")
    db = torch.zeros(Co, device="cuda")
    assert libraft.raft_unet_conv_wgrad(ws._p(dy), ws._p(x0), C0, ws._p(x1), C1, ws._p(dw), ws._p(db),
                                        N, H, W, Co, None) == 0
    ref_dw = oracle.conv3x3_wgrad(_f64(dy), xc)
    assert rel_l2(_f64(dw), ref_dw) <= 1e-4, rel_l2(_f64(dw), ref_dw)
    assert rel_l2(_f64(db), _f64(dy).sum(axis=(0, 1, 2))) <= 1e-4
    # data gradient: flipped/transposed weights, output split back into the two inputs
    wt = torch.empty(C0 + C1, 3, 3, Co, dtype=torch.bfloat16, device="cuda")
    assert libraft.raft_unet_flip_weights(ws._p(w), ws._p(wt), Co, C0 + C1, None) == 0
    d0 = torch.empty(N, H, W, C0, dtype=torch.bfloat16, device="cuda")
    d1 = torch.empty(N, H, W, C1, dtype=torch.bfloat16, device="cuda")
    assert libraft.raft_unet_conv_fwd(ws._p(dy), Co, None, 0, ws._p(wt), None, ws._p(d0), ws._p(d1), C0,
                                      N, H, W, C0 + C1, 0, None) == 0
    ref_dx = oracle.conv3x3_dgrad(_f64(dy), _f64(w))
    assert rel_l2(_f64(d0), ref_dx[..., :C0]) <= 1e-2
    assert rel_l2(_f64(d1), ref_dx[..., C0:]) <= 1e-2


def test_input_conv_equals_packed_first_layer(oracle):
    """Inference's first layer straight from the one-channel image
    (raft_unet_input_conv) against the training path's packed 32-channel input
    + tensor-core convolution, and against the FP64 oracle on the BF16-rounded
    input: BF16 outputs within rel-L2 1e-2 of the oracle and 2e-3 of the
    packed path (the two sum nine exact products in different orders; measured
    equal)."""
    import torch
    from sscRaft import warmstart as ws
    from sscRaft.rafttypes import libraft
    torch.manual_seed(5)
    N, H, W = 2, 128, 160
    img = torch.rand(N, H, W, device="cuda")
    scale = torch.tensor([3.0, 0.5], device="cuda")
    w = _bf(torch.randn(32, 3, 3, 32, device="cuda") * 0.3)
    w[..., 1:] = 0
    b = torch.randn(32, device="cuda") * 0.1
    y = torch.empty(N, H, W, 32, dtype=torch.bfloat16, device="cuda")
    assert libraft.raft_unet_input_conv(ws._p(img), ws._p(scale), ws._p(w), 32, ws._p(b), ws._p(y), N, H, W, None) == 0
    x = torch.empty(N, H, W, 32, dtype=torch.bfloat16, device="cuda")
    assert libraft.raft_unet_input(ws._p(img), ws._p(scale), ws._p(x), N, H, W, 32, None) == 0
    yp = torch.empty_like(y)
    assert libraft.raft_unet_conv_fwd(ws._p(x), 32, None, 0, ws._p(w), ws._p(b), ws._p(yp), None, 0,
                                      N, H, W, 32, 1, None) == 0
    ref = oracle.conv3x3(_f64(x), _f64(w), _f64(b), relu=True)
    e_or, e_pk = rel_l2(_f64(y), ref), rel_l2(_f64(y), _f64(yp))
    print(f"input conv vs oracle {e_or:.2e}, vs packed tensor-core layer {e_pk:.2e}")
    assert e_or <= 1e-2, e_or
    assert e_pk <= 2e-3, e_pk

def test_input_wgrad_equals_packed_first_layer_gradient(oracle):
    """The first layer's weight gradient (channel 0 of each tap) and bias
    gradient computed from the image (raft_unet_input_wgrad) against the
    general weight gradient on the packed 32-channel input and against the
    FP64 oracle: rel-L2 <= 1e-5 and <= 1e-4."""
    import torch
    from sscRaft import warmstart as ws
    from sscRaft.rafttypes import libraft
    torch.manual_seed(6)
    N, H, W = 2, 96, 160
    img = torch.rand(N, H, W, device="cuda")
    scale = torch.tensor([2.0, 0.7], device="cuda")
    dpre = _bf(torch.randn(N, H, W, 32, device="cuda"))
    dw = torch.zeros(32, 3, 3, 32, device="cuda")
    db = torch.zeros(32, device="cuda")
    work = torch.empty(N * H * 320, device="cuda")
    assert libraft.raft_unet_input_wgrad(ws._p(img), ws._p(scale), ws._p(dpre), ws._p(dw), 32, ws._p(db), ws._p(work),
                                         work.numel(), N, H, W, None) == 0
    x = torch.empty(N, H, W, 32, dtype=torch.bfloat16, device="cuda")
    assert libraft.raft_unet_input(ws._p(img), ws._p(scale), ws._p(x), N, H, W, 32, None) == 0
    dw_p = torch.zeros_like(dw)
    db_p = torch.zeros_like(db)
    assert libraft.raft_unet_conv_wgrad(ws._p(dpre), ws._p(x), 32, None, 0, ws._p(dw_p), ws._p(db_p),
                                        N, H, W, 32, None) == 0
    ref = oracle.conv3x3_wgrad(_f64(dpre), _f64(x))
    assert float(dw[..., 1:].abs().max()) == 0.0
    e_pk = rel_l2(_f64(dw)[..., 0], _f64(dw_p)[..., 0])
    e_or = rel_l2(_f64(dw)[..., 0], ref[..., 0])
    e_b = rel_l2(_f64(db), _f64(dpre).sum(axis=(0, 1, 2)))
    print(f"input wgrad vs packed {e_pk:.2e}, vs oracle {e_or:.2e}, bias {e_b:.2e}")
    assert e_pk <= 1e-5, e_pk
    assert e_or <= 1e-4, e_or
    assert e_b <= 1e-5, e_b

@pytest.mark.parametrize("C", [32, 8, 24])
def test_head_backward_vs_fp64(C):
    """raft_unet_head backward: dh[p][c] = bf16(g[p] * w[c]) bit for bit (one
    FP32 product, rounded to nearest even), dw[c] = sum_p g[p] h[p][c] and
    db = sum_p g[p] within 1e-5 of FP64.  C = 32 and 8 take the 16-byte-vector
    kernel (8-channel groups per thread), C = 24 the scalar one."""
    import torch
    from sscRaft import warmstart as ws
    from sscRaft.rafttypes import libraft
    torch.manual_seed(C)
    N, HW = 3, 257 * 129
    h = _bf(torch.randn(N, HW, C, device="cuda"))
    w = torch.randn(C, device="cuda")
    g = torch.randn(N, HW, device="cuda")
    dh = torch.empty_like(h)
    dw = torch.zeros(C, device="cuda")
    db = torch.zeros(1, device="cuda")
    assert libraft.raft_unet_head(1, ws._p(h), ws._p(w), None, None, None, ws._p(g), ws._p(dh), ws._p(dw),
                                  ws._p(db), N, HW, C, None) == 0
    torch.cuda.synchronize()
    want_dh = (g[..., None] * w).to(torch.bfloat16)
    assert torch.equal(dh.view(torch.int16), want_dh.view(torch.int16))
    gd, hd = _f64(g), _f64(h)
    assert rel_l2(_f64(dw), np.einsum("np,npc->c", gd, hd)) <= 1e-5
    assert abs(float(db.item()) - gd.sum()) <= 1e-5 * np.abs(gd).sum()


def _torch_unet(net, img, scale):
    """The same network in plain PyTorch FP32 (NCHW), for the gradient check."""
    import torch
    import torch.nn.functional as F
    P = {}
    for name, *_ in net.LAYERS:
        P[name] = (net.w[name].permute(0, 3, 1, 2).clone().requires_grad_(True),
                   net.b[name].clone().requires_grad_(True))
    hw = net.w["head"].clone().requires_grad_(True)
    hb = net.b["head"].clone().requires_grad_(True)
    x = (img * scale[:, None, None])[:, None]
    x = torch.cat([x, torch.zeros(x.shape[0], 31, *x.shape[2:], device=x.device)], 1)

    def c(n, t):
        return F.relu(F.conv2d(t, P[n][0], P[n][1], padding=1))
    s0 = c("e0b", c("e0a", x))
    s1 = c("e1b", c("e1a", F.avg_pool2d(s0, 2)))
    s2 = c("e2b", c("e2a", F.avg_pool2d(s1, 2)))
    bt = c("e3b", c("e3a", F.avg_pool2d(s2, 2)))
    up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")  # noqa: E731
    d2 = c("d2b", c("d2a", torch.cat([up(bt), s2], 1)))
    d1 = c("d1b", c("d1a", torch.cat([up(d2), s1], 1)))
    d0 = c("d0b", c("d0a", torch.cat([up(d1), s0], 1)))
    out = (d0 * hw[None, :, None, None]).sum(1) + hb + img * scale[:, None, None]
    return out, P, hw, hb


def test_network_gradients_vs_torch_fp32():
    import torch
    from sscRaft import warmstart as ws
    dev = torch.device("cuda", 0)
    net = ws.UNet(dev, seed=3)
    net.w["head"].normal_(0, 0.1)
    torch.manual_seed(1)
    img = torch.rand(2, 64, 64, device=dev) + 0.5
    target = img * 1.3 + 0.1 * torch.rand(2, 64, 64, device=dev)
    sc = ws.input_scale(img)
    out = net.forward(img, sc, keep=True)
    g = torch.empty_like(out)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    from sscRaft.rafttypes import libraft
    libraft.raft_unet_mse(ws._p(out), ws._p(target), ws._p(sc), ws._p(g), ws._p(loss), 2, 64 * 64, None)
    net.backward(g)
    tout, P, hw, hb = _torch_unet(net, img, sc)
    tloss = ((tout - target * sc[:, None, None]) ** 2).mean()
    tloss.backward()
    assert abs(float(loss) - float(tloss)) <= 2e-2 * float(tloss)
    assert rel_l2(out.detach().cpu().numpy(), tout.detach().cpu().numpy()) <= 2e-2
    for name, *_ in net.LAYERS:
        gw = net.gw[name].permute(0, 3, 1, 2).cpu().numpy()
        e = rel_l2(gw, P[name][0].grad.cpu().numpy())
        assert e <= 5e-2, (name, e)
    assert rel_l2(net.gw["head"].cpu().numpy(), hw.grad.cpu().numpy()) <= 5e-2


def test_training_reduces_loss_and_warm_start_helps():
    import torch
    from sscRaft import warmstart as ws
    dev = torch.device("cuda", 0)
    inputs, labels, trans, ang = ws.make_pairs(96, 70_000, dev, N=128, A=96, em_iters=60, chunk=48)
    net = ws.UNet(dev, seed=0)
    losses = ws.train(net, inputs[:80], labels[:80], epochs=24, batch=8, lr=2e-3)
    assert np.mean(losses[-8:]) < 0.75 * np.mean(losses[:8]), (np.mean(losses[:8]), np.mean(losses[-8:]))
    # held-out: the network's output is closer to the EM label than its own FBP input
    x, y = inputs[80:].contiguous(), labels[80:].contiguous()
    sc = ws.input_scale(x)
    out = net.forward(x, sc)
    mse_net = float(((out - y * sc[:, None, None]) ** 2).mean())
    mse_fbp = float((((x - y) * sc[:, None, None]) ** 2).mean())
    assert mse_net < 0.8 * mse_fbp, (mse_net, mse_fbp)
    r = ws.evaluate(net, inputs[80:], trans[80:], ang, plain_iters=40, max_warm_iters=40)
    # the trained network's start is closer to the data than the uniform start,
    # and reaches the plain-EM target residual in fewer iterations
    assert r["residual_start_warm_median"] < r["residual_start_plain_median"]
    assert r["warm_iterations_median"] < r["plain_iterations"]


def test_shipped_weights_reach_plain_em100_residual():
    """The shipped network (512^2 x 720 angles) on held-out seeds: its start
    is within 1% of the plain 100-iteration EM residual after at most two EM
    iterations, and FBP + U-Net + those iterations take at least 4x less
    device time than plain EM-100."""
    import os
    import torch
    from sscRaft import synthetic as S
    from sscRaft import warmstart as ws
    dev = torch.device("cuda", 0)
    assert os.path.exists(ws.default_weights())
    net = ws.UNet.from_file(ws.default_weights(), dev)
    assert 1.9e6 < net.n_params() < 2.1e6
    n = 16
    trans = torch.empty((n, 720, 512), dtype=torch.float32, device=dev)
    ws.make_transmissions(n, ws.HELDOUT_SEED0 + 1000, dev, chunk=n, out=trans)
    r = ws.evaluate_wall(net, trans, S.uniform_angles(720), max_iters=20)
    assert r["all_reached"] and r["learned_iterations_max"] <= 2, r
    assert r["residual_start_learned_median"] < r["residual_start_fbp_median"], r
    assert r["speedup_learned_vs_plain"] >= 4.0, r
