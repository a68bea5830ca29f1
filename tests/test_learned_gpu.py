"""Learned warm start: the whole U-Net's forward pass and parameter gradients on the tcgen05 kernels
against a float64 CPU reference of the same network (torch autograd on the same BF16-rounded
weights and input), and a short training run on solver-generated data."""

import numpy as np
import pytest
import torch
import torch.nn.functional as F

from continuum_liquid_b200 import learned, scenes

pytestmark = pytest.mark.gpu


def reference_unet(net, x0, target, mask):
    """float64 CPU restatement of learned.UNet.forward and its loss."""
    P = net.params.detach().cpu().double()
    params = {}
    for name, cin, cout in learned.LAYERS:
        o, rows, cols = net.w[name]
        w = P[o : o + rows * cols].view(3, 3, 3, cin, cout).to(torch.bfloat16).double()  # convs use BF16 weights
        w = w.permute(4, 3, 0, 1, 2).contiguous().requires_grad_(True)
        ob, c = net.b[name]
        params[name] = (w, P[ob : ob + c].clone().requires_grad_(True))
    o, c = net.head_w
    hw = P[o : o + c].clone().requires_grad_(True)
    hb = P[net.head_b[0] : net.head_b[0] + 1].clone().requires_grad_(True)

    def conv(x, name):
        w, b = params[name]
        return torch.relu(F.conv3d(x, w, b, padding=1))

    x = x0.double().permute(0, 4, 1, 2, 3)
    c1 = conv(x, "enc0a")
    e0 = conv(c1, "enc0b")
    c3 = conv(F.avg_pool3d(e0, 2), "enc1a")
    e1 = conv(c3, "enc1b")
    c5 = conv(F.avg_pool3d(e1, 2), "enc2a")
    e2 = conv(c5, "enc2b")
    u1 = torch.cat([F.interpolate(e2, scale_factor=2, mode="nearest"), e1], 1)
    d1 = conv(conv(u1, "dec1a"), "dec1b")
    u0 = torch.cat([F.interpolate(d1, scale_factor=2, mode="nearest"), e0], 1)
    d0 = conv(conv(u0, "dec0a"), "dec0b")
    out = (d0 * hw.view(1, -1, 1, 1, 1)).sum(1) + hb
    out = out.reshape(-1)
    m = mask.double()
    loss = (((out - target.double()) * m) ** 2).sum() / m.sum()
    loss.backward()
    grads = {name: (w.grad, b.grad) for name, (w, b) in params.items()}
    return out.detach(), loss.item(), grads, hw.grad, hb.grad


def test_unet_forward_and_gradients_match_float64_reference(backend):
    torch.manual_seed(0)
    net = learned.UNet(backend, seed=3)
    o, c = net.head_w  # a nonzero head so every layer's gradient is exercised
    net.params[o : o + c] = torch.randn(c, device="cuda") * 0.25
    vol = learned.Vol(2, 8, 8, 12)
    bufs = net.buffers(vol)
    x0 = torch.zeros(vol.voxels, 8)
    x0[:, :4] = torch.randn(vol.voxels, 4)
    x0 = x0.to(torch.bfloat16)
    bufs["x0"].copy_(x0.cuda())
    target = torch.randn(vol.voxels)
    mask = (torch.rand(vol.voxels) < 0.7).float()
    bufs["target"].copy_(target.cuda())
    bufs["mask"].copy_(mask.cuda())
    out = net.forward(vol)
    loss = net.loss_and_grad(vol)
    net.backward(vol)
    torch.cuda.synchronize()
    ref_out, ref_loss, ref_grads, ref_hw, ref_hb = reference_unet(net, x0.view(2, 8, 8, 12, 8), target, mask)
    got = out.cpu().double()
    assert torch.linalg.norm(got - ref_out) <= 0.03 * torch.linalg.norm(ref_out)
    assert loss.item() == pytest.approx(ref_loss, rel=0.05)
    G = net.grads.cpu().double()
    for name, cin, cout in learned.LAYERS:
        o, rows, cols = net.w[name]
        g = G[o : o + rows * cols].view(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2)
        r = ref_grads[name][0]
        cos = torch.nn.functional.cosine_similarity(g.reshape(-1), r.reshape(-1), dim=0).item()
        assert cos > 0.99, (name, cos)
        assert torch.linalg.norm(g - r) <= 0.1 * torch.linalg.norm(r), name
        ob, c = net.b[name]
        assert torch.linalg.norm(G[ob : ob + c] - ref_grads[name][1]) <= 0.1 * torch.linalg.norm(ref_grads[name][1]) + 1e-6
    o, c = net.head_w
    assert torch.linalg.norm(G[o : o + c] - ref_hw) <= 0.05 * torch.linalg.norm(ref_hw)
    assert backend.device_error() == 0


def test_training_on_solver_frames_reduces_loss_and_reports_gain(backend):
    """Train briefly on solves of one dam break, evaluate the warm start on another seed: the loss
    must drop, and with the fallback rule the learned guess is only used where it is better."""
    train_frames = learned.capture_frames(backend, scenes.dam_break(48, seed=0), steps=12)
    test_frames = learned.capture_frames(backend, scenes.dam_break(48, seed=100), steps=8)
    net = learned.UNet(backend, seed=0)
    untrained = learned.LearnedWarmStart(net, test_frames[0].rhs.shape, test_frames[0].dx)
    f0 = test_frames[0]
    assert torch.equal(untrained(f0.rhs, f0.op0, f0.solid, f0.p_prev), f0.p_prev * ((f0.op0 & 64) != 0))
    history = learned.train(net, train_frames, iterations=120, batch=4, crop=32, log_every=10)
    assert history[-1] < 0.5 * history[0]
    ws = learned.LearnedWarmStart(net, test_frames[0].rhs.shape, test_frames[0].dx)
    from continuum_liquid_b200.pressure_solve import PressureSolver

    ps = PressureSolver(backend, test_frames[0].rhs.shape, test_frames[0].dx, autotune=False)
    gains = []
    for f in test_frames:
        ps.rhs.copy_(f.rhs)
        ps.hierarchy.op0.copy_(f.op0)
        rel_prev = ps.relative_residual(f.p_prev)
        rel_net = ps.relative_residual(ws(f.rhs, f.op0, f.solid, f.p_prev))
        gains.append(rel_prev / rel_net)
    assert all(np.isfinite(gains))
    print("initial residual ratio previous/learned per test frame:", [round(g, 3) for g in gains])
