"""tcgen05 3-D convolutions (forward, data gradient, weight gradient) against a float64 CPU
reference (torch conv3d and autograd on the same BF16-rounded inputs)."""

import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def kpad(k):
    return (k + 63) // 64 * 64


def torch_weight(w, cin, cout):
    # w[tap * cin + ci][co], tap = (dz+1)*9 + (dy+1)*3 + (dx+1)  ->  [co][ci][kz][ky][kx]
    return w.view(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2).contiguous()


@pytest.mark.parametrize("B,D,H,W,cin,cout", [(1, 6, 8, 10, 8, 16), (2, 5, 7, 9, 16, 32), (1, 8, 8, 8, 32, 64),
                                             (1, 4, 6, 8, 96, 32), (2, 4, 4, 6, 48, 16)])
def test_conv3d_forward_and_gradients(backend, B, D, H, W, cin, cout):
    g = torch.Generator().manual_seed(B * 1000 + cin * 10 + cout)
    x = torch.randn(B, D, H, W, cin, generator=g).to(torch.bfloat16)
    w = (torch.randn(27 * cin, cout, generator=g) * (2.0 / (27 * cin)) ** 0.5).to(torch.bfloat16).float()
    bias = torch.randn(cout, generator=g) * 0.1
    dy = torch.randn(B, D, H, W, cout, generator=g).to(torch.bfloat16)
    V = B * D * H * W
    kp, kp2 = kpad(27 * cin), kpad(27 * cout)
    dev = "cuda"
    xd, wd_, bd, dyd = x.to(dev), w.to(dev), bias.to(dev), dy.to(dev)
    wf = torch.empty(cout, kp, dtype=torch.bfloat16, device=dev)
    wdm = torch.empty(cin, kp2, dtype=torch.bfloat16, device=dev)
    backend.call("clb_conv3d_arrange_weights", wd_, wf, wdm, cin, cout, kp, kp2)
    y = torch.empty(B, D, H, W, cout, dtype=torch.bfloat16, device=dev)
    backend.call("clb_conv3d_forward", xd, wf, bd, y, B, D, H, W, cin, cout, kp, 1)
    # float64 reference
    xr = x.double().permute(0, 4, 1, 2, 3).contiguous().requires_grad_(True)
    wr = torch_weight(w.double(), cin, cout).requires_grad_(True)
    pre = F.conv3d(xr, wr, bias.double(), padding=1)
    yr = torch.relu(pre)
    torch.cuda.synchronize()
    got = y.float().cpu().permute(0, 4, 1, 2, 3)
    scale = yr.abs().max().item()
    torch.testing.assert_close(got.double(), yr.detach(), rtol=2e-2, atol=1e-2 * scale)
    # gradients of sum(pre * dy): data gradient (no mask) and weight gradient
    pre.backward(dy.double().permute(0, 4, 1, 2, 3))
    if cin % 16 == 0:
        dx = torch.empty(B, D, H, W, cin, dtype=torch.bfloat16, device=dev)
        backend.call("clb_conv3d_dgrad", dyd, wdm, None, dx, B, D, H, W, cout, cin, kp2)
        torch.cuda.synchronize()
        ref = xr.grad.permute(0, 2, 3, 4, 1)
        torch.testing.assert_close(dx.float().cpu().double(), ref, rtol=2e-2, atol=1e-2 * ref.abs().max().item())
        # with the ReLU mask of the input activation
        dxm = torch.empty_like(dx)
        backend.call("clb_conv3d_dgrad", dyd, wdm, xd, dxm, B, D, H, W, cout, cin, kp2)
        torch.cuda.synchronize()
        refm = ref * (x.double() > 0)
        torch.testing.assert_close(dxm.float().cpu().double(), refm, rtol=2e-2, atol=1e-2 * ref.abs().max().item())
    dw = torch.zeros(27 * cin, cout, device=dev)
    backend.call("clb_conv3d_wgrad", xd, dyd, dw, B, D, H, W, cin, cout, 3)
    torch.cuda.synchronize()
    refw = wr.grad.permute(2, 3, 4, 1, 0).reshape(27 * cin, cout)
    torch.testing.assert_close(dw.cpu().double(), refw, rtol=1e-3, atol=1e-3 * refw.abs().max().item())
    assert backend.device_error() == 0
