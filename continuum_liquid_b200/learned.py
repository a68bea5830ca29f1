"""Learned warm start for the pressure solve (no counterpart in the reference).

A 3-level 3-D U-Net (channels 16/32/64, 3x3x3 convolutions with ReLU, 2x2x2 average pooling,
nearest upsampling with skip concatenation, a 1x1x1 output head; ~0.36M parameters) maps
(divergence right-hand side, liquid mask, solid mask, previous-step pressure) to the change of the
pressure since the previous step. The guess is p = p_prev + s * out, formed in FP32 so that the
previous pressure keeps its precision; the head starts at zero, so the untrained network returns
p_prev exactly.
Every convolution runs on the library's BF16 implicit-GEMM kernels on tcgen05 with FP32
accumulation (forward, data gradient and weight gradient); training uses Adam on FP32 master
weights. Inputs and the target are normalised per sample by s = max |previous pressure| over the
liquid: channel 0 is b * dx^2 / s, channel 3 is p_prev / s, the target is (p - p_prev) / s.

The solver uses the network's pressure as the initial guess of the FP64-refined W-cycles only when
its relative residual is below that of the previous-step pressure; the same tolerance judges every
solve, so only the cycle count changes.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from .backend import Backend

LAYERS = [
    ("enc0a", 8, 16),
    ("enc0b", 16, 16),
    ("enc1a", 16, 32),
    ("enc1b", 32, 32),
    ("enc2a", 32, 64),
    ("enc2b", 64, 64),
    ("dec1a", 96, 32),
    ("dec1b", 32, 32),
    ("dec0a", 48, 16),
    ("dec0b", 16, 16),
]
HEAD_C = 16
BF16 = torch.bfloat16


def kpad(k: int) -> int:
    return (k + 63) // 64 * 64


@dataclass
class Vol:
    B: int
    D: int
    H: int
    W: int

    @property
    def voxels(self) -> int:
        return self.B * self.D * self.H * self.W

    def half(self) -> "Vol":
        return Vol(self.B, self.D // 2, self.H // 2, self.W // 2)

    def args(self):
        return (self.B, self.D, self.H, self.W)


class UNet:
    """Parameters, Adam state and per-shape activation buffers of the warm-start network."""

    def __init__(self, kernels: Backend, seed: int = 0):
        self.k = kernels
        dev = kernels.device
        sizes = []
        for _, cin, cout in LAYERS:
            sizes += [27 * cin * cout, cout]
        sizes += [HEAD_C, 1]
        self.n_params = int(sum(sizes))
        self.params = torch.zeros(self.n_params, dtype=torch.float32, device=dev)
        self.grads = torch.zeros_like(self.params)
        self.adam_m = torch.zeros_like(self.params)
        self.adam_v = torch.zeros_like(self.params)
        self.step_count = 0
        self.w, self.b = {}, {}
        off = 0
        for name, cin, cout in LAYERS:
            self.w[name] = (off, 27 * cin, cout)
            off += 27 * cin * cout
            self.b[name] = (off, cout)
            off += cout
        self.head_w = (off, HEAD_C)
        off += HEAD_C
        self.head_b = (off, 1)
        gen = torch.Generator().manual_seed(seed)
        init = torch.zeros(self.n_params)
        for name, cin, cout in LAYERS:
            o, rows, cols = self.w[name]
            init[o : o + rows * cols] = torch.randn(rows * cols, generator=gen) * math.sqrt(2.0 / (27 * cin))
        self.params.copy_(init)  # head weights and biases start at zero
        # BF16 operand matrices of every convolution
        self.wf, self.wd = {}, {}
        for name, cin, cout in LAYERS:
            self.wf[name] = torch.zeros((cout, kpad(27 * cin)), dtype=BF16, device=dev)
            self.wd[name] = torch.zeros((cin, kpad(27 * cout)), dtype=BF16, device=dev) if name != "enc0a" else None
        self.arrange()
        self._buffers: dict[tuple, dict] = {}
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)

    # -- parameter views ---------------------------------------------------------------------------
    def _view(self, t, entry):
        o = entry[0]
        n = int(np.prod(entry[1:]))
        return t[o : o + n]

    def weight(self, name):
        return self._view(self.params, self.w[name])

    def bias(self, name):
        return self._view(self.params, self.b[name])

    def arrange(self) -> None:
        """Rebuild the BF16 operand matrices from the FP32 master weights."""
        for name, cin, cout in LAYERS:
            self.k.call("clb_conv3d_arrange_weights", self.weight(name), self.wf[name], self.wd[name], cin, cout,
                        kpad(27 * cin), kpad(27 * cout))

    # -- buffers -----------------------------------------------------------------------------------
    def buffers(self, vol: Vol) -> dict:
        key = vol.args()
        if key not in self._buffers:
            if vol.D % 4 or vol.H % 4 or vol.W % 4:
                raise ValueError("U-Net volumes need extents divisible by 4")
            dev = self.k.device
            v0, v1, v2 = vol.voxels, vol.half().voxels, vol.half().half().voxels
            spec = {
                "x0": (v0, 8), "c1": (v0, 16), "e0": (v0, 16), "p1": (v1, 16), "c3": (v1, 32), "e1": (v1, 32),
                "p2": (v2, 32), "c5": (v2, 64), "e2": (v2, 64), "u1": (v1, 96), "d1a": (v1, 32), "d1": (v1, 32),
                "u0": (v0, 48), "d0a": (v0, 16), "d0": (v0, 16),
                "dd0": (v0, 16), "dd0a": (v0, 16), "du0": (v0, 48), "dd1": (v1, 32), "de0": (v0, 16),
                "dd1a": (v1, 32), "du1": (v1, 96), "de2": (v2, 64), "de1": (v1, 32), "dc5": (v2, 64),
                "dp2": (v2, 32), "dc3": (v1, 32), "dp1": (v1, 16), "dc1": (v0, 16),
            }
            bufs = {n: torch.zeros(shape, dtype=BF16, device=dev) for n, shape in spec.items()}
            bufs["out"] = torch.zeros(v0, dtype=torch.float32, device=dev)
            bufs["dout"] = torch.zeros(v0, dtype=torch.float32, device=dev)
            bufs["target"] = torch.zeros(v0, dtype=torch.float32, device=dev)
            bufs["mask"] = torch.zeros(v0, dtype=torch.float32, device=dev)
            self._buffers[key] = bufs
        return self._buffers[key]

    # -- forward / backward ------------------------------------------------------------------------
    def _conv(self, x, name, y, vol: Vol, relu=1):
        _, cin, cout = next(l for l in LAYERS if l[0] == name)
        self.k.call("clb_conv3d_forward", x, self.wf[name], self.bias(name), y, *vol.args(), cin, cout,
                    kpad(27 * cin), relu)

    def forward(self, vol: Vol) -> torch.Tensor:
        """Run the network on buffers(vol)['x0']; returns the FP32 output [B*D*H*W]."""
        b = self.buffers(vol)
        v1, v2 = vol.half(), vol.half().half()
        k = self.k
        self._conv(b["x0"], "enc0a", b["c1"], vol)
        self._conv(b["c1"], "enc0b", b["e0"], vol)
        k.call("clb_unet_avgpool2", b["e0"], b["p1"], *vol.args(), 16)
        self._conv(b["p1"], "enc1a", b["c3"], v1)
        self._conv(b["c3"], "enc1b", b["e1"], v1)
        k.call("clb_unet_avgpool2", b["e1"], b["p2"], *v1.args(), 32)
        self._conv(b["p2"], "enc2a", b["c5"], v2)
        self._conv(b["c5"], "enc2b", b["e2"], v2)
        k.call("clb_unet_upsample_concat", b["e2"], b["e1"], b["u1"], *v1.args(), 64, 32)
        self._conv(b["u1"], "dec1a", b["d1a"], v1)
        self._conv(b["d1a"], "dec1b", b["d1"], v1)
        k.call("clb_unet_upsample_concat", b["d1"], b["e0"], b["u0"], *vol.args(), 32, 16)
        self._conv(b["u0"], "dec0a", b["d0a"], vol)
        self._conv(b["d0a"], "dec0b", b["d0"], vol)
        k.call("clb_unet_head_forward", b["d0"], self._view(self.params, self.head_w),
               self._view(self.params, self.head_b), b["out"], vol.voxels, HEAD_C)
        return b["out"]

    def _layer_backward(self, name, x, dy, dx, vol: Vol, mask=True):
        _, cin, cout = next(l for l in LAYERS if l[0] == name)
        k = self.k
        chunks = (vol.voxels + 63) // 64
        mtiles = (27 * cin + 127) // 128
        per_block = max(1, (chunks * mtiles) // (148 * 8))
        k.call("clb_conv3d_wgrad", x, dy, self._view(self.grads, self.w[name]), *vol.args(), cin, cout, per_block)
        k.call("clb_unet_bias_grad", dy, self._view(self.grads, self.b[name]), vol.voxels, cout)
        if dx is not None:
            k.call("clb_conv3d_dgrad", dy, self.wd[name], x if mask else None, dx, *vol.args(), cout, cin,
                   kpad(27 * cout))

    def backward(self, vol: Vol) -> None:
        """Gradients of the loss whose output gradient is in buffers(vol)['dout'] (accumulated into a
        zeroed gradient buffer)."""
        b = self.buffers(vol)
        v1, v2 = vol.half(), vol.half().half()
        k = self.k
        self.grads.zero_()
        b["de0"].zero_()
        b["de1"].zero_()
        k.call("clb_unet_head_backward", b["d0"], self._view(self.params, self.head_w), b["dout"], b["dd0"],
               self._view(self.grads, self.head_w), self._view(self.grads, self.head_b), vol.voxels, HEAD_C)
        self._layer_backward("dec0b", b["d0a"], b["dd0"], b["dd0a"], vol)
        self._layer_backward("dec0a", b["u0"], b["dd0a"], b["du0"], vol)
        k.call("clb_unet_upsample_concat_backward", b["du0"], b["dd1"], b["de0"], *vol.args(), 32, 16)
        self._layer_backward("dec1b", b["d1a"], b["dd1"], b["dd1a"], v1)
        self._layer_backward("dec1a", b["u1"], b["dd1a"], b["du1"], v1)
        k.call("clb_unet_upsample_concat_backward", b["du1"], b["de2"], b["de1"], *v1.args(), 64, 32)
        self._layer_backward("enc2b", b["c5"], b["de2"], b["dc5"], v2)
        self._layer_backward("enc2a", b["p2"], b["dc5"], b["dp2"], v2, mask=False)
        k.call("clb_unet_avgpool2_backward", b["dp2"], b["e1"], b["de1"], *v1.args(), 32)
        self._layer_backward("enc1b", b["c3"], b["de1"], b["dc3"], v1)
        self._layer_backward("enc1a", b["p1"], b["dc3"], b["dp1"], v1, mask=False)
        k.call("clb_unet_avgpool2_backward", b["dp1"], b["e0"], b["de0"], *vol.args(), 16)
        self._layer_backward("enc0b", b["c1"], b["de0"], b["dc1"], vol)
        self._layer_backward("enc0a", b["x0"], b["dc1"], None, vol)

    def loss_and_grad(self, vol: Vol) -> torch.Tensor:
        """Masked MSE between out and target (buffers) -> dout; returns the device loss scalar."""
        b = self.buffers(vol)
        self.loss.zero_()
        count = float(b["mask"].sum().item()) or 1.0
        self.k.call("clb_unet_mse", b["out"], b["target"], b["mask"], b["dout"], self.loss, vol.voxels, 1.0 / count)
        return self.loss

    def adam_step(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step_count += 1
        self.k.call("clb_adam_step", self.params, self.grads, self.adam_m, self.adam_v, self.n_params, float(lr),
                    beta1, beta2, eps, self.step_count)
        self.arrange()

    # -- persistence -------------------------------------------------------------------------------
    def save(self, path, meta: dict | None = None) -> None:
        """FP32 master weights (and optional JSON metadata: how they were trained and evaluated)."""
        import json

        np.savez_compressed(path, params=self.params.cpu().numpy(), step=self.step_count,
                            meta=np.asarray(json.dumps(meta or {})))

    def load(self, path) -> None:
        data = np.load(path)
        self.params.copy_(torch.from_numpy(data["params"]).to(self.params.device))
        self.step_count = int(data["step"])
        self.arrange()


# ------------------------------------------------------------------------------------------------
# Inputs from the solver, training data, the warm start
# ------------------------------------------------------------------------------------------------
@dataclass
class Frame:
    """One solve: right-hand side, packed operator, solid mask, previous and converged pressure."""

    rhs: torch.Tensor
    op0: torch.Tensor
    solid: torch.Tensor | None
    p_prev: torch.Tensor
    p_conv: torch.Tensor
    dx: float
    scale: float
    weight: float = 1.0  # loss weight: the relative residual the previous-step pressure starts from


def pressure_scale(p: torch.Tensor, op0: torch.Tensor) -> float:
    fluid = (op0 & 64) != 0
    return float(p.abs().masked_fill(~fluid, 0).max().item())


def pack(net: UNet, vol: Vol, slot: int, rhs, op0, solid, p, dx, s, origin=(0, 0, 0), target=None) -> None:
    b = net.buffers(vol)
    nx, ny, nz = rhs.shape
    net.k.call("clb_unet_pack_input", rhs, op0, solid, p, float(dx * dx / s), float(1.0 / s), nx, ny, nz, *origin,
               b["x0"], slot, vol.D, vol.H, vol.W)
    if target is not None:
        net.k.call("clb_unet_pack_target", target, p, op0, float(1.0 / s), nx, ny, nz, *origin, b["target"],
                   b["mask"], slot, vol.D, vol.H, vol.W)


def capture_frames(kernels: Backend, scene, steps: int, tol: float = 1e-6, skip: int = 2) -> list[Frame]:
    """Run a scene with the plain solver (previous-step warm start, flexible CG to ``tol``) and record
    every solve after the first `skip`."""
    from .solver import StepOptions, scene_solver

    opts = StepOptions(flip_ratio=scene.flip_ratio, tol=tol, gravity=scene.gravity, rho=scene.rho, nu=scene.nu)
    sim = scene_solver(kernels, scene, opts)
    frames = []
    for step in range(steps):
        sim.pre_solve()
        p_prev = sim.pressure.clone()
        stats = sim.solve()
        ps = sim.pressure_solver
        if step >= skip:
            s = pressure_scale(p_prev, ps.hierarchy.op0)
            if s > 0:
                frames.append(Frame(ps.rhs.clone(), ps.hierarchy.op0.clone(),
                                    None if sim.obstacle is None else sim.obstacle, p_prev, sim.pressure.clone(),
                                    sim.dx, s, float(stats.initial_rel_residual or 1.0)))
        sim.post_solve()
    return frames


def train(net: UNet, frames: list[Frame], iterations: int, batch: int = 8, crop: int = 64, lr: float = 1e-3,
          seed: int = 0, log_every: int = 0, weighted: bool = False) -> list[float]:
    """Adam on random crops of the captured solves; returns the loss history. ``weighted`` scales each
    crop's squared error by its frame's weight (relative to the mean weight)."""
    rng = np.random.default_rng(seed)
    vol = Vol(batch, crop, crop, crop)
    b = net.buffers(vol)
    per_slot = vol.D * vol.H * vol.W
    mean_w = float(np.mean([f.weight for f in frames])) or 1.0
    history = []
    for it in range(iterations):
        for slot in range(batch):
            f = frames[int(rng.integers(len(frames)))]
            nx, ny, nz = f.rhs.shape
            origin = tuple(int(rng.integers(0, max(1, n - crop + 1))) for n in (nx, ny, nz))
            pack(net, vol, slot, f.rhs, f.op0, f.solid, f.p_prev, f.dx, f.scale, origin, target=f.p_conv)
            if weighted:
                b["mask"][slot * per_slot: (slot + 1) * per_slot].mul_(f.weight / mean_w)
        net.forward(vol)
        loss = net.loss_and_grad(vol)
        net.backward(vol)
        net.adam_step(lr)
        if log_every and (it % log_every == 0 or it == iterations - 1):
            history.append(float(loss.item()))
    return history


class LearnedWarmStart:
    """Callable used by the pressure solve: the network's pressure for the prepared system."""

    def __init__(self, net: UNet, grid_shape, dx: float):
        self.net = net
        self.grid_shape = tuple(int(s) for s in grid_shape)
        self.dx = float(dx)
        self.vol = Vol(1, *(((n + 3) // 4) * 4 for n in self.grid_shape))
        self.guess = torch.zeros(self.grid_shape, dtype=torch.float32, device=net.k.device)

    def __call__(self, rhs, op0, solid, p_prev) -> torch.Tensor | None:
        s = pressure_scale(p_prev, op0)
        if s <= 0.0:
            return None
        pack(self.net, self.vol, 0, rhs, op0, solid, p_prev, self.dx, s)
        out = self.net.forward(self.vol)
        nx, ny, nz = self.grid_shape
        self.net.k.call("clb_unet_unpack_output", out, p_prev, op0, float(s), self.guess, nx, ny, nz, self.vol.D,
                        self.vol.H, self.vol.W)
        return self.guess


def evaluate(kernels: Backend, net: UNet | None, frames: list[Frame], tol: float = 1e-6) -> list[dict]:
    """Flexible-CG cycles to ``tol`` on each captured system from the previous-step pressure and, with
    ``net``, from the solver's choice between it and the network's guess (the lower residual)."""
    from .autotune import tune_hierarchy
    from .pressure_solve import PressureSolver

    rows = []
    solvers: dict = {}
    for f in frames:
        shape = tuple(f.rhs.shape)
        if shape not in solvers:
            ps = PressureSolver(kernels, shape, f.dx)
            ws = LearnedWarmStart(net, shape, f.dx) if net is not None else None
            solvers[shape] = (ps, ws)
        ps, ws = solvers[shape]
        ps.rhs.copy_(f.rhs)
        ps.hierarchy.op0.copy_(f.op0)
        ps.hierarchy.build_coarse()
        if not ps.tuned:
            tune_hierarchy(ps.hierarchy, ps.correction, ps.residual)
            ps.tuned = True
        row = {"shape": shape}
        for name, warm in (("previous", None), ("learned", ws)):
            if name == "learned" and warm is None:
                continue
            p = f.p_prev.clone()
            st = ps.solve_prepared(p, tol, use_graph=False, warm_start=warm, solid=f.solid)
            row[name] = {"cycles": st.cycles, "initial_rel": st.initial_rel_residual, "guess": st.warm_start,
                         "learned_rel": st.learned_rel_residual}
        rows.append(row)
    return rows


def default_weights_path() -> Path:
    return Path(__file__).resolve().parent / "weights" / "warm_start_unet.npz"
