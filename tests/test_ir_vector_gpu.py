"""The FP64 pressure init and store of the mixed-precision solve, four cells per thread: on a grid
whose rows are a multiple of 4 cells with aligned buffers (the vector kernels) they write the same
values as the one-cell kernels (forced by buffers offset by one element) and as numpy: p64 = p32 at
interior cells whose operator byte has the fluid bit (64), 0 elsewhere; p32 = (float) p64."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def expected_init(p32, op0):
    nx, ny, nz = p32.shape
    interior = np.zeros(p32.shape, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    return np.where(interior & ((op0 & 64) != 0), p32.astype(np.float64), 0.0)


@pytest.mark.parametrize("shape", [(34, 30, 40), (12, 9, 8)])
def test_ir_init_vector_and_scalar_paths(backend, shape):
    rng = np.random.default_rng(5)
    C = int(np.prod(shape))
    p32 = rng.standard_normal(shape).astype(np.float32)
    op0 = rng.integers(0, 256, size=shape, dtype=np.uint8)
    want = expected_init(p32, op0)
    dev = "cuda"
    # aligned, rows of 4k cells: the vector kernel
    p_d = torch.from_numpy(p32).to(dev)
    op_d = torch.from_numpy(op0).to(dev)
    out_v = torch.full(shape, np.nan, dtype=torch.float64, device=dev)
    backend.call("clb_mg_ir_init", p_d, op_d, out_v, *shape)
    # the same data one element into larger buffers: not 16-byte aligned, so the one-cell kernel
    p_off = torch.zeros(C + 1, dtype=torch.float32, device=dev)
    p_off[1:] = p_d.reshape(-1)
    out_off = torch.full((C + 1,), np.nan, dtype=torch.float64, device=dev)
    backend.call("clb_mg_ir_init", p_off[1:], op_d, out_off[1:], *shape)
    torch.cuda.synchronize()
    assert np.array_equal(out_v.cpu().numpy(), want)
    assert np.array_equal(out_off[1:].cpu().numpy().reshape(shape), want)
    assert backend.device_error() == 0


@pytest.mark.parametrize("cells", [34 * 30 * 40, 4 * 1001, 4 * 1001 + 3])
def test_ir_store_vector_and_scalar_paths(backend, cells):
    rng = np.random.default_rng(6)
    p64 = rng.standard_normal(cells) * np.exp(rng.uniform(-30, 30, cells))
    want = p64.astype(np.float32)
    dev = "cuda"
    src = torch.from_numpy(p64).to(dev)
    out_v = torch.full((cells,), np.nan, dtype=torch.float32, device=dev)
    backend.call("clb_mg_ir_store", src, out_v, cells)
    src_off = torch.zeros(cells + 1, dtype=torch.float64, device=dev)
    src_off[1:] = src
    out_off = torch.full((cells + 1,), np.nan, dtype=torch.float32, device=dev)
    backend.call("clb_mg_ir_store", src_off[1:], out_off[1:], cells)
    torch.cuda.synchronize()
    assert np.array_equal(out_v.cpu().numpy(), want)
    assert np.array_equal(out_off[1:].cpu().numpy(), want)
    assert backend.device_error() == 0
