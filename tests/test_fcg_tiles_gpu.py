"""The FCG dots and the refinement / FCG steps on the level-0 fluid tiles (csrc/mg_fcg_tiles.cuh) against
the row kernels: per cell the same pressure, direction and residual bit for bit, the sums equal up to
their FP64 summation order, and the same sums on every run."""

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import multigrid

pytestmark = pytest.mark.gpu

F32 = np.float32


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def system(backend, shape, seed):
    rng = np.random.default_rng(seed)
    ff = np.zeros(shape, F32)
    nx, ny, nz = shape
    ff[1 : (3 * nx) // 4, 1 : (2 * ny) // 3, 1 : nz - 1] = 1.0
    ff[rng.random(shape) < 0.05] = 0
    u, v, w = (rng.standard_normal(shape).astype(F32) for _ in range(3))
    dx = F32(1.0 / nx)
    h = multigrid.MultigridHierarchy(backend, shape, float(dx))
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator((dev(u), dev(v), dev(w)), dev(ff), rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    fluid = (host(h.op0) & 64) != 0
    interior = np.zeros(shape, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    live = fluid & interior

    def field(scale, dtype=np.float32):
        return dev((rng.standard_normal(shape) * scale * live).astype(dtype))

    return h, rhs, live, field


@pytest.mark.parametrize("shape", [(64, 48, 128), (40, 36, 44), (33, 30, 70)])
def test_tile_step_and_dots_match_rows(backend, shape):
    h, rhs, live, field = system(backend, shape, 71)
    assert int(h.tile_counts[0].item()) > 0
    listed = host(h.tiles[0])[: int(h.tile_counts[0].item())]
    assert np.all(np.diff(listed) > 0)  # ascending: the sums' order is fixed
    delta = float(F32(1.0 / shape[0]))
    cells = int(np.prod(shape))
    blocks = backend.residual_partials(cells)
    z, d, r = field(1.0), field(0.5), field(2.0)
    p_in = field(3.0, np.float64)
    state = torch.tensor([0.7, -0.3, 5.0, 1.0], dtype=torch.float64, device="cuda")

    # the scalars the steps use: the row dots' (each path's own dots differ in the last bits)
    common = state.clone()
    part4 = torch.zeros(4 * blocks, dtype=torch.float64, device="cuda")
    backend.call("clb_mg_fcg_dots", z, d, r, h.op0, delta, *shape, part4, common)

    def outputs(tiles: bool):
        p_out = torch.zeros(shape, dtype=torch.float64, device="cuda")
        d_out = torch.zeros(shape, dtype=torch.float32, device="cuda")
        r_out = torch.zeros(shape, dtype=torch.float32, device="cuda")
        part = torch.zeros((blocks, 2), dtype=torch.float64, device="cuda")
        part4 = torch.zeros(4 * blocks, dtype=torch.float64, device="cuda")
        out = torch.zeros(2, dtype=torch.float64, device="cuda")
        st = state.clone()
        if tiles:
            backend.call_hierarchy("clb_mg_fcg_dots_tiles", h.struct, z, d, r, part4, st)
            backend.call_hierarchy("clb_mg_fcg_step_tiles", h.struct, p_in, z, d, p_out, d_out, common, rhs, r_out,
                                   part, out)
        else:
            backend.call("clb_mg_fcg_dots", z, d, r, h.op0, delta, *shape, part4, st)
            backend.call("clb_mg_fcg_step", p_in, z, d, p_out, d_out, common, rhs, h.op0, delta, *shape, r_out, part,
                         out)
        ir_out = torch.zeros(shape, dtype=torch.float64, device="cuda")
        ir_r = torch.zeros(shape, dtype=torch.float32, device="cuda")
        ir_norms = torch.zeros(2, dtype=torch.float64, device="cuda")
        if tiles:
            backend.call_hierarchy("clb_mg_ir_step_tiles", h.struct, p_in, z, ir_out, rhs, ir_r, part, ir_norms)
        else:
            backend.call("clb_mg_ir_step", p_in, z, ir_out, rhs, h.op0, delta, *shape, ir_r, part, ir_norms)
        return [host(x) for x in (st, p_out, d_out, r_out, out, ir_out, ir_r, ir_norms)]

    rows = outputs(False)
    tiles = outputs(True)
    again = outputs(True)
    for a, b in zip(tiles, again):
        assert np.array_equal(a, b)  # the same on every run
    for k in (1, 2, 3, 5, 6):  # per-cell values: bit for bit
        assert np.array_equal(tiles[k], rows[k]), k
    for k in (0, 4, 7):  # FP64 sums: another summation order
        np.testing.assert_allclose(tiles[k], rows[k], rtol=1e-12, atol=0)
    assert np.abs(tiles[3][~live]).max() == 0
    assert backend.device_error() == 0
