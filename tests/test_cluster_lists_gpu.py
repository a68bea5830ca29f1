"""The fluid-cell lists of the cluster visit (clb_mg_hierarchy.cluster_lists), built once per solve by
clb_mg_build_coarse: their entries equal a numpy enumeration of each CTA's fluid cells of each colour in
slot order, and W-cycles that take them equal W-cycles whose launches list the cells themselves, bit
for bit, in FP32 and FP16 storage."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import multigrid

pytestmark = pytest.mark.gpu

F32 = np.float32
CLUSTER_MAX = 16  # CTAs per cluster launch


def liquid_system(shape, seed):
    rng = np.random.default_rng(seed)
    ff = np.zeros(shape, F32)
    ff[1:-1, 1 : shape[1] // 2 + 2, 1:-1] = 1.0
    ff[rng.random(shape) < 0.05] = 0
    ff[[0, -1]] = 0
    ff[:, [0, -1]] = 0
    ff[:, :, [0, -1]] = 0
    vel = [torch.from_numpy(rng.standard_normal(shape).astype(F32)).cuda() for _ in range(3)]
    return torch.from_numpy(ff).cuda(), vel


def colour_cells(colour, nx, ny, nz):
    """Grid indices of the interior cells of one colour in slot order (mg_bottom.cuh colour_cell)."""
    half, my = (nz - 1) // 2, ny - 2
    out = []
    for r in range((nx - 2) * my * half):
        row, s = divmod(r, half)
        i, j = 1 + row // my, 1 + row % my
        k = 1 + 2 * s + ((i + j + 1 + colour) & 1)
        if i <= nx - 2 and k <= nz - 2:
            out.append((i * ny + j) * nz + k)
    return np.asarray(out, np.int64)


def diagonal(h, level):
    """The diagonal a launch stages: the operator's, -1 where the cell is not fluid."""
    d = h.op[level].reshape(-1, 4)[:, 0].float().cpu().numpy()
    m = h.mask[level].reshape(-1).cpu().numpy()
    return np.where(m != 0, d, -1.0)


def expected_lists(h):
    """The lists k_cluster_lists writes, from the staged diagonals on the host."""
    lc, la, lb = h.levels - 3, h.levels - 2, h.levels - 1
    (nx, ny, nz), sa, sb = h.shapes[lc], h.shapes[la], h.shapes[lb]
    CA, CB = int(np.prod(sa)), int(np.prod(sb))
    pairs = (nx - 1) // 2
    cs = min(pairs, CLUSTER_MAX - 1)
    own_max = 2 * ((pairs + cs - 1) // cs)
    list_len = own_max * ny * nz // 2 + 1
    bottom_ints = (4 + 2 * (CA // 2 + 1) + 2 * (CB // 2 + 1) + 3) & ~3
    slab_ints = (2 * list_len + 2 + 3) & ~3
    da, db, dc = diagonal(h, la), diagonal(h, lb), diagonal(h, lc)
    parts = {}
    for colour in range(2):
        a = colour_cells(colour, *sa)
        parts[("a", colour)] = a[da[a] >= 0]
        b = colour_cells(colour, *sb)
        parts[("b", colour)] = b[db[b] >= 0]
    for s in range(cs):
        p0, p1 = s * pairs // cs, (s + 1) * pairs // cs
        i_lo, i_hi = 2 * p0 + 1, min(2 * p1 + 1, nx - 1)
        np_, flip = i_hi - i_lo + 2, (i_lo - 1) & 1
        for colour in range(2):
            c = colour_cells(colour ^ flip, np_, ny, nz)
            parts[(s, colour)] = c[dc[(i_lo - 1) * ny * nz + c] >= 0]
    return parts, dict(CA=CA, CB=CB, cs=cs, list_len=list_len, bottom_ints=bottom_ints, slab_ints=slab_ints)


@pytest.mark.parametrize("fp16", [False, True])
@pytest.mark.parametrize("shape", [(130, 130, 130), (126, 125, 121)])
def test_cluster_lists_enumerate_the_fluid_cells(backend, shape, fp16):
    h = multigrid.MultigridHierarchy(backend, shape, 1.0 / shape[0], fp16_max_size=64 if fp16 else 0)
    assert h.cluster_lists is not None
    ff, vel = liquid_system(shape, 17)
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator(vel, ff, rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    got = h.cluster_lists.cpu().numpy()
    parts, g = expected_lists(h)
    assert len(got) == g["bottom_ints"] + g["cs"] * g["slab_ints"]
    la, lb = g["CA"] // 2 + 1, g["CB"] // 2 + 1
    for colour in range(2):
        a, b = parts[("a", colour)], parts[("b", colour)]
        assert got[colour] == len(a) and got[2 + colour] == len(b)
        off_a = 4 + colour * la
        assert np.array_equal(got[off_a : off_a + len(a)], a), ("A", colour)
        off_b = 4 + 2 * la + colour * lb
        assert np.array_equal(got[off_b : off_b + len(b)], b), ("B", colour)
    for s in range(g["cs"]):
        base = g["bottom_ints"] + s * g["slab_ints"]
        for colour in range(2):
            c = parts[(s, colour)]
            assert got[base + 2 * g["list_len"] + colour] == len(c), (s, colour)
            off = base + colour * g["list_len"]
            assert np.array_equal(got[off : off + len(c)], c), (s, colour)
    assert sum(len(parts[(s, 0)]) for s in range(g["cs"])) > 0
    assert backend.device_error() == 0


@pytest.mark.parametrize("fp16", [False, True])
@pytest.mark.parametrize("shape", [(130, 130, 130), (126, 125, 121)])
def test_w_cycles_with_and_without_prebuilt_lists(backend, shape, fp16):
    """A launch that lists its cells itself (cluster_lists NULL) and one that takes the lists built
    once per solve give the same W-cycles bit for bit (cells of one colour are independent)."""
    h = multigrid.MultigridHierarchy(backend, shape, 1.0 / shape[0], fp16_max_size=64 if fp16 else 0)
    ff, vel = liquid_system(shape, 19)
    rhs = torch.zeros(shape, dtype=torch.float32, device="cuda")
    h.rhs_operator(vel, ff, rhs, 1.0 / 240.0, 1000.0)
    h.build_coarse()
    h.residual_norms(torch.zeros_like(rhs), rhs)
    lists = h.struct.cluster_lists
    out = []
    try:
        for use in (True, False):
            h.struct.cluster_lists = lists if use else None
            e = torch.zeros_like(rhs)
            for _ in range(2):
                h.w_cycle(e, rhs)
            out.append(e)
    finally:
        h.struct.cluster_lists = lists
    assert torch.equal(out[0], out[1])
    assert out[0].abs().max() > 0
    assert backend.device_error() == 0
