"""The allocation-free scan entry point against the scan that takes caller scratch.

clb_exclusive_prefix_sum_static serves callers that cannot allocate device memory (their host
application owns the whole device memory budget, or a cudaMalloc would add a device-wide
synchronisation to work in flight): its look-back scratch is a fixed array inside the library. This
file runs last (pytest collects it after the other test files), through the C ABI, and works both
alone in a fresh process and after the rest of the suite.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LIMIT = 67108864  # CLB_SCAN_STATIC_MAX_COUNT


def scan_with_scratch(backend, values):
    n = values.numel()
    out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")[:n]
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    scratch = torch.zeros(backend.scan_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    backend.call("clb_exclusive_prefix_sum", values, out, total, n, scratch, scratch.numel())
    return out, total


def scan_static(backend, values):
    n = values.numel()
    out = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")[:n]
    total = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    backend.call("clb_exclusive_prefix_sum_static", values, out, total, n)
    return out, total


def test_static_scan_matches_scratch_scan_on_two_calls(backend):
    rng = np.random.default_rng(2024)
    # two calls in a row: a large scan, then a smaller one over different values, so look-back state
    # left by the first call would corrupt the second if the array were not cleared
    for n in (16777216 + 77, 100003):
        values = torch.from_numpy(rng.integers(0, 9, n).astype(np.int32)).cuda()
        got, got_total = scan_static(backend, values)
        want, want_total = scan_with_scratch(backend, values)
        torch.cuda.synchronize()
        assert torch.equal(got, want)
        assert int(got_total.item()) == int(want_total.item()) == int(values.sum().item())
    assert backend.device_error() == 0


def test_static_scan_rejects_counts_above_its_limit(backend):
    values = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(RuntimeError, match="fixed scratch limit"):
        backend.call("clb_exclusive_prefix_sum_static", values, values, None, LIMIT + 1)
