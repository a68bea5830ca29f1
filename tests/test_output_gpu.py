"""Particle cache writer: a device frame is written as it was when submitted, although the solver
thread does not wait for its copy and later work overwrites the device buffer."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from continuum_liquid_b200 import output

pytestmark = pytest.mark.gpu


def test_submitted_device_frames_keep_their_values(tmp_path):
    cache = output.create_cache(tmp_path, fps=24, start_frame=1, end_frame=8)
    writer = output.create_output(cache)
    n = 2_000_000
    dev = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    try:
        for frame in range(1, 8):
            dev.fill_(float(frame))
            dev[:, 1] += torch.arange(n, device="cuda", dtype=torch.float32) * 1e-3
            output.submit_output(writer, particles=dev, particle_count=n - frame, frame=frame)
            dev.mul_(-3.0)  # queued after the copy: must not reach the file
    finally:
        output.close_output(writer)
    for frame in range(1, 8):
        got = output.read_particles(cache, frame)
        assert got.shape == (n - frame, 3)
        assert np.all(got[:, 0] == np.float32(frame)) and np.all(got[:, 2] == np.float32(frame))
        np.testing.assert_array_equal(got[:, 1], np.float32(frame) + np.arange(n - frame, dtype=np.float32) * np.float32(1e-3))
