"""The committed warm-start weights (continuum_liquid_b200/weights, written by
``python -m continuum_liquid_b200.train_warm_start``) against the solver without them, on solves the
network never saw (held-out seed of the 128^3 collider pool)."""

from __future__ import annotations

import json

import numpy as np
import pytest

from continuum_liquid_b200 import learned, scenes

pytestmark = pytest.mark.gpu


def test_committed_weights_gain_on_held_out_solves(backend):
    path = learned.default_weights_path()
    assert path.exists(), "train the network first: python -m continuum_liquid_b200.train_warm_start"
    with np.load(path) as data:
        meta = json.loads(str(data["meta"]))
    assert meta["iterations"] >= 1000 and meta["evaluation"]["collider_pool_128"]["frames"] > 0
    net = learned.UNet(backend)
    net.load(path)
    frames = learned.capture_frames(backend, scenes.collider_pool(128, seed=104), steps=10, skip=2)
    rows = learned.evaluate(backend, net, frames)
    prev = sum(r["previous"]["cycles"] for r in rows)
    lrn = sum(r["learned"]["cycles"] for r in rows)
    start_prev = np.mean([r["previous"]["initial_rel"] for r in rows])
    start_lrn = np.mean([r["learned"]["initial_rel"] for r in rows])
    print(f"held-out 128^3 collider pool, {len(rows)} solves: cycles {prev} -> {lrn}; "
          f"starting relative residual {start_prev:.3f} -> {start_lrn:.3f}")
    # the solver takes the network's guess only when it starts lower, so it never starts higher
    assert start_lrn <= start_prev
    assert start_lrn < 0.8 * start_prev  # the trained network halves it on these solves
    assert lrn <= prev
    assert backend.device_error() == 0
