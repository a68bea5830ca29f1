"""The replica harness on two CPU ranks over gloo: independent scenes, barriers, max over ranks."""

from __future__ import annotations

import multiprocessing as mp
import os
import socket
import time

import numpy as np


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scene_run(seed: int, steps: int):
    from continuum_liquid_b200 import scenes
    from oracle import oracle

    s = scenes.dam_break(12, seed=seed)
    pos, vel = scenes.seed_particles(s)
    sim = oracle.OracleSim(s.grid_shape, s.dx, pos, vel, dt=s.dt, flip_ratio=0.95, gravity=s.gravity)
    for _ in range(steps):
        sim.step()
    return sim.pos


def _rank_main(rank: int, world: int, port: int, steps: int, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from continuum_liquid_b200.replicas import ReplicaGroup, throughput

    group = ReplicaGroup("gloo", timeout_s=60)
    try:
        group.barrier()
        t0 = time.perf_counter()
        pos = _scene_run(seed=100 + rank, steps=steps)
        if rank == 1:
            time.sleep(0.2)  # this rank is the slow one
        own_ms = (time.perf_counter() - t0) * 1e3
        group.barrier()
        value, slowest = throughput(group, steps, own_ms)
        out.put((rank, own_ms, slowest, value, pos))
    finally:
        group.close()


def test_two_rank_replicas_over_gloo(oracle):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port, steps, world = _free_port(), 2, 2
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, steps, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((out.get(timeout=240) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    own = [r[1] for r in results]
    slowest = {r[2] for r in results}
    assert slowest == {max(own)}  # every rank got the slowest rank's time
    assert own[1] >= 200.0
    for rank, _, slow, value, pos in results:
        assert np.isclose(value, world * steps / (slow / 1e3))
        # replicas are independent: each equals the same scene run alone
        assert np.array_equal(pos, _scene_run(seed=100 + rank, steps=steps))
