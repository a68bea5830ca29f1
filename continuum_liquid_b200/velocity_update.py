"""Grid force stage (mirrors Solver/Kernel/velocity_update.py)."""

from __future__ import annotations

import numpy as np

from .backend import Backend

FIELD_DTYPE = np.float32


def update_velocity(kernels: Backend, queue, velocity, result, fluid_fraction, gravity, fx, fy, fz, rho, nu, dx, dt,
                    grid_shape):
    """velocity_update.py:8-52: result = u + dt (g + f/rho) where fluid, + nu dt laplacian(u) inside."""
    nx, ny, nz = grid_shape
    u, v, w = velocity
    ru, rv, rw = result
    kernels.call(
        "clb_update_velocity",
        u,
        v,
        w,
        ru,
        rv,
        rw,
        fluid_fraction,
        float(FIELD_DTYPE(gravity[0])),
        float(FIELD_DTYPE(gravity[1])),
        float(FIELD_DTYPE(gravity[2])),
        float(FIELD_DTYPE(fx)),
        float(FIELD_DTYPE(fy)),
        float(FIELD_DTYPE(fz)),
        float(FIELD_DTYPE(rho)),
        float(FIELD_DTYPE(nu)),
        float(FIELD_DTYPE(1.0 / (float(dx) * float(dx)))),
        float(FIELD_DTYPE(dt)),
        nx,
        ny,
        nz,
        stream=queue,
    )
    return result
