"""Moving colliders (no counterpart in the reference, whose colliders are voxelised once at set-up and
never move: solver.py:132-139, voxelise_mesh.py:138-163).

A scene's colliders may move together as one rigid body, ``RigidMotion(velocity, angular_velocity,
pivot)``, given in world units (m/s, rad/s, m) and constant over the bake. At time t the collider's
triangles are its rest triangles rotated by the angle |W| t about the axis W / |W| through the pivot,
then moved by V t; the solid's velocity at a point x is V + W x (x - (pivot + V t)).

A step at time t (the step's start) voxelises the colliders at their pose at t with the reference's
ray-parity test, then uses the solid's velocity in the obstacle conditions: solid faces of the grid
take the solid's velocity component, and particles inside the solid are pushed out as the reference
pushes them, losing only the inward part of their velocity relative to the solid. A collider at rest
(V = W = 0) gives exactly the reference's results.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class RigidMotion:
    velocity: tuple[float, float, float] = (0.0, 0.0, 0.0)
    angular_velocity: tuple[float, float, float] = (0.0, 0.0, 0.0)
    pivot: tuple[float, float, float] = (0.0, 0.0, 0.0)

    @classmethod
    def from_config(cls, motion: dict | None) -> "RigidMotion | None":
        """A config entry {"velocity": [..], "angular_velocity": [..], "pivot": [..]} (any key may be
        missing), or None."""
        if not motion:
            return None
        return cls(tuple(float(x) for x in motion.get("velocity", (0.0, 0.0, 0.0))),
                   tuple(float(x) for x in motion.get("angular_velocity", (0.0, 0.0, 0.0))),
                   tuple(float(x) for x in motion.get("pivot", (0.0, 0.0, 0.0))))

    def rotation(self, t: float) -> np.ndarray:
        """The rotation matrix at time t (Rodrigues' formula, float64)."""
        w = np.asarray(self.angular_velocity, dtype=np.float64)
        speed = float(np.linalg.norm(w))
        if speed == 0.0:
            return np.eye(3)
        k = w / speed
        K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
        a = speed * float(t)
        return np.eye(3) + np.sin(a) * K + (1.0 - np.cos(a)) * (K @ K)

    def pivot_at(self, t: float) -> np.ndarray:
        return np.asarray(self.pivot, dtype=np.float64) + np.asarray(self.velocity, dtype=np.float64) * float(t)

    def transform(self, triangles: np.ndarray, t: float) -> np.ndarray:
        """World-space triangles (T, 3, 3) at rest -> their pose at time t, float32."""
        tri = np.asarray(triangles, dtype=np.float64).reshape(-1, 3)
        c0 = np.asarray(self.pivot, dtype=np.float64)
        moved = (tri - c0) @ self.rotation(t).T + self.pivot_at(t)
        return np.ascontiguousarray(moved.reshape(-1, 3, 3), dtype=np.float32)

    def parameters(self, t: float, origin) -> np.ndarray:
        """The 9 float32 kernel parameters at time t: V, W and the pivot in grid-local coordinates
        (world minus the domain origin)."""
        c = self.pivot_at(t) - np.asarray(origin, dtype=np.float64)
        return np.array([*self.velocity, *self.angular_velocity, *c], dtype=np.float32)


def motion_arg(parameters: np.ndarray) -> ctypes.Array:
    """The 9 parameters as the host float array the C entry points take."""
    values = np.asarray(parameters, dtype=np.float32).reshape(9)
    return (ctypes.c_float * 9)(*[float(x) for x in values])
