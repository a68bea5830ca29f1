"""Continuum Liquid B200 backend: the FLIP/PIC timestep hot path of the Continuum Liquid add-on
(particle binning and counting sort, P2G, G2P and advection, collider voxelisation, multigrid
W-cycle pressure solve) as hand-written sm_100a CUDA behind the add-on's Python stage interface.

The CUDA library (libclb200.so) is loaded through ``backend.Backend``; there is no CPU fallback.
"""

__version__ = "0.1.0"
