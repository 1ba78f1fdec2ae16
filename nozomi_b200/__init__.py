"""nozomi_b200 — B200-native Monte Carlo spin random walk for diffusion MRI.

A drop-in for nozomi's simulation engine (simulation_toolkit/simulation_engine):
the same geometry, engine and waveform classes (``SimGeometry3D``,
``Structure3D``, ``DiffSim3d``, ``DwiSim3d``, ``PGDiffWaveform`` ...), the same
substrate pickle format and CLI, computed by hand-written sm_100a kernels in
libnozomi_b200.so through a C ABI (include/nozomi_b200.h).
"""
__version__ = "0.1.0"
