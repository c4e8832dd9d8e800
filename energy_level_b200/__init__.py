"""B200-native matrix-free many-body ED for the Rydberg Hamiltonian.

Hot path: hand-written sm_100a CUDA kernels in ``libel_b200.so`` (C ABI in
``include/energy_level_b200.h``), reached from Python through ctypes.  The
reference-facing entry points mirror the energy-level engine's manybody API:
``matrix_free.b200_lanczos_ground_state``, ``kpm.kpm_moments_b200``,
``engine.evolve_manybody`` and ``backends.solve_equilibrium``.
"""
__version__ = "0.1.0"
