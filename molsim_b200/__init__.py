"""B200-native force/energy path for MOLSIM (TomHoefken/molsim).

The compute path is libmolsim_gpu.so (hand-written CUDA for sm_100a behind the
C-ABI in include/molsim_gpu.h).  This package holds the Python mirror of the
reference's entry points (engine.py), the seeded system generators
(systems.py) and the build recipe (build.py).
"""
from .engine import Engine, MolsimGpuError, alpha_to_ncut, pot_tab, prepare, rcut_to_alpha  # noqa: F401
