"""B200-native quasistatic 3D xi-step engine with lcodePy's Simulation API.

The compute path is liblcb.so (hand-written sm_100a CUDA behind a C ABI,
include/lcb.h); this package is the host side that mirrors the reference's
``lcode`` interface (Simulation, Config, beam generator, diagnostics hooks).
"""
__version__ = "0.1.0"

from .config import Config, default_config_values  # noqa: F401
from .beam_generator import generate_beam, particle_dtype3d  # noqa: F401


def __getattr__(name):
    # CUDA-dependent parts load lazily so that host-only tools (config,
    # generator, build) import on machines without a GPU.
    if name == "Simulation":
        from .simulation import Simulation
        return Simulation
    raise AttributeError(name)
