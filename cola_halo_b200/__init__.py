"""B200-native particle-mesh force, COLA time step and 2LPT setup for
cola_halo, behind the reference's C entry points (libcolagpu.so).

    from cola_halo_b200 import Simulation, Schedule
"""
from .schedule import Schedule, output_scale_factors, run_time_loop  # noqa: F401
from .types import (PARTICLE_DTYPE, PARTICLE_MIN_DTYPE, HostParticles,  # noqa: F401
                    HostSnapshot, Particles, Snapshot)


def __getattr__(name):
    # GPU-facing classes load the CUDA library on first use only.
    if name in ("Simulation", "kick_coeffs", "drift_coeffs", "fft_r2c", "fft_c2r"):
        from . import sim
        return getattr(sim, name)
    raise AttributeError(name)
