"""B200-native rebuild of PM++'s single-GPU particle-mesh path.

The hot path runs hand-written sm_100a CUDA kernels from libpmb200.so (C ABI,
include/pmb200.h); this package is the host-side mirror of PM++'s Python API:

* Configuration, Cosmology / SimpleLCDM / boltzmann, Particles
* cic.scatter / cic.gather and their adjoints
* gravity, nbody (forward) and nbody_adj (hand-written reverse sweep)
* lpt, white_noise_nested, linear_modes
* delta_to_pk / density_to_pk / particles_to_pk
"""
from .configuration import Configuration
from .cosmology import Cosmology, SimpleLCDM, boltzmann, growth, linear_power
from .particles import Particles, pmid_to_idx
from . import cic
from .cic import scatter, gather, scatter_vjp, gather_vjp
from .gravity import gravity, gravity_vjp, gravity_streamed
from .nbody import (nbody, nbody_adj, integrate, kick, drift, NBodyRun, kick_adj, drift_adj_from_output,
                    force_adj, integrate_adj, nbody_low_memory, nbody_scheduled, nbody_static_halo_scheduled,
                    nbody_init, nbody_step, nbody_collect, nbody_observe)
from . import observers, checkpoint, corrections, meshcnn, slab
from .slab import SlabPM, LocalComm, ProcessGroupComm
from .observers import density_projection_observer, nbody_kappa
from .checkpoint import save_state, load_state

__all__ = [
    "Configuration", "Cosmology", "SimpleLCDM", "boltzmann", "growth", "linear_power", "Particles", "pmid_to_idx", "cic", "scatter",
    "gather", "scatter_vjp", "gather_vjp", "gravity", "gravity_vjp", "nbody", "nbody_adj", "integrate", "kick",
    "drift", "NBodyRun", "kick_adj", "drift_adj_from_output", "force_adj", "integrate_adj", "gravity_streamed",
    "nbody_low_memory", "nbody_scheduled", "nbody_static_halo_scheduled", "nbody_init", "nbody_step",
    "nbody_collect", "nbody_observe", "observers", "checkpoint", "density_projection_observer", "nbody_kappa",
    "save_state", "load_state", "corrections", "meshcnn", "slab", "SlabPM", "LocalComm", "ProcessGroupComm"
]
from . import modes, lpt, power_spectrum, pipeline  # noqa: E402
from .modes import white_noise_nested, linear_modes  # noqa: E402
from .lpt import lpt as lpt_displacements  # noqa: E402
from .power_spectrum import delta_to_pk, density_to_pk, particles_to_pk  # noqa: E402
