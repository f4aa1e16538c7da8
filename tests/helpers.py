"""Shared fixtures for the parity tests: seeded particle sets and configs."""
import numpy as np

from oracle import pm as opm


def random_particles(conf_o, seed=0, spread=3.0, lattice=True):
    """Lattice (gen_grid) particles with seeded random displacements of a few cells."""
    rng = np.random.default_rng(seed)
    pmid, disp = opm.gen_grid(conf_o)
    disp = (disp + rng.normal(0, spread * conf_o.cell_size, size=disp.shape)).astype(np.float32)
    if not lattice:
        pmid = rng.integers(0, min(conf_o.mesh_shape), size=pmid.shape).astype(np.int16)
    return pmid, disp


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
