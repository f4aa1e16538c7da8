"""Particle-state checkpoints: save a run's state at a scale factor and resume
it later (the reference keeps no on-disk state; its run segments pass
``Particles`` between configurations, nbody/solver.py:645-679).

The file is a NumPy ``.npz`` with pmid (int16, N x 3), disp / vel / acc
(float32, N x 3; vel and acc optional), unused_index (bool, N; optional), the
scale factor ``a``, and the geometry it was written for (ptcl_spacing,
ptcl_grid_shape, mesh_shape), checked on load."""
from __future__ import annotations

import numpy as np
import torch

from .particles import Particles

FORMAT_VERSION = 1


def save_state(path, ptcl, a, conf):
    """Write ptcl (at scale factor a) to path (a .npz file)."""
    arrays = {"format_version": np.int64(FORMAT_VERSION), "a": np.float64(a),
              "ptcl_spacing": np.float64(conf.ptcl_spacing),
              "ptcl_grid_shape": np.asarray(conf.ptcl_grid_shape, np.int64),
              "mesh_shape": np.asarray(conf.mesh_shape, np.int64), "pmid": ptcl.pmid.cpu().numpy(),
              "disp": ptcl.disp.cpu().numpy()}
    for name in ("vel", "acc"):
        t = getattr(ptcl, name)
        if t is not None:
            arrays[name] = t.cpu().numpy()
    if getattr(ptcl, "unused_index", None) is not None:
        arrays["unused_index"] = ptcl.unused_index.cpu().numpy().astype(bool)
    with open(path, "wb") as f:
        np.savez(f, **arrays)


def load_state(path, conf, device=None):
    """Read a checkpoint written by save_state for the same geometry.
    Returns (Particles on device (conf.device by default), a)."""
    with np.load(path) as z:
        if int(z["format_version"]) != FORMAT_VERSION:
            raise ValueError(f"checkpoint format {int(z['format_version'])} is not {FORMAT_VERSION}")
        if (float(z["ptcl_spacing"]) != conf.ptcl_spacing
                or tuple(z["ptcl_grid_shape"].tolist()) != tuple(conf.ptcl_grid_shape)
                or tuple(z["mesh_shape"].tolist()) != tuple(conf.mesh_shape)):
            raise ValueError("checkpoint geometry differs from the configuration")
        dev = conf.device if device is None else torch.device(device)
        t = lambda k: torch.from_numpy(np.ascontiguousarray(z[k])).to(dev) if k in z.files else None
        ptcl = Particles(conf, t("pmid"), t("disp"), t("vel"), t("acc"), unused_index=t("unused_index"))
        return ptcl, float(z["a"])
