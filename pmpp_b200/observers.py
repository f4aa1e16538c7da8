"""Forward-only observers and saved maps (nbody/observers.py:18-126).

Projections run on the device: the deterministic CIC deposit, then
``pmb_project_density`` (one windowed periodic sum along an axis, FP64 in a
fixed order).  Observers see the state after every macro step and are not
part of the adjoint."""
from __future__ import annotations

import numpy as np
import torch

from ._lib import call
from .cic import scatter
from .runtime import require_cuda, stream_handle


def project(mesh, axis, start=0, stop=None, max_width=None):
    """Sum of the planes start .. stop-1 (periodic; at most max_width of them)
    of a (nx, ny, nz) float32 device mesh along axis; the other two axes
    remain (core/utils.py:420-463 wraparound_slice, summed)."""
    require_cuda(mesh)
    if mesh.dtype != torch.float32 or mesh.dim() != 3:
        raise ValueError("project expects a (nx, ny, nz) float32 mesh")
    mesh = mesh.contiguous()
    nx, ny, nz = mesh.shape
    if axis not in (0, 1, 2):
        raise ValueError(f"axis must be 0, 1 or 2, got {axis}")
    stop = mesh.shape[axis] if stop is None else int(stop)
    shape = [s for i, s in enumerate(mesh.shape) if i != axis]
    out = torch.empty(shape, dtype=torch.float32, device=mesh.device)
    call("pmb_project_density", mesh.data_ptr(), nx, ny, nz, int(axis), int(start), stop,
         -1 if max_width is None else int(max_width), out.data_ptr(), stream_handle(mesh.device))
    return out


def density_projection_observer(axis, normalize=False):
    """Observer (a, ptcl, cosmo, conf) -> the CIC density summed over axis,
    divided by its mean with normalize (observers.py:18-56)."""

    def observer(a, ptcl, cosmo, conf):
        del a, cosmo
        proj = project(scatter(ptcl, conf), axis)
        if normalize:
            proj = proj / proj.double().mean().float()
        return proj

    return observer


def saved_maps_collector(conf):
    """Collector filling (len(to_save_a), 3, nMesh, nMesh) maps: at the step
    whose a_next is within 1e-6 of to_save_a[i], the three axis projections of
    the density over the periodic window slice_to_save[i] .. slice_to_save[i+1]
    (at most max_slice_width planes) (observers.py:86-126)."""
    to_save_a = np.asarray(conf.to_save_a, dtype=np.float64)

    def collector(state, a_prev, a_next, ptcl, cosmo, conf_step):
        del a_prev, cosmo
        hits = np.flatnonzero(np.isclose(float(a_next), to_save_a, atol=1e-6, rtol=0))
        if hits.size == 0:
            return state
        i = int(hits[0])
        dens = scatter(ptcl, conf_step)
        lo, hi = conf.slice_to_save[i], conf.slice_to_save[i + 1]
        for axis in range(3):
            state[i, axis] = project(dens, axis, lo, hi, conf.max_slice_width)
        return state

    return collector


def nbody_kappa(ptcl, cosmo, conf, reverse=False):
    """The saved-map forward run (observers.py:59-126): the final particles
    when conf.to_save_a is None, else the stacked maps."""
    from .nbody import nbody, nbody_collect
    if conf.to_save_a is None:
        return nbody(ptcl, cosmo, conf, reverse=reverse)
    if conf.slice_to_save is None or len(conf.slice_to_save) < len(conf.to_save_a) + 1:
        raise ValueError("slice_to_save needs len(to_save_a) + 1 plane indices")
    n = conf.nMesh
    maps = torch.zeros((len(conf.to_save_a), 3, n, n), dtype=torch.float32, device=ptcl.disp.device)
    return nbody_collect(ptcl, cosmo, conf, saved_maps_collector(conf), maps, reverse=reverse)
