"""Stable per-cell particle order (pmb_sort_by_cell).

Key = raveled lower-corner cell ((x*My + y)*Mz + z) of the CIC binning
(cic/enmesh.py:139-147, core/utils.py:292-326); equal keys keep source
order, the tie rule of the reference's merges (cuda/route_kernels.cu:641-644).
"""
from __future__ import annotations

import torch

from ._lib import call, lib
from .runtime import require_cuda, stream_handle, workspace


def sort_by_cell(ptcl, conf):
    """Return (keys (N,) uint32 as int32 tensor view, perm (N,) int32)."""
    require_cuda(ptcl.pmid, ptcl.disp)
    n = len(ptcl)
    nx, ny, nz = conf.mesh_shape
    dev = ptcl.disp.device
    keys = torch.empty(n, dtype=torch.int32, device=dev)
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    sb = lib().pmb_sort_by_cell_scratch_bytes(n, nx, ny, nz)
    ws = workspace(sb, dev, "radix")
    call("pmb_sort_by_cell", ptcl.pmid.data_ptr(), ptcl.disp.data_ptr(), n, nx, ny, nz, float(conf.cell_size),
         keys.data_ptr(), perm.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle(dev))
    return keys, perm
