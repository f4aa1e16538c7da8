"""Particle state (nbody/particles.py:33-127) as device tensors.

pmid int16 (N,3) anchor mesh cells, disp/vel/acc float32 (N,3); attr an
optional dict of per-particle attributes in the float dtype.
"""
from __future__ import annotations

from dataclasses import dataclass, replace
from typing import Optional

import torch


@dataclass
class Particles:
    conf: object
    pmid: torch.Tensor
    disp: torch.Tensor
    vel: Optional[torch.Tensor] = None
    acc: Optional[torch.Tensor] = None
    attr: Optional[dict] = None
    # bool (N,): True marks an unused (padding) slot, left out of every CIC
    # operation (particles.py:33-127 unused_index; cic/scatter.py:258)
    unused_index: Optional[torch.Tensor] = None

    def __post_init__(self):
        if self.attr is not None:  # custom per-particle features in the float dtype (particles.py:115-118)
            self.attr = {k: torch.as_tensor(v).to(self.conf.float_dtype) for k, v in self.attr.items()}

    def __len__(self):
        return self.pmid.shape[0]

    def __getitem__(self, key):
        """The particles selected by key (an index, slice or mask) in every field."""
        g = lambda t: None if t is None else t[key]
        attr = None if self.attr is None else {k: v[key] for k, v in self.attr.items()}
        return Particles(self.conf, self.pmid[key], self.disp[key], g(self.vel), g(self.acc), attr,
                         g(self.unused_index))

    def replace(self, **kw):
        return replace(self, **kw)

    def clone(self):
        c = lambda t: None if t is None else t.clone()
        attr = None if self.attr is None else {k: v.clone() for k, v in self.attr.items()}
        return Particles(self.conf, self.pmid, c(self.disp), c(self.vel), c(self.acc), attr, c(self.unused_index))

    def valid_mask(self):
        """uint8 (N,) device mask of the used slots (1) for the C ABI, or None
        when every slot is used."""
        if self.unused_index is None:
            return None
        u = torch.as_tensor(self.unused_index, device=self.disp.device)
        return (~u.to(torch.bool)).to(torch.uint8).contiguous()

    def raveled_id(self, dtype=torch.int64, wrap=False):
        """Raveled mesh index of each anchor, ((x My) + y) Mz + z (particles.py:729-772).
        int64 by default (the reference's uint64 is not a full torch dtype)."""
        if dtype.is_floating_point or dtype.is_complex or dtype == torch.bool:
            raise TypeError("raveled particle IDs require an integer dtype")
        if self.conf.mesh_size - 1 > torch.iinfo(dtype).max:
            raise OverflowError(f"mesh size {self.conf.mesh_size} does not fit {dtype}")
        pmid = self.pmid
        if wrap:
            pmid = torch.remainder(pmid, torch.tensor(self.conf.mesh_shape, dtype=pmid.dtype, device=pmid.device))
        _, my, mz = self.conf.mesh_shape
        p = pmid.to(dtype)
        return (p[:, 0] * (my * mz) + p[:, 1] * mz + p[:, 2]).to(dtype)

    @staticmethod
    def pmid_to_pos(pmid, disp, conf):
        """pmid * cell + disp, wrapped into the box (particles.py:800-816)."""
        pos = pmid.to(disp.dtype) * conf.cell_size + disp
        return torch.remainder(pos, torch.tensor(conf.box_size, dtype=pos.dtype, device=pos.device))

    @staticmethod
    def pos_to_pmid(pos, conf):
        """Nearest-cell anchors (wrapped) and displacements of positions (particles.py:818-840)."""
        p = Particles.from_pos(conf, pos, wrap=True)
        return p.pmid, p.disp

    @classmethod
    def from_pmid(cls, conf, pmid, disp, vel=None, acc=None):
        """Particles from anchors and displacements as given (particles.py:546-571)."""
        return cls(conf, torch.as_tensor(pmid), torch.as_tensor(disp), vel, acc)

    @classmethod
    def from_ptcl(cls, ptcl, conf=None, wrap=True):
        """A copy of ptcl's state in conf's dtypes, anchors wrapped into the mesh
        unless wrap is False (particles.py:573-613)."""
        conf = ptcl.conf if conf is None else conf
        pmid = ptcl.pmid.to(torch.int16)
        if wrap:
            pmid = torch.remainder(pmid, torch.tensor(conf.mesh_shape, dtype=torch.int16, device=pmid.device))
        return cls(conf, pmid, ptcl.disp.to(conf.float_dtype), ptcl.vel, ptcl.acc)

    @classmethod
    def gen_grid(cls, conf, vel=False, acc=False, device=None):
        """Uniform Lagrangian lattice (particles.py:615-727, single device):
        pmid = rint(linspace(0, Mx, nx)), disp = exact integer remainder * cell / n."""
        device = conf.device if device is None else torch.device(device)
        pm, dp = [], []
        for sp, sm in zip(conf.ptcl_grid_shape, conf.mesh_shape):
            p = torch.round(torch.linspace(0, sm, sp + 1, dtype=torch.float64, device=device)[:-1]).to(torch.int64)
            d = (torch.arange(sp, device=device, dtype=torch.int64) * sm - p * sp).to(torch.float64) * (conf.cell_size / sp)
            pm.append(p.to(torch.int16))
            dp.append(d.to(conf.float_dtype))
        pmid = torch.stack(torch.meshgrid(*pm, indexing="ij"), dim=-1).reshape(-1, 3).contiguous()
        disp = torch.stack(torch.meshgrid(*dp, indexing="ij"), dim=-1).reshape(-1, 3).contiguous()
        z = torch.zeros_like(disp)
        return cls(conf, pmid, disp, z.clone() if vel else None, z.clone() if acc else None)

    @classmethod
    def from_pos(cls, conf, pos, vel=None, acc=None, wrap=True):
        """Anchor every particle at its nearest mesh cell (particles.py:441-479,
        single device): pmid = rint(pos / cell), disp = pos - pmid * cell in the
        positions' dtype, then cast; with wrap, pmid modulo the mesh.  Anchors
        of different particles may coincide."""
        pos = torch.as_tensor(pos)
        pmid = torch.round(pos / conf.cell_size)  # half to even, like rint
        disp = pos - pmid * conf.cell_size
        pmid = pmid.to(torch.int16)
        if wrap:
            pmid = torch.remainder(pmid, torch.tensor(conf.mesh_shape, dtype=torch.int16, device=pmid.device))
        return cls(conf, pmid.contiguous(), disp.to(conf.float_dtype).contiguous(), vel, acc)

    @classmethod
    def from_pos_sharded(cls, conf, pos, vel=None, acc=None, wrap=True):
        """from_pos (one device; particles.py:481-494)."""
        return cls.from_pos(conf, pos, vel=vel, acc=acc, wrap=wrap)

    @classmethod
    def from_ordered_pos(cls, conf, pos, vel=None, acc=None, wrap=True):
        """Positions given in particle-grid order (LPT outputs, snapshots) keep
        the lattice anchors of gen_grid, which are unique where rounding the
        positions would collide (particles.py:497-545).  disp is the nearest
        periodic image of pos - anchor, computed in the working float dtype.
        ``wrap`` is accepted for signature parity; the nearest-image offset
        already wraps."""
        del wrap
        pos = torch.as_tensor(pos)
        grid = cls.gen_grid(conf, device=pos.device)
        if pos.shape[0] != grid.pmid.shape[0]:
            raise ValueError("from_ordered_pos requires a full particle-grid ordered position array: "
                             f"expected {grid.pmid.shape[0]} particles, got {pos.shape[0]}.")
        dt = conf.float_dtype
        p = pos.to(dt)
        anchor = grid.pmid.to(dt) * torch.tensor(conf.cell_size, dtype=dt, device=p.device)
        box = torch.tensor(conf.box_size, dtype=dt, device=p.device)
        half = torch.tensor(0.5, dtype=dt, device=p.device) * box
        disp = torch.remainder(p - anchor + half, box) - half
        return cls(conf, grid.pmid, disp.contiguous(), vel, acc)

    def pos(self, dtype=torch.float64, wrap=True):
        """particles.py:773-798."""
        pos = self.pmid.to(dtype) * self.conf.cell_size + self.disp.to(dtype)
        if wrap:
            pos = torch.remainder(pos, torch.tensor(self.conf.box_size, dtype=dtype, device=pos.device))
        return pos


def pmid_to_idx(pmid, conf, unused_index=None, dtype=torch.int32):
    """Flat cell key ((x mod Mx) My + (y mod My)) Mz + (z mod Mz) of each anchor;
    entries flagged in unused_index get -1 (core/utils.py:292-326)."""
    m = [torch.tensor(s, dtype=dtype, device=pmid.device) for s in conf.mesh_shape]
    ix, iy, iz = (torch.remainder(pmid[:, d].to(dtype), m[d]) for d in range(3))
    idx = (ix * m[1] + iy) * m[2] + iz
    if unused_index is not None:
        idx = torch.where(torch.as_tensor(unused_index, device=idx.device), torch.full_like(idx, -1), idx)
    return idx
