"""Particle state (nbody/particles.py:33-127) as device tensors.

pmid int16 (N,3) anchor mesh cells, disp/vel/acc float32 (N,3).
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

    def __len__(self):
        return self.pmid.shape[0]

    def replace(self, **kw):
        return replace(self, **kw)

    def clone(self):
        c = lambda t: None if t is None else t.clone()
        return Particles(self.conf, self.pmid, c(self.disp), c(self.vel), c(self.acc))

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
