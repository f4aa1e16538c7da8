"""Cloud-in-cell scatter and gather with their hand-written adjoints.

Public API mirrors pmpp.cic (cic/scatter.py:235-275, cic/gather.py:323-360):
``scatter(ptcl, conf, mesh=None, val=None)`` and ``gather(ptcl, conf, mesh)``
with the reference's trailing-channel mesh layout (Mx, My, Mz[, C]); the
adjoints ``scatter_vjp`` / ``gather_vjp`` restate ``_scatter_bwd`` /
``_gather_bwd`` (scatter.py:386-437, gather.py:517-548).  ``Scatter`` and
``Gather`` are torch.autograd Functions wrapping the same kernels.

Every call sorts the particles by lower-corner mesh row on the device
(pmb_sort_rows, or pmb_sort_rows_ex with a mesh offset or unused slots) and
runs the deterministic pull scatter / sorted gather.  ``offset`` moves the
mesh origin as in the reference (cic/enmesh.py:128-147); slots flagged in
``ptcl.unused_index`` take no part (cic/scatter.py:258-272,
cic/gather.py:356-357); an explicit ``cell_size`` resamples onto a mesh of
another cell size through the per-particle pmb_cic_general_* kernels.
"""
from __future__ import annotations

import torch

from ._lib import call, lib
from .runtime import ptr, require_cuda, stream_handle, workspace


def offset3(offset):
    """Mesh offset as three floats (a scalar applies to every axis)."""
    o = torch.as_tensor(offset, dtype=torch.float64).reshape(-1).tolist()
    if len(o) == 1:
        o = o * 3
    if len(o) != 3:
        raise ValueError(f"offset must be a scalar or have 3 entries, got {len(o)}")
    return [float(x) for x in o]


class SortedParticles:
    """Device buffer of particles sorted by lower-corner mesh row.

    offset: mesh origin in the particles' frame; valid: uint8 (N,) mask of the
    used slots (None: all)."""

    def __init__(self, pmid, disp, conf, mesh_shape=None, drift_vel=None, drift=0.0, offset=0.0, valid=None):
        require_cuda(pmid, disp, drift_vel, valid)
        if disp.dtype != torch.float32:
            raise TypeError("the cell-sorted CIC kernels take float32 displacements (the float64 build has its own "
                            "deposit and force)")
        self.conf = conf
        self.shape = tuple(mesh_shape or conf.mesh_shape)
        self.n = pmid.shape[0]
        nx, ny, nz = self.shape
        L = lib()
        dev = disp.device
        self.buf = torch.empty(L.pmb_sorted_bytes(self.n, nx, ny, nz), dtype=torch.uint8, device=dev)
        sb = L.pmb_sort_scratch_bytes(self.n, nx, ny, nz)
        scratch = workspace(sb, dev, "sort")
        o = offset3(offset)
        if valid is None and o == [0.0, 0.0, 0.0]:
            call("pmb_sort_rows", pmid.data_ptr(), disp.data_ptr(), ptr(drift_vel), float(drift), self.n, nx, ny, nz,
                 float(conf.cell_size), self.buf.data_ptr(), scratch.data_ptr(), scratch.numel(), stream_handle(dev))
        else:
            call("pmb_sort_rows_ex", pmid.data_ptr(), disp.data_ptr(), ptr(drift_vel), float(drift), self.n, nx, ny,
                 nz, float(conf.cell_size), o[0], o[1], o[2], ptr(valid), self.buf.data_ptr(), scratch.data_ptr(),
                 scratch.numel(), stream_handle(dev))

    def scatter(self, val=None, val_const=None, channels=1, mode=0, src_mul=1.0, out=None, val_sorted=False):
        """Deposit; val (n, channels) is in particle order, or in sorted order
        with val_sorted (as written by interp_grad's u_sorted)."""
        nx, ny, nz = self.shape
        dev = self.buf.device
        if out is None:
            out = torch.empty((channels, nx, ny, nz), dtype=torch.float32, device=dev)
        s16 = workspace(16, dev, "scale16")
        vc = float(self.conf.mesh_size / self.conf.ptcl_num) if (val is None and val_const is None) else (
            0.0 if val_const is None else float(val_const))
        call("pmb_scatter_rows", self.buf.data_ptr(), self.n, nx, ny, nz, channels, ptr(val), int(val_sorted), vc,
             mode, float(src_mul), out.data_ptr(), s16.data_ptr(), stream_handle(dev))
        return out

    def gather(self, mesh_planar, out=None, vel=None, kick=0.0):
        nx, ny, nz = self.shape
        C = mesh_planar.shape[0]
        if out is None:
            out = torch.empty((self.n, C), dtype=torch.float32, device=mesh_planar.device)
        call("pmb_gather_rows", self.buf.data_ptr(), self.n, nx, ny, nz, C, mesh_planar.data_ptr(), out.data_ptr(),
             ptr(vel), float(kick), stream_handle(mesh_planar.device))
        return out

    def interp_grad(self, mesh_planar, u=None, u_const=0.0, disp_cot=None, accumulate=False, wsum=False, u_sorted=None):
        nx, ny, nz = self.shape
        C = mesh_planar.shape[0]
        dev = mesh_planar.device
        if disp_cot is None:
            disp_cot = torch.empty((self.n, 3), dtype=torch.float32, device=dev)
            accumulate = False
        ws = torch.empty((self.n, C), dtype=torch.float32, device=dev) if wsum else None
        call("pmb_interp_grad_rows", self.buf.data_ptr(), self.n, nx, ny, nz, C, mesh_planar.data_ptr(), ptr(u),
             float(u_const), float(self.conf.cell_size), int(accumulate), disp_cot.data_ptr(), ptr(ws), ptr(u_sorted),
             stream_handle(dev))
        return disp_cot, ws


def _planar(mesh, conf):
    """(Mx,My,Mz[,C]) -> contiguous (C,Mx,My,Mz) float32."""
    mesh = mesh.to(torch.float32)
    if mesh.dim() == 3:
        return mesh.unsqueeze(0).contiguous(), False
    return mesh.permute(3, 0, 1, 2).contiguous(), True


def _channels_last(m, had_channels):
    return m.permute(1, 2, 3, 0) if had_channels else m[0]


def _val_array(val, n, device):
    """None / scalar / (N,) / (N,C) -> (tensor or None, constant, channels)."""
    if val is None:
        return None, None, 1
    if not torch.is_tensor(val) or val.dim() == 0:
        return None, float(val), 1
    v = val.to(device=device, dtype=torch.float32)
    if v.dim() == 1:
        return v.contiguous(), None, 1
    return v.reshape(n, -1).contiguous(), None, v.reshape(n, -1).shape[1]


def _masked_val(v, valid):
    """Zero the values of unused slots (cic/scatter.py:268-272)."""
    if v is None or valid is None:
        return v
    keep = valid.to(torch.bool)
    return torch.where(keep.reshape((-1, ) + (1, ) * (v.dim() - 1)), v, torch.zeros_like(v)).contiguous()


class _General:
    """Argument pack of the pmb_cic_general_* entry points (explicit cell size)."""

    def __init__(self, ptcl, conf, mesh_shape, offset, cell_size):
        require_cuda(ptcl.pmid, ptcl.disp)
        self.valid = ptcl.valid_mask()
        self.n = len(ptcl)
        self.head = (ptcl.pmid.data_ptr(), ptcl.disp.data_ptr(), ptr(self.valid), self.n, *conf.mesh_shape,
                     float(conf.cell_size), *offset3(offset), float(cell_size), *mesh_shape)
        self.shape = tuple(mesh_shape)
        self.dev = ptcl.disp.device


def _general_scatter(g, val, vc, C):
    nx, ny, nz = g.shape
    out = torch.empty((C, nx, ny, nz), dtype=torch.float32, device=g.dev)
    sb = lib().pmb_cic_general_scratch_bytes(nx, ny, nz, C)
    scratch = workspace(sb, g.dev, "cic_general")
    call("pmb_cic_general_scatter", *g.head, C, ptr(val), float(vc or 0.0), out.data_ptr(), scratch.data_ptr(),
         scratch.numel(), stream_handle(g.dev))
    return out


def _general_interp_grad(g, mp, u, u_const, wsum=False):
    C = mp.shape[0]
    disp_cot = torch.empty((g.n, 3), dtype=torch.float32, device=g.dev)
    ws = torch.empty((g.n, C), dtype=torch.float32, device=g.dev) if wsum else None
    call("pmb_cic_general_interp_grad", *g.head, C, mp.data_ptr(), ptr(u), float(u_const), disp_cot.data_ptr(),
         ptr(ws), stream_handle(g.dev))
    return disp_cot, ws


def scatter(ptcl, conf, mesh=None, val=None, offset=0, cell_size=None):
    """CIC deposit (cic/scatter.py:235-275); val defaults to mesh_size/ptcl_num.

    Unused slots (ptcl.unused_index) deposit nothing; offset moves the mesh
    origin; cell_size resamples onto a mesh of that cell size (the shape of
    ``mesh`` when given, else the configuration's mesh shape)."""
    if conf.float_dtype == torch.float64:
        if mesh is not None or offset not in (0, 0.0) or cell_size is not None or (val is not None and
                                                                                     not isinstance(val, float)):
            raise NotImplementedError("the float64 build deposits a constant value on the configuration mesh")
        from . import x64
        return x64.scatter(ptcl, conf, val)
    valid = ptcl.valid_mask()
    v, vc, C = _val_array(val, len(ptcl), ptcl.disp.device)
    v = _masked_val(v, valid)
    if v is None and vc is None:
        vc = float(conf.mesh_size / conf.ptcl_num)
    if cell_size is not None:
        shape = tuple(mesh.shape[:3]) if mesh is not None else tuple(conf.mesh_shape)
        out = _general_scatter(_General(ptcl, conf, shape, offset, cell_size), v, vc, C)
    else:
        sp = SortedParticles(ptcl.pmid, ptcl.disp, conf, offset=offset, valid=valid)
        out = sp.scatter(val=v, val_const=vc, channels=C)
    out = out[0] if (v is None or v.dim() == 1) else out.permute(1, 2, 3, 0)
    if mesh is not None:
        out = out + mesh
    return out


def gather(ptcl, conf, mesh, offset=0, cell_size=None):
    """CIC interpolation (cic/gather.py:323-360); unused slots gather 0.
    offset / cell_size as the private _gather (cic/gather.py:447-472)."""
    mp, had = _planar(mesh, conf)
    shape = tuple(mesh.shape[:3])
    if cell_size is not None:
        g = _General(ptcl, conf, shape, offset, cell_size)
        out = torch.empty((g.n, mp.shape[0]), dtype=torch.float32, device=g.dev)
        call("pmb_cic_general_gather", *g.head, mp.shape[0], mp.data_ptr(), out.data_ptr(), stream_handle(g.dev))
    else:
        sp = SortedParticles(ptcl.pmid, ptcl.disp, conf, mesh_shape=shape, offset=offset, valid=ptcl.valid_mask())
        out = sp.gather(mp)
    return out if had else out[:, 0]


def scatter_vjp(ptcl, conf, mesh_cot, val=None, offset=0, cell_size=None):
    """Adjoint of scatter (scatter.py:386-437): returns (disp_cot, val_cot).

    val_cot is summed over particles when val is a scalar (or None); unused
    slots get zero cotangents.  The float64 build takes constant values on the
    configuration mesh."""
    if conf.float_dtype == torch.float64:
        if offset not in (0, 0.0) or cell_size is not None or not (val is None or isinstance(val, float)) or \
                tuple(mesh_cot.shape) != tuple(conf.mesh_shape) or ptcl.valid_mask() is not None:
            raise NotImplementedError("the float64 deposit adjoint takes a constant value on the configuration mesh")
        from . import x64
        return x64.scatter_vjp(ptcl, conf, mesh_cot, val)
    valid = ptcl.valid_mask()
    shape = tuple(mesh_cot.shape[:3])
    mp, had = _planar(mesh_cot, conf)
    v, vc, C = _val_array(val, len(ptcl), ptcl.disp.device)
    v = _masked_val(v, valid)
    if v is None and vc is None:
        vc = float(conf.mesh_size / conf.ptcl_num)
    if cell_size is not None:
        disp_cot, wsum = _general_interp_grad(_General(ptcl, conf, shape, offset, cell_size), mp, v,
                                              0.0 if vc is None else vc, wsum=True)
    else:
        sp = SortedParticles(ptcl.pmid, ptcl.disp, conf, mesh_shape=shape, offset=offset, valid=valid)
        disp_cot, wsum = sp.interp_grad(mp, u=v, u_const=0.0 if vc is None else vc, wsum=True)
    if v is None:
        val_cot = wsum.sum(dtype=torch.float64).to(torch.float32)
    else:
        val_cot = wsum if had else wsum[:, 0]
    # scatter.py:427-435: no displacement cotangent where the value is zero
    if v is not None:
        nz = (v != 0) if v.dim() == 1 else (v != 0).any(dim=1)
        disp_cot = torch.where(nz[:, None], disp_cot, torch.zeros_like(disp_cot))
    elif vc == 0:
        disp_cot = torch.zeros_like(disp_cot)
    return disp_cot, val_cot


def gather_vjp(ptcl, conf, mesh, val_cot, offset=0, cell_size=None):
    """Adjoint of gather (gather.py:517-548): returns (disp_cot, mesh_cot);
    unused slots contribute nothing."""
    valid = ptcl.valid_mask()
    shape = tuple(mesh.shape[:3])
    mp, had = _planar(mesh, conf)
    vc = _masked_val(val_cot.to(torch.float32).reshape(len(ptcl), -1).contiguous(), valid)
    if cell_size is not None:
        g = _General(ptcl, conf, shape, offset, cell_size)
        disp_cot, _ = _general_interp_grad(g, mp, vc, 0.0)
        mesh_cot = _general_scatter(g, vc, None, vc.shape[1])
    else:
        sp = SortedParticles(ptcl.pmid, ptcl.disp, conf, mesh_shape=shape, offset=offset, valid=valid)
        disp_cot, _ = sp.interp_grad(mp, u=vc)
        mesh_cot = sp.scatter(val=vc, channels=vc.shape[1])
    return disp_cot, _channels_last(mesh_cot, had)


class Scatter(torch.autograd.Function):
    """Differentiable CIC density (constant particle value) w.r.t. disp."""

    @staticmethod
    def forward(ctx, disp, pmid, conf):
        ctx.save_for_backward(disp, pmid)
        ctx.conf = conf
        from .particles import Particles
        return scatter(Particles(conf, pmid, disp.detach().contiguous()), conf)

    @staticmethod
    def backward(ctx, mesh_cot):
        disp, pmid = ctx.saved_tensors
        from .particles import Particles
        dc, _ = scatter_vjp(Particles(ctx.conf, pmid, disp.detach().contiguous()), ctx.conf,
                            mesh_cot.contiguous())
        return dc, None, None


class Gather(torch.autograd.Function):
    """Differentiable CIC gather w.r.t. disp and the mesh."""

    @staticmethod
    def forward(ctx, disp, mesh, pmid, conf):
        ctx.save_for_backward(disp, mesh, pmid)
        ctx.conf = conf
        from .particles import Particles
        return gather(Particles(conf, pmid, disp.detach().contiguous()), conf, mesh.detach())

    @staticmethod
    def backward(ctx, val_cot):
        disp, mesh, pmid = ctx.saved_tensors
        from .particles import Particles
        dc, mc = gather_vjp(Particles(ctx.conf, pmid, disp.detach().contiguous()), ctx.conf, mesh.detach(),
                            val_cot.contiguous())
        return dc, mc, None, None
