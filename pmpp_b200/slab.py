"""Slab-decomposed particle-mesh force and KDK integration over several GPUs.

The mesh is cut into x slabs of nx / P planes, one per rank (one process per
GPU through torch.distributed: NCCL between GPUs, gloo on CPU), and every
rank owns the particles whose lower CIC corner lies in its slab.  Reference:
distributed/mesh_halo.py:74-181 (mesh halo exchange), distributed/fft.py:
439-884 (slab rFFT with all-to-all transposes) and cuda/route_kernels.cu:
147-1317 (routing particles to the owning rank, fail-closed capacity).

One force evaluation on rank r (all ranks in step):

1. deposit of the owned particles on a local mesh of nx/P + 1 planes, the
   last plane being the next slab's first (the CIC corners at x + 1).  The
   particles' x anchors are re-based so that the local binning is the global
   one shifted by the slab origin: the same cells and bitwise the same
   fractions;
2. mesh halo: that plane goes to rank r + 1, which adds it to its first plane;
3. Poisson source, rfft over (y, z) of the slab, all-to-all transpose to ky
   slabs of ny / P columns, fft over x, the Green x gradient multiplier
   (the pmb_green_gradient kernel on the tables of the ky slab), inverse fft
   over x, transpose back, irfft over (y, z): three force slabs;
4. force halo: rank r + 1's first plane comes back as local plane nx/P, and
   the owned particles gather from the local mesh (the cell-sorted gather).

After every drift the particles go to the rank that owns their new cell: the
matrix of per-rank counts is gathered first, so every rank sees the same
totals and, when one would exceed its capacity, every rank raises the same
error before any particle moves (fail closed, no rank left in a collective).

The collectives go through a communicator: ProcessGroupComm (one rank per
process) or LocalComm, which runs P ranks in one process on one device with
the same exchange semantics (used to check the decomposition on one GPU).
The transforms of step 3 are cuFFT's (through torch.fft); the deposit,
gather, multiplier and kicks are this package's kernels.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from ._lib import call
from .cic import SortedParticles
from .gravity import _om32
from .nbody import _f32, _schedule
from .runtime import stream_handle

# per-particle fields routed with a particle after pmid (3 x int16): float32 x 3 each
_FIELDS = ("disp", "vel", "acc", "disp_cot", "vel_cot", "acc_cot")


class ProcessGroupComm:
    """One rank per process over torch.distributed (NCCL on GPUs, gloo on CPU)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.local = [self.rank]

    def count_matrix(self, counts):
        """counts[0][j]: this rank's item count for rank j -> the P x P matrix
        (row i: rank i's counts) on every rank."""
        c = torch.tensor([int(v) for v in counts[0]], dtype=torch.int64)
        if self.dist.get_backend(self.group) == "nccl":
            c = c.cuda()
        rows = [torch.empty_like(c) for _ in range(self.world)]
        self.dist.all_gather(rows, c, group=self.group)
        return np.stack([r.cpu().numpy() for r in rows])

    def alltoallv(self, sends, matrix):
        """sends[0]: 1-D tensor of this rank's segments for ranks 0..P-1 in
        order (lengths matrix[rank]); returns the segments received from ranks
        0..P-1 in order, concatenated."""
        send = sends[0].contiguous()
        scnt = [int(v) for v in matrix[self.rank]]
        rcnt = [int(v) for v in matrix[:, self.rank]]
        recv = torch.empty(sum(rcnt), dtype=send.dtype, device=send.device)
        self.dist.all_to_all_single(recv, send, rcnt, scnt, group=self.group)
        return [recv]

    def allreduce_sum(self, value):
        """Sum of a float over the ranks (float64)."""
        t = torch.tensor([float(value)], dtype=torch.float64)
        if self.dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())

    def shift(self, tensors, offset):
        """Rank r receives the tensor of rank (r - offset) mod P."""
        t = tensors[0].contiguous()
        if self.world == 1:
            return [t.clone()]
        out = torch.empty_like(t)
        dst = (self.rank + offset) % self.world
        src = (self.rank - offset) % self.world
        ops = [self.dist.P2POp(self.dist.isend, t, dst, self.group),
               self.dist.P2POp(self.dist.irecv, out, src, self.group)]
        for req in self.dist.batch_isend_irecv(ops):
            req.wait()
        return [out]


class LocalComm:
    """P ranks in one process: the same exchanges as ProcessGroupComm, as copies."""

    def __init__(self, world):
        self.world = int(world)
        self.rank = None
        self.local = list(range(self.world))

    def count_matrix(self, counts):
        return np.array([[int(v) for v in c] for c in counts], dtype=np.int64)

    def alltoallv(self, sends, matrix):
        P = self.world
        segs = [list(torch.split(sends[i].contiguous(), [int(v) for v in matrix[i]])) for i in range(P)]
        return [torch.cat([segs[i][j] for i in range(P)]) for j in range(P)]

    def allreduce_sum(self, value):
        return float(value)  # the local ranks' values are already summed by the caller

    def shift(self, tensors, offset):
        P = self.world
        return [tensors[(r - offset) % P].clone() for r in range(P)]


@dataclass
class SlabParticles:
    """The particles one rank owns: global lattice anchors pmid (int16 x 3),
    displacements, velocities and accelerations (float32 x 3), and in a
    reverse sweep their cotangents."""
    pmid: torch.Tensor
    disp: torch.Tensor
    vel: torch.Tensor
    acc: torch.Tensor = None
    disp_cot: torch.Tensor = None
    vel_cot: torch.Tensor = None
    acc_cot: torch.Tensor = None


def _as_bytes(t):
    return t.contiguous().view(torch.uint8).reshape(t.shape[0], -1)


class SlabPM:
    """Slab-decomposed PM force and KDK integration (float32 build, continuum
    Green's function with the particle-Nyquist masks, spectral gradient)."""

    def __init__(self, conf, comm, capacity=None):
        nx, ny, nz = conf.mesh_shape
        P = comm.world
        if nx % P or ny % P:
            raise ValueError(f"mesh {conf.mesh_shape} does not split into {P} slabs along x and y")
        if conf.float_dtype != torch.float32:
            raise NotImplementedError("the slab decomposition runs in the float32 build")
        self.conf = conf
        self.comm = comm
        self.P = P
        self.nxl, self.nyl = nx // P, ny // P
        self.capacity = capacity
        self._tab = {}

    # -- ownership and routing -------------------------------------------------
    def cell_x(self, pmid, disp):
        """Global lower-corner x cell and floor(disp_x / cell), as the sort bins them
        (IEEE division, non-finite displacements binned as zero)."""
        q = disp[:, 0] / np.float32(self.conf.cell_size)
        q = torch.where(torch.isfinite(q), q, torch.zeros_like(q))
        fl = torch.floor(q).to(torch.int64)
        cx = torch.remainder(pmid[:, 0].to(torch.int64) + fl, self.conf.mesh_shape[0])
        return cx, fl

    def owner(self, pmid, disp):
        return self.cell_x(pmid, disp)[0] // self.nxl

    def cell_key(self, pmid, disp):
        """Raveled global lower-corner cell (x-major), binned as the sort bins it."""
        nx, ny, nz = self.conf.mesh_shape
        q = disp / np.float32(self.conf.cell_size)
        q = torch.where(torch.isfinite(q), q, torch.zeros_like(q))
        c = pmid.to(torch.int64) + torch.floor(q).to(torch.int64)
        c = torch.remainder(c, torch.tensor([nx, ny, nz], device=c.device))
        return (c[:, 0] * ny + c[:, 1]) * nz + c[:, 2]

    def distribute(self, pmid, disp, vel=None):
        """Each local rank's share of a particle set every process holds."""
        vel = torch.zeros_like(disp) if vel is None else vel
        own = self.owner(pmid, disp)
        out = []
        for r in self.comm.local:
            m = own == r
            out.append(SlabParticles(pmid[m].contiguous(), disp[m].contiguous(), vel[m].contiguous()))
        return out

    def migrate(self, states):
        """Route every particle to the rank owning its cell (after a drift).
        Received particles are merged in stable cell-key order (ties: source
        rank, then order there), as the reference's merge path keeps them.
        Raises on every rank, before moving anything, when a rank's total would
        exceed the capacity."""
        P = self.P
        # the fields every rank carries (the same on all ranks: a collective decision)
        fields = [f for f in _FIELDS if getattr(states[0], f) is not None]
        row = 6 + 12 * len(fields)
        sends, counts = [], []
        for st in states:
            dest = self.owner(st.pmid, st.disp)
            order = torch.argsort(dest, stable=True)
            rows = torch.cat([_as_bytes(st.pmid)] + [_as_bytes(getattr(st, f)) for f in fields], dim=1)
            sends.append(rows[order].reshape(-1))
            counts.append((torch.bincount(dest, minlength=P) * row).tolist())
        matrix = self.comm.count_matrix(counts)
        totals = matrix.sum(axis=0) // row
        if self.capacity is not None and int(totals.max()) > self.capacity:
            worst = int(np.argmax(totals))
            raise RuntimeError(f"slab routing: rank {worst} would hold {int(totals[worst])} particles, "
                               f"over its capacity {self.capacity}")
        recvs = self.comm.alltoallv(sends, matrix)
        out = []
        for rb in recvs:
            rows = rb.reshape(-1, row)
            pmid = rows[:, :6].contiguous().view(torch.int16)
            disp = rows[:, 6:18].contiguous().view(torch.float32)
            rows = rows[torch.argsort(self.cell_key(pmid, disp), stable=True)]
            vals = {f: rows[:, 6 + 12 * k:18 + 12 * k].contiguous().view(torch.float32) for k, f in enumerate(fields)}
            out.append(SlabParticles(rows[:, :6].contiguous().view(torch.int16), **vals))
        return out

    # -- force ------------------------------------------------------------------
    def _local_anchor(self, r, st):
        """pmid with x re-based so that binning on the local mesh gives cell x - x0."""
        cx, fl = self.cell_x(st.pmid, st.disp)
        p = st.pmid.clone()
        p[:, 0] = (cx - r * self.nxl - fl).to(torch.int16)
        return p

    def tables(self, r, device):
        """Green tables of rank r's ky slab: [kx ky kz cx cy cz (mx my mz)] with ky, cy, my cut."""
        key = (r, str(device))
        if key not in self._tab:
            conf = self.conf
            s = slice(r * self.nyl, (r + 1) * self.nyl)
            ks = list(conf.kvec)
            cs = [conf._neg_k(k, conf.cell_size) for k in ks]
            parts = [ks[0], ks[1][s], ks[2], cs[0], cs[1][s], cs[2]]
            if conf.has_particle_nyquist_masks:
                m = conf.particle_nyquist_masks()
                parts += [m[0], m[1][s], m[2]]
            self._tab[key] = torch.from_numpy(np.concatenate(parts).astype(np.float32)).to(device)
        return self._tab[key]

    def green(self, r, spec):
        """Rank r's multiplier: spec (nx, ny/P, nz/2+1) -> three gradient spectra."""
        nx, _, nz = self.conf.mesh_shape
        out = torch.empty((3,) + tuple(spec.shape), dtype=torch.complex64, device=spec.device)
        call("pmb_green_gradient", spec.data_ptr(), out.data_ptr(), nx, self.nyl, nz, self.tables(r, spec.device).data_ptr(),
             int(self.conf.has_particle_nyquist_masks), 0, None, None, 0, float(1.0 / self.conf.mesh_size),
             stream_handle(spec.device))
        return out

    def green_adjoint(self, r, spec3, post):
        """Transpose of rank r's multiplier: three spectra (3, nx, ny/P, nz/2+1) -> one."""
        nx, _, nz = self.conf.mesh_shape
        out = torch.empty(tuple(spec3.shape[1:]), dtype=torch.complex64, device=spec3.device)
        call("pmb_green_gradient_adjoint", spec3.data_ptr(), out.data_ptr(), nx, self.nyl, nz,
             self.tables(r, spec3.device).data_ptr(), int(self.conf.has_particle_nyquist_masks), 0, None, None, 0,
             float(post), stream_handle(spec3.device))
        return out[None]

    def _spectral(self, fields, mult, c_out):
        """Distributed transform of real slabs (c_in, nx/P, ny, nz): rfft over
        (y, z), all-to-all to ky slabs, fft over x, mult(r, spectra (c_in, nx,
        ny/P, nz/2+1)) -> (c_out, ...), inverse fft over x, all-to-all back,
        irfft over (y, z): real slabs (c_out, nx/P, ny, nz).  Unnormalised both
        ways, like the single-GPU chain."""
        nx, ny, nz = self.conf.mesh_shape
        P, nxl, nyl, nzh = self.P, self.nxl, self.nyl, nz // 2 + 1
        c_in = fields[0].shape[0]
        sends = []
        for f in fields:
            A = torch.fft.rfft2(f, dim=(2, 3))  # (c_in, nxl, ny, nzh)
            A = A.reshape(c_in, nxl, P, nyl, nzh).permute(2, 0, 1, 3, 4)  # ky slab j first
            sends.append(torch.view_as_real(A.contiguous()).reshape(-1))
        seg = c_in * nxl * nyl * nzh * 2
        recvs = self.comm.alltoallv(sends, np.full((P, P), seg, dtype=np.int64))
        backs = []
        for r, rb in zip(self.comm.local, recvs):
            B = torch.view_as_complex(rb.reshape(P, c_in, nxl, nyl, nzh, 2))  # rank order = x order
            B = B.permute(1, 0, 2, 3, 4).reshape(c_in, nx, nyl, nzh)
            G = mult(r, torch.fft.fft(B, dim=1).contiguous())
            g = torch.fft.ifft(G, dim=1, norm="forward")  # (c_out, nx, nyl, nzh)
            backs.append(torch.view_as_real(g.reshape(c_out, P, nxl, nyl, nzh).transpose(0, 1).contiguous()).reshape(-1))
        recvs = self.comm.alltoallv(backs, np.full((P, P), c_out * seg // c_in, dtype=np.int64))
        out = []
        for rb in recvs:
            g = torch.view_as_complex(rb.reshape(P, c_out, nxl, nyl, nzh, 2))  # rank order = ky order
            g = g.permute(1, 2, 0, 3, 4).reshape(c_out, nxl, ny, nzh)
            out.append(torch.fft.irfft2(g, s=(ny, nz), dim=(2, 3), norm="forward").contiguous())
        return out

    def spectral_force(self, sources, green=None):
        """Force slabs (3, nx/P, ny, nz) from Poisson-source slabs (nx/P, ny, nz):
        distributed rfft, multiplier, inverse.  green(r, spec) is the multiplier
        (the kernel by default)."""
        green = self.green if green is None else green
        mult = lambda r, spec: green(r, spec[0].contiguous())
        return self._spectral([s[None] for s in sources], mult, 3)

    def force(self, states, omega_m):
        """Accelerations of every local rank's particles (in their order)."""
        sorted_, exts = self._forward(states, omega_m)
        acc = [sp.gather(ext) for sp, ext in zip(sorted_, exts)]
        for st, a in zip(states, acc):
            st.acc = a
        return acc

    def _forward(self, states, omega_m):
        """Cell-sorted particles on the local meshes and the force meshes with
        their halo plane (3, nx/P + 1, ny, nz) of every local rank."""
        conf = self.conf
        nx, ny, nz = conf.mesh_shape
        L = self.nxl + 1
        sorted_ = [SortedParticles(self._local_anchor(r, st), st.disp, conf, mesh_shape=(L, ny, nz))
                   for r, st in zip(self.comm.local, states)]
        dens = [sp.scatter(channels=1, mode=0)[0] for sp in sorted_]  # (L, ny, nz)
        halo = self.comm.shift([d[self.nxl] for d in dens], 1)
        src_mul = np.float32(1.5 * _om32(omega_m))
        sources = []
        for d, h in zip(dens, halo):
            rho = d[: self.nxl].clone()
            rho[0] += h
            sources.append((rho - 1.0) * src_mul)
        F = self.spectral_force(sources)
        fh = self.comm.shift([f[:, 0] for f in F], -1)
        exts = [torch.cat([f, h[:, None]], dim=1).contiguous() for f, h in zip(F, fh)]  # (3, nxl + 1, ny, nz)
        return sorted_, exts

    def force_vjp(self, states, acc_cots, omega_m):
        """Displacement cotangents (d acc / d disp)^T acc_cot of every local
        rank's particles, the force recomputed at their positions; also sets
        each state's acc.  The transpose of force(): gather adjoint (position
        term, and the 3-channel deposit of acc_cot on the local mesh), the force
        halo plane back to the rank it came from, the distributed transform with
        the transposed multiplier (into the density cotangent, the source scale
        included), the density halo plane back, and the deposit's position term."""
        conf = self.conf
        nx, ny, nz = conf.mesh_shape
        sorted_, exts = self._forward(states, omega_m)
        dcs, mesh_cots = [], []
        for st, sp, ext, ac in zip(states, sorted_, exts, acc_cots):
            st.acc = sp.gather(ext)
            cot_sorted = torch.empty_like(ac)
            dc, _ = sp.interp_grad(ext, u=ac.contiguous(), u_sorted=cot_sorted)
            dcs.append(dc)
            mesh_cots.append(sp.scatter(val=cot_sorted, channels=3, mode=0, val_sorted=True))  # (3, L, ny, nz)
        back = self.comm.shift([m[:, self.nxl] for m in mesh_cots], 1)
        fields = []
        for m, b in zip(mesh_cots, back):
            g = m[:, : self.nxl].clone()
            g[:, 0] += b
            fields.append(g)
        post = float(np.float32(1.5 * _om32(omega_m)) / conf.mesh_size)
        rho_cots = self._spectral(fields, lambda r, spec: self.green_adjoint(r, spec, post), 1)
        hb = self.comm.shift([rc[0, 0] for rc in rho_cots], -1)
        vc = float(conf.mesh_size / conf.ptcl_num)
        for sp, rc, h, dc in zip(sorted_, rho_cots, hb, dcs):
            dens_cot = torch.cat([rc[0], h[None]], dim=0)[None].contiguous()  # (1, nxl + 1, ny, nz)
            sp.interp_grad(dens_cot, u_const=vc, disp_cot=dc, accumulate=True)
        return dcs

    # -- time integration -------------------------------------------------------
    def nbody(self, states, cosmo, a_nbody=None):
        """KDK integration (the stage list of nbody.integrate) on the slabs;
        particles are routed after every drift."""
        conf = self.conf
        a = conf.a_nbody if a_nbody is None else np.asarray(a_nbody)
        self.force(states, cosmo.Omega_m)
        for a_prev, a_next in zip(a[:-1], a[1:]):
            for st in _schedule(a_prev, a_next, conf):
                if st[0] == "drift":
                    D = _f32(cosmo.drift_factor(st[1], st[2], st[3]))
                    for p in states:
                        call("pmb_axpy", p.disp.data_ptr(), p.vel.data_ptr(), p.disp.numel(), D,
                             stream_handle(p.disp.device))
                    states = self.migrate(states)
                    self.force(states, cosmo.Omega_m)
                else:
                    K = _f32(cosmo.kick_factor(st[1], st[2], st[3]))
                    for p in states:
                        call("pmb_axpy", p.vel.data_ptr(), p.acc.data_ptr(), p.vel.numel(), K,
                             stream_handle(p.vel.device))
        return states

    def nbody_adj(self, states, cosmo, a_nbody=None):
        """Reverse sweep on the slabs from the final state.  states hold pmid,
        disp, vel, acc at the last time and the cotangents disp_cot, vel_cot
        (acc_cot: zero when None).  Runs the per-operation adjoints of
        nbody.integrate_adj (kick adjoint, force adjoint, drift adjoint, force
        recompute) with the particles and their cotangents routed after every
        reverse drift, then the initial force's adjoint.  Returns the initial
        states (with their cotangents) and the Omega_m cotangent, summed over
        all ranks."""
        conf = self.conf
        a = conf.a_nbody if a_nbody is None else np.asarray(a_nbody)
        om32 = _om32(cosmo.Omega_m)
        for st in states:
            for f in ("disp_cot", "vel_cot", "acc_cot"):
                t = getattr(st, f)
                setattr(st, f, torch.zeros_like(st.disp) if t is None else t.clone().float().contiguous())
        om_local = 0.0

        def force_adj(states):
            dcs = self.force_vjp(states, [st.acc_cot for st in states], cosmo.Omega_m)
            tot = 0.0
            for st, dc in zip(states, dcs):
                st.disp_cot += dc
                tot += float((st.acc_cot.double() * st.acc.double()).sum())
                st.acc_cot.zero_()
            return tot / om32

        for a_prev, a_next in list(zip(a[:-1], a[1:]))[::-1]:
            for st in reversed(_schedule(a_prev, a_next, conf)):
                if st[0] == "kick":
                    K, dK = cosmo.kick_factor(st[1], st[2], st[3], with_grad=True)
                    for p in states:
                        dot = torch.zeros(1, dtype=torch.float64, device=p.vel.device)
                        call("pmb_kick_adj", p.vel.data_ptr(), p.acc.data_ptr(), p.vel_cot.data_ptr(),
                             p.acc_cot.data_ptr(), p.vel.numel(), _f32(K), dot.data_ptr(), stream_handle(p.vel.device))
                        om_local += dK * float(dot.item())
                    continue
                _, a_vel, a_disp, a_disp_next, a_acc_in = st
                om_local += force_adj(states)
                D, dD = cosmo.drift_factor(a_vel, a_disp, a_disp_next, with_grad=True)
                for p in states:
                    dot = torch.zeros(1, dtype=torch.float64, device=p.disp.device)
                    call("pmb_drift_adj", p.disp.data_ptr(), p.vel.data_ptr(), p.disp_cot.data_ptr(),
                         p.vel_cot.data_ptr(), p.disp.numel(), _f32(D), dot.data_ptr(), stream_handle(p.disp.device))
                    om_local += dD * float(dot.item())
                states = self.migrate(states)
                self.force(states, cosmo.Omega_m)
        om_local += force_adj(states)
        return states, self.comm.allreduce_sum(om_local)

    def collect(self, states):
        """Concatenate local ranks' particles and order them by anchor cell
        (LocalComm, or the local ranks of one process)."""
        _, ny, nz = self.conf.mesh_shape
        pmid = torch.cat([s.pmid for s in states]).to(torch.int64)
        ids = (pmid[:, 0] * ny + pmid[:, 1]) * nz + pmid[:, 2]
        order = torch.argsort(ids)
        cat = lambda name: torch.cat([getattr(s, name) for s in states])[order]
        return cat("pmid"), cat("disp"), cat("vel"), (cat("acc") if states[0].acc is not None else None)
