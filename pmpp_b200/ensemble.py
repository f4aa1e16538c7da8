"""Ensembles of independent PM simulations of uneven sizes (pmb_ens_* C ABI).

The reference advances one simulation per call (nbody/solver.py:253-273).
``Ensemble`` advances many together: every PM stage (sort with the drift
fused, Poisson-source scatter, R2C, Green x gradient, 3 x C2R, gather with the
closing kick fused, the opening kick) is one persistent launch over all
members, FFTs are one batched cuFFT plan per distinct mesh shape, and the
kick-drift-kick step is captured once in a CUDA graph and replayed for every
step (per-member time factors come from a device table indexed by a
device-side step counter).  Each member gets exactly the single-simulation
arithmetic, so with one member per mesh shape an ensemble run equals
``NBodyRun.forward`` of every member bit for bit.

``autotune`` is the project's tuner: it times the persistent scatter per mesh
shape over candidate tile shapes, and the particle / cell stages over thread
and CTA-per-SM counts, keeps the fastest, and can cache the choice in a JSON
file keyed by device and ensemble layout.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import torch

from . import modes as _modes
from ._lib import call, lib
from .gravity import _om32
from .nbody import _schedule
from .particles import Particles
from .runtime import stream_handle

STAGES = {"kick": 0, "sort": 1, "scatter": 2, "r2c": 3, "green": 4, "c2r": 5, "gather": 6}
TILE_CANDIDATES = ((1, 1), (1, 2), (2, 1), (2, 2), (1, 4), (4, 1), (2, 4), (4, 2), (3, 3), (4, 4))
LAUNCH_CANDIDATES = ((128, 8), (256, 4), (256, 8), (512, 2), (512, 4), (1024, 2))


def _f32(x):
    return float(np.float32(x))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def step_factors(conf, cosmo):
    """[nsteps][3] float32 (opening kick, drift, closing kick) of the default
    kick-drift-kick splitting (integrator.py:125-170, 760-778)."""
    a = conf.a_nbody
    out = np.zeros((len(a) - 1, 3), np.float32)
    for k, (a0, a1) in enumerate(zip(a[:-1], a[1:])):
        st = _schedule(a0, a1, conf)
        if [s[0] for s in st] != ["kick", "drift", "kick"]:
            raise NotImplementedError("ensembles support the default kick-drift-kick splitting only")
        out[k, 0] = _f32(cosmo.kick_factor(st[0][1], st[0][2], st[0][3]))
        out[k, 1] = _f32(cosmo.drift_factor(st[1][1], st[1][2], st[1][3]))
        out[k, 2] = _f32(cosmo.kick_factor(st[2][1], st[2][2], st[2][3]))
    return out


class Ensemble:
    """Independent PM simulations advanced together.

    confs / cosmos: one Configuration and Cosmology per member (any particle
    grid, mesh and box; the same number of N-body steps).  Members are stored
    by decreasing mesh size with equal shapes contiguous; every method takes
    and returns them in the caller's order."""

    def __init__(self, confs, cosmos, device=None):
        if len(confs) != len(cosmos) or not confs:
            raise ValueError("one cosmology per configuration, at least one member")
        self.device = torch.device(device if device is not None else confs[0].device)
        self.confs, self.cosmos = list(confs), list(cosmos)
        n = len(confs)
        self.order = sorted(range(n), key=lambda i: (-confs[i].mesh_size, confs[i].mesh_shape, i))
        cs = [confs[i] for i in self.order]
        nsteps = {len(c.a_nbody) - 1 for c in confs}
        if len(nsteps) != 1:
            raise ValueError("members must take the same number of N-body steps")
        self.nsteps = nsteps.pop()
        counts = np.array([c.ptcl_num for c in cs], np.int64)
        shapes = np.array([c.mesh_shape for c in cs], np.int32).reshape(-1)
        cells = np.array([c.cell_size for c in cs], np.float32)
        vals = np.array([c.mesh_size / c.ptcl_num for c in cs], np.float32)
        muls = np.array([1.5 * _om32(self.cosmos[i].Omega_m) for i in self.order], np.float32)
        masks = np.array([int(c.has_particle_nyquist_masks) for c in cs], np.int32)
        h = ctypes.c_void_p()
        call("pmb_ens_create", n, _ptr(counts), _ptr(shapes), _ptr(cells), _ptr(vals), _ptr(muls), _ptr(masks),
             self.nsteps, ctypes.byref(h))
        self.handle = h
        L = lib()
        self.ntot = int(L.pmb_ens_size(h, 0))
        ncells, nspec = int(L.pmb_ens_size(h, 1)), int(L.pmb_ens_size(h, 2))
        dev = self.device
        self.pstart = np.concatenate([[0], np.cumsum(counts)])
        self.pmid = torch.empty((self.ntot, 3), dtype=torch.int16, device=dev)
        self.disp = torch.zeros((self.ntot, 3), dtype=torch.float32, device=dev)
        self.vel = torch.zeros_like(self.disp)
        self.acc = torch.zeros_like(self.disp)
        self.rho = torch.empty(ncells, dtype=torch.float32, device=dev)
        self.rho_hat = torch.empty(nspec, dtype=torch.complex64, device=dev)
        self.grad_hat = torch.empty(3 * nspec, dtype=torch.complex64, device=dev)
        self.force_meshes = torch.empty(3 * ncells, dtype=torch.float32, device=dev)
        tabs = [c.spectral_tables("mesh", dev, 0) for c in cs]
        self.table_offsets = np.concatenate([[0], np.cumsum([t.numel() for t in tabs])[:-1]]).astype(np.int64)
        self.tables = torch.cat(tabs)
        wb = int(L.pmb_ens_workspace_bytes(h))
        self.workspace = torch.empty(wb + 256, dtype=torch.uint8, device=dev)
        base = self.workspace.data_ptr()
        self.ws_ptr = (base + 255) // 256 * 256
        s = stream_handle(dev)
        call("pmb_ens_bind", h, self.pmid.data_ptr(), self.disp.data_ptr(), self.vel.data_ptr(), self.acc.data_ptr(),
             self.rho.data_ptr(), self.rho_hat.data_ptr(), self.grad_hat.data_ptr(), self.force_meshes.data_ptr(),
             self.tables.data_ptr(), _ptr(self.table_offsets), self.ws_ptr, wb, s)
        fac = np.stack([step_factors(confs[i], cosmos[i]) for i in self.order], axis=1)  # [steps][nsims][3]
        self.factors = np.ascontiguousarray(fac, dtype=np.float32)
        call("pmb_ens_set_factors", h, self.nsteps, _ptr(self.factors), s)
        torch.cuda.synchronize(dev)
        self.graph = None
        self.tuning = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize(self.device)
                lib().pmb_ens_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ---- member slices ----------------------------------------------------
    def _slot(self, i):
        j = self.order.index(i)
        return slice(int(self.pstart[j]), int(self.pstart[j + 1]))

    def load(self, ptcls):
        """Copy each member's pmid / disp / vel (Particles, caller order)."""
        for i, p in enumerate(ptcls):
            sl = self._slot(i)
            self.pmid[sl].copy_(p.pmid)
            self.disp[sl].copy_(p.disp)
            if p.vel is not None:
                self.vel[sl].copy_(p.vel)
            else:
                self.vel[sl].zero_()

    def particles(self, i, clone=True):
        sl = self._slot(i)
        c = (lambda t: t.clone()) if clone else (lambda t: t)
        return Particles(self.confs[i], c(self.pmid[sl]), c(self.disp[sl]), c(self.vel[sl]), c(self.acc[sl]))

    # ---- initial conditions ---------------------------------------------------
    def _prepare_ics(self):
        """Device tables, lattices and scratch of the per-member 2LPT sequence."""
        dev = self.device
        L = lib()
        self._ic = []
        half = max(c.ptcl_grid_shape[0] * c.ptcl_grid_shape[1] * (c.ptcl_grid_shape[2] // 2 + 1) for c in self.confs)
        cells = max(c.ptcl_num for c in self.confs)
        wsb = max(int(L.pmb_lpt_workspace_bytes(*c.ptcl_grid_shape)) for c in self.confs)
        self._ic_modes = torch.empty((2, half), dtype=torch.complex64, device=dev)
        self._ic_fields = torch.empty((6, cells), dtype=torch.float32, device=dev)
        self._ic_ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        for i, (conf, cos) in enumerate(zip(self.confs, self.cosmos)):
            lat = Particles.gen_grid(conf, device=dev)
            fac, _ = cos.lpt_factors(conf.a_start)
            self._ic.append({
                "lin": _modes._Tables(cos, conf, dev), "pmid": lat.pmid, "disp": lat.disp,
                "ptab": conf.spectral_tables("particle", dev),
                "fac": tuple(_f32(x) for x in (fac[0, 0], fac[0, 2], fac[1, 0], fac[1, 2])),
            })
        self._ic_graph = None

    def _ic_sequence(self, seeds):
        s = stream_handle(self.device)
        ma, mb = self._ic_modes[0], self._ic_modes[1]
        for i, (conf, cos) in enumerate(zip(self.confs, self.cosmos)):
            d = self._ic[i]
            gx, gy, gz = conf.ptcl_grid_shape
            sl = self._slot(i)
            self.pmid[sl].copy_(d["pmid"])
            self.disp[sl].copy_(d["disp"])
            self.vel[sl].zero_()
            call("pmb_white_noise_nested", int(seeds[i]) & 0xFFFFFFFF, gx, gy, gz, ma.data_ptr(), None, s)
            tb = d["lin"]
            call("pmb_linear_modes", ma.data_ptr(), mb.data_ptr(), None, gx, gy, gz, tb.k.data_ptr(), tb.tk.data_ptr(),
                 tb.tt.data_ptr(), int(tb.tk.numel()), float(cos.A_s), float(cos.n_s), float(cos.Omega_m),
                 float(cos.k_pivot), 1.0, float(conf.box_vol), s)
            D1, V1, D2, V2 = d["fac"]
            p0 = self.pmid[sl]
            call("pmb_lpt", mb.data_ptr(), gx, gy, gz, float(conf.ptcl_spacing), float(conf.ptcl_cell_vol),
                 d["ptab"].data_ptr(), int(conf.lpt_order), D1, V1, D2, V2, p0.data_ptr(), self.disp[sl].data_ptr(),
                 self.vel[sl].data_ptr(), conf.ptcl_num, float(conf.cell_size), self._ic_fields.data_ptr(), None,
                 self._ic_ws.data_ptr(), self._ic_ws.numel(), s)

    def initial_conditions(self, seeds, graph=True):
        """2LPT initial conditions of every member (nested white noise with the
        member's seed -> linear modes -> 2LPT at a_start), written straight into
        the ensemble's particle buffers.  The per-member kernel sequence is the
        single-simulation one (so members equal ``lpt(linear_modes(
        white_noise_nested(seed)))`` bit for bit); with graph it is captured once
        in a CUDA graph per seed list and replayed."""
        seeds = tuple(int(x) for x in seeds)
        if len(seeds) != len(self.confs):
            raise ValueError("one seed per member")
        if not hasattr(self, "_ic"):
            self._prepare_ics()
        if not graph:
            self._ic_sequence(seeds)
            return
        if self._ic_graph is None or self._ic_graph[0] != seeds:
            self._ic_sequence(seeds)  # uncaptured first: cuFFT plans exist before capture
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._ic_sequence(seeds)
            self._ic_graph = (seeds, g)
        self._ic_graph[1].replay()

    def run(self, seeds, graph=True):
        """Initial conditions plus the N-body run; returns the final Particles."""
        self.initial_conditions(seeds, graph=graph)
        if graph and self.graph is None:
            self.capture()
        self.set_step(0)
        self.force()
        for _ in range(self.nsteps):
            if graph:
                self.graph.replay()
            else:
                self.step()
        return [self.particles(i) for i in range(len(self.confs))]

    # ---- stages -------------------------------------------------------------
    def stage(self, name, drift=0, kick=0):
        call("pmb_ens_stage", self.handle, STAGES[name], drift, kick, stream_handle(self.device))

    def force(self, drift=0, kick=0):
        call("pmb_ens_force", self.handle, drift, kick, stream_handle(self.device))

    def set_step(self, k):
        call("pmb_ens_set_step", self.handle, k, stream_handle(self.device))

    def step(self):
        call("pmb_ens_step", self.handle, stream_handle(self.device))

    def capture(self):
        """Capture one kick-drift-kick step (pmb_ens_step) in a CUDA graph."""
        self.force()  # uncaptured call: uploads descriptors, creates FFT plans
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step()
        self.graph = g
        return g

    def forward(self, ptcls=None, graph=True):
        """Initial force, then every kick-drift-kick step; returns the members'
        final Particles in caller order."""
        if ptcls is not None:
            self.load(ptcls)
        if graph and self.graph is None:
            self.capture()
        self.set_step(0)
        self.force()
        for _ in range(self.nsteps):
            if graph:
                self.graph.replay()
            else:
                self.step()
        return [self.particles(i) for i in range(len(self.confs))]

    # ---- autotuner ------------------------------------------------------------
    def _time(self, fn, reps):
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(self.device)
        return e0.elapsed_time(e1) / reps

    def _layout_key(self):
        name = torch.cuda.get_device_name(self.device)
        members = sorted(f"{c.ptcl_grid_shape}/{c.mesh_shape}" for c in self.confs)
        return name + "|" + ",".join(members)

    def _apply(self, tiles, launches):
        rx = np.array([tiles[str(self.confs[i].mesh_shape)][0] for i in self.order], np.int32)
        ry = np.array([tiles[str(self.confs[i].mesh_shape)][1] for i in self.order], np.int32)
        call("pmb_ens_set_tiles", self.handle, _ptr(rx), _ptr(ry))
        for name, (th, ct) in launches.items():
            call("pmb_ens_set_launch", self.handle, STAGES[name], th, ct)

    def autotune(self, reps=5, cache=None):
        """Pick scatter tile shapes per mesh shape and launch shapes per stage
        by timing the persistent launches on the loaded particles."""
        key = self._layout_key()
        if cache is not None and os.path.exists(cache):
            with open(cache) as f:
                saved = json.load(f)
            if key in saved:
                self.tuning = saved[key]
                self._apply(self.tuning["tiles"], {k: tuple(v) for k, v in self.tuning["launches"].items()})
                return self.tuning
        shapes = []
        for i in self.order:
            ms = self.confs[i].mesh_shape
            if ms not in shapes:
                shapes.append(ms)
        tiles = {str(ms): (2, 2) for ms in shapes}
        launches = {}
        self._apply(tiles, launches)
        self.stage("sort")
        timings = {}
        for ms in shapes:
            best = None
            for rx, ry in TILE_CANDIDATES:
                if rx > ms[0] or ry > ms[1] or rx * ry * ms[2] * 12 > 200 * 1024:
                    continue
                trial = dict(tiles)
                trial[str(ms)] = (rx, ry)
                self._apply(trial, launches)
                t = self._time(lambda: self.stage("scatter"), reps)
                timings[f"scatter{ms}:{rx}x{ry}"] = t
                if best is None or t < best[0]:
                    best = (t, (rx, ry))
            tiles[str(ms)] = best[1]
        self._apply(tiles, launches)
        for name in ("sort", "green", "gather"):
            best = None
            for th, ct in LAUNCH_CANDIDATES:
                call("pmb_ens_set_launch", self.handle, STAGES[name], th, ct)
                t = self._time(lambda: self.stage(name), reps)
                timings[f"{name}:{th}x{ct}"] = t
                if best is None or t < best[0]:
                    best = (t, (th, ct))
            launches[name] = best[1]
            call("pmb_ens_set_launch", self.handle, STAGES[name], *best[1])
        launches["kick"] = launches["gather"]
        self._apply(tiles, launches)
        self.graph = None  # launch shapes changed: recapture
        self.tuning = {"tiles": {k: list(v) for k, v in tiles.items()},
                       "launches": {k: list(v) for k, v in launches.items()}, "timings_ms": timings}
        if cache is not None:
            saved = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    saved = json.load(f)
            saved[key] = self.tuning
            with open(cache, "w") as f:
                json.dump(saved, f, indent=1)
        return self.tuning
