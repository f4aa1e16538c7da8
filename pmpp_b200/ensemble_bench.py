"""Ensemble throughput: many independent simulations of uneven sizes.

Default workload: 96 simulations, 32 each of 64^3 particles / 128^3 mesh,
96^3 / 192^3 and 128^3 / 256^3; boxes U[128, 512] Mpc/h, Omega_m ~
U[0.25, 0.35], sigma8 ~ U[0.7, 0.9] (numpy PCG64 seed 4), nested white noise
with the member index as seed, 2LPT at a = 0.1, then 20 log-spaced
kick-drift-kick steps to a = 1.

Timed with CUDA events: the initial conditions looped eagerly and as the
ensemble's graph-replayed batch, the ensemble N-body run (autotuned persistent
launches, one graph-replayed step per macro step), the whole ensemble run
(batched ICs + N-body; sims/s), and the same N-body runs looped one
simulation at a time, eagerly and with each member's whole run captured in its
own CUDA graph.  The ensemble's final positions are checked against the looped
runs.

    python -m pmpp_b200.ensemble_bench --per-size 32 --out ensemble.json
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import lpt as _lpt
from . import modes as _modes
from .configuration import Configuration
from .cosmology import Cosmology
from .ensemble import Ensemble
from .graphs import GraphedForward
from .nbody import NBodyRun

SIZES = ((64, 2), (96, 2), (128, 2))


def members(per_size=32, nsteps=20, sizes=SIZES, seed=4, device="cuda"):
    rng = np.random.Generator(np.random.PCG64(seed))
    a = np.geomspace(0.1, 1.0, nsteps + 1)
    confs, coss = [], []
    for n, mesh in sizes:
        for _ in range(per_size):
            box = float(rng.uniform(128.0, 512.0))
            om, s8 = float(rng.uniform(0.25, 0.35)), float(rng.uniform(0.7, 0.9))
            conf = Configuration(box / n, (n, ) * 3, mesh, a_start=0.1, a_custom=a, device=device)
            confs.append(conf)
            coss.append(Cosmology.from_sigma8(conf, s8, n_s=0.96, Omega_m=om, Omega_b=0.05, h=0.7))
    return confs, coss


def initial_conditions(confs, coss):
    return [_lpt.lpt(_modes.linear_modes(_modes.white_noise_nested(k, c), cs, c), cs, c)
            for k, (c, cs) in enumerate(zip(confs, coss))]


class _Timer:
    def __enter__(self):
        torch.cuda.synchronize()
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)
        self.e0.record()
        return self

    def __exit__(self, *exc):
        self.e1.record()
        torch.cuda.synchronize()
        self.ms = self.e0.elapsed_time(self.e1)


def run(per_size=32, nsteps=20, reps=3, sizes=SIZES, tune_cache=None, loop=True):
    confs, coss = members(per_size, nsteps, sizes)
    ics = initial_conditions(confs, coss)  # warm-up of the IC kernels and plans
    with _Timer() as t_ic:
        ics = initial_conditions(confs, coss)
    ens = Ensemble(confs, coss)
    ens.load(ics)
    ens.force()
    tuning = ens.autotune(cache=tune_cache)
    out = ens.forward(ics, graph=True)  # capture + warm-up
    times = []
    for _ in range(reps):
        with _Timer() as t:
            ens.forward(ics, graph=True)
        times.append(t.ms)
    t_ens = float(np.median(times))
    # whole ensemble run: batched, graph-replayed 2LPT initial conditions + N-body
    seeds = list(range(len(confs)))
    ens.run(seeds, graph=True)
    full = []
    for _ in range(reps):
        with _Timer() as t:
            ens.run(seeds, graph=True)
        full.append(t.ms)
    t_full = float(np.median(full))
    with _Timer() as t_icg:
        ens.initial_conditions(seeds, graph=True)
    n_total = sum(c.ptcl_num for c in confs)
    res = {
        "config": {"members": len(confs), "sizes": [f"{n}^3/{(n * m)}^3" for n, m in sizes], "per_size": per_size,
                   "kdk_steps": nsteps, "particles": n_total, "mesh_cells": sum(c.mesh_size for c in confs)},
        "ic_ms_loop": t_ic.ms,
        "ic_ms_graphed": t_icg.ms,
        "ensemble_nbody_ms": t_ens,
        "ensemble_run_ms": t_full,
        "ensemble_particle_steps_per_s": n_total * nsteps / (t_ens * 1e-3),
        "ensemble_sims_per_s": len(confs) / (t_full * 1e-3),
        "tuning": {"tiles": tuning["tiles"], "launches": tuning["launches"]},
    }
    if loop:
        runs = [NBodyRun(c, cs) for c, cs in zip(confs, coss)]
        refs = [r.forward(ic) for r, ic in zip(runs, ics)]
        with _Timer() as t_loop:
            refs = [r.forward(ic) for r, ic in zip(runs, ics)]
        err = max(float((o.disp - r.disp).abs().max() / r.disp.abs().max()) for o, r in zip(out, refs))
        del refs
        graphs = [GraphedForward(c, cs, ic) for c, cs, ic in zip(confs, coss, ics)]
        with _Timer() as t_graph:
            for g in graphs:
                g()
        del graphs
        res.update({
            "loop_eager_nbody_ms": t_loop.ms,
            "loop_graphed_nbody_ms": t_graph.ms,
            "speedup_vs_loop_eager": t_loop.ms / t_ens,
            "speedup_vs_loop_graphed": t_graph.ms / t_ens,
            "loop_sims_per_s": len(confs) / ((t_loop.ms + t_ic.ms) * 1e-3),
            "max_rel_disp_diff_vs_loop": err,
        })
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--per-size", type=int, default=32)
    ap.add_argument("--sizes", default="64:2,96:2,128:2", help="particles-per-side:mesh-factor list")
    ap.add_argument("--nsteps", type=int, default=20)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--tune-cache", default=None)
    ap.add_argument("--no-loop", action="store_true")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    sizes = tuple(tuple(int(v) for v in item.split(":")) for item in args.sizes.split(","))
    res = run(args.per_size, args.nsteps, args.reps, sizes=sizes, tune_cache=args.tune_cache, loop=not args.no_loop)
    print(json.dumps(res))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)
    return res


if __name__ == "__main__":
    main()
