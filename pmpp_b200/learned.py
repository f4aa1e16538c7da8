"""Learned Green's-function correction experiment: a coarse force mesh standing in
for a 3x finer one.

128^3 particles in a 256 Mpc/h box; the coarse run uses a 128^3 force mesh with
the ``LearnedGreen`` correction, the target is the same initial conditions run
with a plain 384^3 force mesh.  Omega_m ~ U[0.25, 0.35] and sigma8 ~ U[0.7, 0.9]
per seed.  Training minimises the mean squared log ratio of the coarse P(k)
to the fine P(k) (both measured on the 128^3 analysis mesh, CIC deconvolved)
for k <= 0.5 h/Mpc, with gradients from the hand-written adjoints
(P(k) loss adjoint -> N-body reverse sweep -> per-|n|^2 transfer cotangents ->
MLP backward kernel).  Evaluation on held-out seeds: max |P/P_fine - 1| for
k <= 0.5 h/Mpc and the cross-correlation of the final densities, for the
plain and the learned coarse runs, and the GPU time of a learned 128^3 run
against a plain 384^3 run.

    python -m pmpp_b200.learned --train 64 --test 16 --iters 300 --out learned.json

Under torchrun the training seeds are split across ranks (one GPU each) and
the MLP gradient is averaged over ranks every step (the one all-reduce of the
replicated path); rank 0 evaluates and writes the results.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import lpt as _lpt
from . import modes as _modes
from . import power_spectrum as _ps
from .configuration import Configuration
from .corrections import LearnedGreen
from .cosmology import Cosmology
from .nbody import NBodyRun
from .particles import Particles

BOX = 256.0
NP = 128


def configs(nsteps=20, device="cuda"):
    a = np.geomspace(0.1, 1.0, nsteps + 1)
    sp = BOX / NP
    coarse = Configuration(sp, (NP, ) * 3, 1, a_start=0.1, a_custom=a, device=device)
    fine = Configuration(sp, (NP, ) * 3, 3, a_start=0.1, a_custom=a, device=device)
    return coarse, fine


def draw_cosmology(seed):
    r = np.random.default_rng(10_000 + seed)
    return float(r.uniform(0.25, 0.35)), float(r.uniform(0.7, 0.9))


class Sample:
    def __init__(self, seed, coarse, fine):
        om, s8 = draw_cosmology(seed)
        kw = dict(n_s=0.96, Omega_m=om, Omega_b=0.05, h=0.7)
        self.seed, self.om, self.s8 = seed, om, s8
        self.cos_c = Cosmology.from_sigma8(coarse, s8, **kw)
        self.cos_f = Cosmology.from_sigma8(fine, s8, **kw)
        for c in (self.cos_c, self.cos_f):
            object.__setattr__(c, "_sigma8_cached", s8)
        noise = _modes.white_noise_nested(seed, coarse)
        lin = _modes.linear_modes(noise, self.cos_c, coarse)
        self.ic = _lpt.lpt(lin, self.cos_c, coarse)  # identical particle grid for both meshes


def run_forward(sample, conf, cosmo, correction=None):
    grid = Particles.gen_grid(conf, vel=True, device=sample.ic.disp.device)
    p0 = Particles(conf, grid.pmid, sample.ic.disp.clone(), sample.ic.vel.clone())
    run = NBodyRun(conf, cosmo, correction)
    out = run.forward(p0)
    return run, out


def pk_of(disp, coarse):
    grid = Particles.gen_grid(coarse, device=disp.device)
    return _ps.particles_to_pk(Particles(coarse, grid.pmid, disp), coarse)


def density(disp, coarse):
    from .cic import SortedParticles
    grid = Particles.gen_grid(coarse, device=disp.device)
    return SortedParticles(grid.pmid, disp, coarse).scatter()[0]


def graphed_runs(smp, coarse, fine, model):
    """CUDA-graph-captured forward runs: learned 128^3 mesh and plain 384^3 mesh."""
    from .graphs import GraphedForward
    pc = Particles(coarse, Particles.gen_grid(coarse, device=smp.ic.disp.device).pmid, smp.ic.disp, smp.ic.vel)
    pf = Particles(fine, Particles.gen_grid(fine, device=smp.ic.disp.device).pmid, smp.ic.disp, smp.ic.vel)
    return GraphedForward(coarse, smp.cos_c, pc, model), GraphedForward(fine, smp.cos_f, pf)


def evaluate(params_path, test_seeds=range(64, 80), nsteps=20, kmax=0.5):
    """Held-out evaluation with stored parameters (float32 .npy of weights then biases).

    Returns plain / learned max |P/P_fine - 1| (k <= kmax) averaged over the
    seeds, the smallest cross-correlation coefficient r(k) (k <= kmax) of the
    final density of each coarse run with the plain 384^3 run's (both
    deposited on the 128^3 grid; power_spectrum.py:308-345), and the
    CUDA-graph times of a learned 128^3 and a plain 384^3 run."""
    coarse, fine = configs(nsteps)
    model = LearnedGreen("cuda", seed=0)
    model.load_parameters(torch.from_numpy(np.load(params_path)))
    ep, el, rp, rl = [], [], [], []
    for s in test_seeds:
        smp = Sample(s, coarse, fine)
        _, out_f = run_forward(smp, fine, smp.cos_f)
        tgt = pk_of(out_f.disp, coarse)
        sel = tgt[0] <= kmax
        _, plain = run_forward(smp, coarse, smp.cos_c)
        _, learn = run_forward(smp, coarse, smp.cos_c, model)
        ep.append(float(np.max(np.abs(pk_of(plain.disp, coarse)[1][sel] / tgt[1][sel] - 1))))
        el.append(float(np.max(np.abs(pk_of(learn.disp, coarse)[1][sel] / tgt[1][sel] - 1))))
        rho_f = density(out_f.disp, coarse)
        for out, acc in ((plain, rp), (learn, rl)):
            k, r = _ps.density_to_cross_correlation(density(out.disp, coarse), rho_f, coarse)[:2]
            acc.append(float(np.min(r[k <= kmax])))
    g_learn, g_fine = graphed_runs(smp, coarse, fine, model)
    tl = gpu_time(g_learn, reps=10)
    tf = gpu_time(g_fine, reps=5)
    return {"seeds": len(ep), "max_pk_err_plain_128": float(np.mean(ep)), "max_pk_err_learned_128": float(np.mean(el)),
            "worst_pk_err_learned_128": float(np.max(el)), "min_r_plain_128": float(np.min(rp)),
            "min_r_learned_128": float(np.min(rl)), "kmax": kmax, "time_ms_learned_128": tl,
            "time_ms_plain_384": tf, "speedup": tf / tl}


def gpu_time(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=64)
    ap.add_argument("--test", type=int, default=16)
    ap.add_argument("--iters", type=int, default=300)
    ap.add_argument("--nsteps", type=int, default=20)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--kmax", type=float, default=0.5)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    from . import replicas
    rank, world, _ = replicas.setup()
    coarse, fine = configs(args.nsteps)
    t0 = time.time()
    mine = [s for s in range(args.train) if s % world == rank]
    ids = mine + (list(range(args.train, args.train + args.test)) if rank == 0 else [])
    samples = {s: Sample(s, coarse, fine) for s in ids}
    targets = {}
    for s, smp in samples.items():
        _, out = run_forward(smp, fine, smp.cos_f)
        targets[s] = (pk_of(out.disp, coarse), density(out.disp, coarse))
    t_data = time.time() - t0
    model = LearnedGreen("cuda", seed=0)  # identical initial parameters on every rank
    history = []
    for it in range(args.iters):
        i = mine[it % len(mine)]
        smp = samples[i]
        run, out = run_forward(smp, coarse, smp.cos_c, model)
        fin = Particles(coarse, Particles.gen_grid(coarse, device=out.disp.device).pmid, out.disp, out.vel, out.acc)
        loss, g = _ps.pk_loss(fin, coarse, targets[i][0][1], kmax=args.kmax)
        model.zero_grad()
        z = torch.zeros_like(g)
        run.adjoint(fin, Particles(coarse, fin.pmid, g, z, z.clone()))
        replicas.average_gradient(model.grad, world)
        model.adam_step(lr=args.lr * (0.5 if it > 0.6 * args.iters else 1.0), clip=10.0)
        history.append(float(loss))
    t_train = time.time() - t0 - t_data
    if rank != 0:
        replicas.teardown(world)
        return None

    def errs(disp, target):
        k, pk, n = pk_of(disp, coarse)
        sel = k <= args.kmax
        ratio = pk[sel] / target[0][1][sel]
        ka, r, _, _, _, _ = _ps.delta_to_cross_correlation(density(disp, coarse), target[1], coarse)
        return float(np.max(np.abs(ratio - 1))), float(np.min(r[ka <= args.kmax]))

    evals = []
    test_ids = range(args.train, args.train + args.test)
    for smp, tgt in zip((samples[s] for s in test_ids), (targets[s] for s in test_ids)):
        _, plain = run_forward(smp, coarse, smp.cos_c)
        _, learn = run_forward(smp, coarse, smp.cos_c, model)
        ep, rp = errs(plain.disp, tgt)
        el, rl = errs(learn.disp, tgt)
        evals.append({"seed": smp.seed, "Omega_m": smp.om, "sigma8": smp.s8, "plain_max_pk_err": ep,
                      "learned_max_pk_err": el, "plain_min_r": rp, "learned_min_r": rl})
    smp = samples[args.train]
    t_learn = gpu_time(lambda: run_forward(smp, coarse, smp.cos_c, model))
    t_fine = gpu_time(lambda: run_forward(smp, fine, smp.cos_f))
    g_learn, g_fine = graphed_runs(smp, coarse, fine, model)
    tg_learn = gpu_time(g_learn, reps=10)
    tg_fine = gpu_time(g_fine, reps=5)
    res = {
        "config": {"particles": NP**3, "box": BOX, "coarse_mesh": coarse.mesh_shape[0], "fine_mesh": fine.mesh_shape[0],
                   "kdk_steps": args.nsteps, "train_seeds": args.train, "test_seeds": args.test,
                   "iters": args.iters, "kmax": args.kmax, "ranks": world},
        "train_loss_first": history[:5], "train_loss_last": history[-5:],
        "test": evals,
        "test_mean_max_pk_err": {"plain": float(np.mean([e["plain_max_pk_err"] for e in evals])),
                                 "learned": float(np.mean([e["learned_max_pk_err"] for e in evals]))},
        "time_ms": {"learned_128": t_learn, "plain_384": t_fine, "speedup": t_fine / t_learn,
                    "graphed_learned_128": tg_learn, "graphed_plain_384": tg_fine, "graphed_speedup": tg_fine / tg_learn},
        "wall_s": {"data": t_data, "train": t_train},
    }
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)
        np.save(args.out.replace(".json", "_params.npy"), model.parameters().cpu().numpy().astype(np.float32))
    print(json.dumps({k: res[k] for k in ("test_mean_max_pk_err", "time_ms", "wall_s", "train_loss_first",
                                          "train_loss_last")}))
    replicas.teardown(world)
    return res


if __name__ == "__main__":
    main()
