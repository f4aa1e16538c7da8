"""Benchmark: forward + adjoint PM N-body throughput on B200.

Workload (default): the full differentiable run -- 512^3 particles, 1024^3
force mesh, 1024 Mpc/h box, SimpleLCDM: nested white noise (seed 1) -> linear
modes -> 2LPT at a = 0.1 -> 32 log-spaced kick-drift-kick steps to a = 1 ->
CIC density -> P(k) -> mean squared log ratio against a fixed target spectrum,
then the hand-written reverse pass back to the white-noise modes, Omega_m
and A_s.  One bench step = one such forward + adjoint run; the metric counts
particles x 32 macro steps per second.  Inputs are larger than L2.

``--impl reference`` times the CPU oracle (NumPy restatement of PM++, the
reference's own JAX stack is not installable here) on the host cores, on a
bounded sample of the same workload: one forward + adjoint KDK step of a
periodic sub-volume at the workload's resolution per bench step.  With
``--gpus N > 1`` outside torchrun the command re-launches itself as N local
ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

METRIC = "particle-steps/s at 512³/1024³ fwd+adj; learned-128³ vs plain-384³ time at 1% P(k)"
UNIT = "particle-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--ptcl", type=int, default=512)
    p.add_argument("--mesh", type=int, default=2)
    p.add_argument("--nsteps", type=int, default=32)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-learned", action="store_true")
    p.add_argument("--cpu-ptcl", type=int, default=64)
    return p.parse_args()


# --------------------------------------------------------------------------
# clocks sampled during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace('.', '', 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace('.', '', 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per particle of one launch, from an ncu
# --set full capture of the same kernels at 256^3 particles / 512^3 mesh (mesh cells = 8 particles);
# traffic scales with particles at a fixed cells-per-particle ratio.
MEASURED_TRAFFIC_PER_PARTICLE = {
    "gather": (1.949012 + 0.193225) * 1e9 / 256**3,       # gather_kernel_x2<3>, no velocities
    "gather_kick": (2.150708 + 0.389332) * 1e9 / 256**3,  # gather_kernel_x2<3> with the folded kicks
    "scatter3": (0.472 + 1.556) * 1e9 / 256**3,
    "scatter": (0.270 + 0.484) * 1e9 / 256**3,
    "scatter_adjoint": (1.075 + 0.189) * 1e9 / 256**3,
    "fft_z_c2r3": (1.660984 + 1.565085) * 1e9 / 256**3,  # z_c2r_kernel, 3 channels, pruned chain
}


# Stages whose launches run in two variants, the second tagged by the stage timer (a gather that also
# applies the folded kicks reads and writes the velocities): the dominant stage's algorithmic bytes and
# traffic are the launch-weighted mean of its variants.
STAGE_VARIANTS = {"gather": ("gather_kick", "gather_kick_only")}


def stage_mix(stage, counts, N, M, conf, live):
    """(algorithmic bytes, measured traffic per particle or None, launch mix) of
    one launch of a stage, weighted over the launch variants the timer counted."""
    from pmpp_b200.roofline import algorithmic_bytes
    nx, ny, nz = conf.mesh_shape
    ab = lambda op: algorithmic_bytes(op, N, M, Mc=nx * ny * (nz // 2 + 1), R=nx * ny, live=live)
    nd = counts[stage]
    parts = {v: counts.get(v, 0) for v in STAGE_VARIANTS.get(stage, ()) if counts.get(v, 0)}
    parts[stage] = nd - sum(parts.values())
    alg = sum(n * ab(v) for v, n in parts.items()) / nd
    traffic = None
    if all(v in MEASURED_TRAFFIC_PER_PARTICLE for v, n in parts.items() if n):
        traffic = sum(n * MEASURED_TRAFFIC_PER_PARTICLE[v] for v, n in parts.items() if n) / nd
    return alg, traffic, (parts if len(parts) > 1 else None)


# CIC stage groups whose combined fraction of the HBM peak the line reports:
# the forward pair (deposit + force gather) and the adjoint CIC stages.
CIC_GROUPS = {"scatter+gather": ("scatter", "gather"),
              "adjoint": ("gather_adjoint", "scatter3", "scatter_adjoint")}


def cic_fractions(breakdown, counts, N, M, conf, live, peak):
    """Combined fraction of the HBM peak of each CIC group: the group's
    algorithmic bytes over the group's device time, per run."""
    out = {}
    for name, stages in CIC_GROUPS.items():
        if not all(s in breakdown for s in stages):
            continue
        byts = sum(stage_mix(s, counts, N, M, conf, live)[0] * breakdown[s]["launches"] for s in stages)
        ms = sum(breakdown[s]["ms_total"] for s in stages)
        out[name] = round(byts / (ms * 1e-3) / 1e9 / peak, 3)
    return out


def live_fractions(conf):
    """(fy, fz): live fractions of ky and kz (nz/2+1 values) of the pass chain
    pruned to the particle-Nyquist box, or None when the chain is not pruned."""
    from pmpp_b200._lib import pmfft_active
    if not conf.has_particle_nyquist_masks or not pmfft_active(*conf.mesh_shape):
        return None
    my, mz = conf.particle_nyquist_masks()[1:]
    return float((my != 0).sum()) / len(my), float((mz != 0).sum()) / len(mz)


def load_peaks():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# --------------------------------------------------------------------------
# CPU baseline: the oracle on a bounded sample
# --------------------------------------------------------------------------
def cpu_sample_rate(ptcl=64, mesh=2, nsteps=1, seed=0, full_ptcl=512):
    """One forward + adjoint KDK step of the oracle on a periodic sub-volume of the
    workload: ptcl^3 particles on a (mesh*ptcl)^3 mesh at the workload's particle
    spacing and cell size (1024 Mpc/h over 512 particles), the first of its 32 log
    steps, FFTs and CIC loops threaded over the host cores.  Particle-steps/s
    of PM depends on the size only through the FFTs' log factor, so the rate
    stands for the full run; the line says so.  Returns (rate, seconds, sample)."""
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from oracle import cosmology as ocos
    from oracle import pm as opm
    cores = os.cpu_count() or 1
    opm.set_fft_workers(cores)
    box = 1024.0 * ptcl / 512
    a = np.geomspace(0.1, 1.0, 33)[:nsteps + 1]
    co = opm.Conf(box / ptcl, (ptcl, ) * 3, mesh_shape=mesh, a_start=0.1, a_custom=a)
    oc = opm.boltzmann(ocos.Cosmo(), co)
    pmid, disp = opm.gen_grid(co)
    rng = np.random.default_rng(seed)
    disp = (disp + rng.normal(0, 0.3 * co.cell_size, size=disp.shape)).astype(np.float32)
    vel = np.zeros_like(disp)
    t0 = time.perf_counter()
    d, v, acc = opm.nbody(pmid, disp, vel, co, oc)
    cot = rng.normal(size=disp.shape).astype(np.float32)
    opm.nbody_adj(pmid, d, v, acc, cot, cot, np.zeros_like(cot), co, oc, om_grads=False)
    dt = time.perf_counter() - t0
    n = ptcl**3
    rate = n * nsteps / dt
    full = full_ptcl**3 * 32 / rate
    sample = (f"oracle (NumPy restatement, {cores} threads) forward + adjoint of {nsteps} KDK step(s) on a "
              f"{ptcl}^3-particle / {mesh * ptcl}^3-mesh periodic sub-volume ({box:.0f} Mpc/h) at the workload's "
              f"resolution ({1024.0 / 512:.0f} Mpc/h spacing), {dt:.2f} s; rate extrapolated to the "
              f"{full_ptcl}^3 / {mesh * full_ptcl}^3 run: {full:.0f} s per 32-step forward + adjoint run")
    return rate, dt, sample


def arm_config(args, world):
    """The workload both arms report under (the reference arm times a bounded sample of it)."""
    n1 = args.ptcl
    box = 1024.0 * n1 / 512
    return {"workload": f"{n1}^3 particles / {args.mesh * n1}^3 mesh, {box:.0f} Mpc/h: noise -> 2LPT(a=0.1) -> "
                        f"{args.nsteps} log KDK steps -> P(k) loss, forward + full reverse pass per step",
            "particles": n1**3, "mesh": (args.mesh * n1)**3,
            "kdk_steps": args.nsteps, "parallelism": f"replicas x{world}", "l2": "inputs larger than L2"}


def run_reference(args):
    """The reference arm: rank 0 times the oracle on host cores (the other ranks
    of a torchrun launch exit without work)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    rates = []
    for i in range(args.warmup + args.steps):
        r, dt, sample = cpu_sample_rate(args.cpu_ptcl, args.mesh, 1, seed=i, full_ptcl=args.ptcl)
        if i >= args.warmup:
            rates.append(r)
    v = float(np.mean(rates))
    cores = os.cpu_count() or 1
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * (args.cpu_ptcl**3) / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": arm_config(args, world),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def run_ours(args):
    import torch

    from pmpp_b200 import replicas
    rank, world, local = replicas.setup("nccl")
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    barrier = lambda w: replicas.barrier(w)
    max_over_ranks = replicas.max_over_ranks
    import pmpp_b200 as pb
    from pmpp_b200 import _lib
    from pmpp_b200.runtime import StageTimer

    n1 = args.ptcl
    box = 1024.0 * n1 / 512
    a = np.geomspace(0.1, 1.0, args.nsteps + 1)
    conf = pb.Configuration(box / n1, (n1, ) * 3, args.mesh, a_start=0.1, a_custom=a, device=dev)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    N = conf.ptcl_num
    M = conf.mesh_size
    from pmpp_b200 import modes as pmodes
    from pmpp_b200 import pipeline
    omega = pmodes.white_noise_nested(replicas.replica_seed(1, rank), conf)
    model = pipeline.ForwardModel(conf, cos)
    # fixed target spectrum: the first run's P(k) modulated by 10%
    with StageTimer():
        model.forward(omega)
        _, pk0, _ = pb.power_spectrum.particles_to_pk(model.final, conf)
    target = pk0 * (1.0 + 0.1 * np.sin(np.arange(len(pk0))))

    def step(om):
        model.forward(om)
        loss, g = model.loss(target)
        return loss, model.backward(g)

    # all device work runs through the staged entry points so a single set of
    # workspaces is allocated
    with StageTimer():
        for _ in range(args.warmup):
            step(omega)
    torch.cuda.synchronize()
    _lib.reset_launch_count()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        with StageTimer() as timer:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                res = step(omega)
            e1.record()
            torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches = _lib.launch_count()
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms, world)
    stages = timer.totals()
    counts = dict(timer.counts)
    value = world * N * args.nsteps / (ms * 1e-3)

    # end to end: white-noise modes in from pinned host memory, the modes
    # gradient and the scalar loss / parameter gradients out, every step
    h_om = omega.cpu().pin_memory()
    h_grad = torch.empty_like(h_om).pin_memory()
    barrier(world)
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    with StageTimer():
        e2.record()
        for _ in range(args.steps):
            om_d = h_om.to(dev, non_blocking=True)
            loss, grads = step(om_d)
            h_grad.copy_(grads["modes"], non_blocking=True)
        e3.record()
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3) / args.steps, world)
    h2d = int(h_om.numel() * 8 + len(target) * 8)
    d2h = int(h_grad.numel() * 8 + 3 * 8 + len(target) * 8)

    if rank != 0:
        replicas.teardown(world)
        return

    peak, peak_kind = load_peaks()
    # hand-written stages only (cuFFT's transforms are library kernels)
    ours = {k: v for k, v in stages.items() if k not in ("fft_r2c", "fft_c2r")}
    dom = max(ours, key=ours.get)
    per_launch_ms = ours[dom] / counts[dom]
    from pmpp_b200.roofline import algorithmic_bytes
    nx, ny, nz = conf.mesh_shape
    live = live_fractions(conf)
    alg, traffic_pp, mix = stage_mix(dom, counts, N, M, conf, live)
    achieved = alg / (per_launch_ms * 1e-3) / 1e9
    stages["other (kick/drift adjoints, LPT, P(k), host)"] = max(ms * args.steps - sum(stages.values()), 0.0)
    counts["other (kick/drift adjoints, LPT, P(k), host)"] = args.steps
    breakdown = {k: {"ms_total": round(v, 3), "launches": counts[k], "share": round(v / (ms * args.steps), 4)}
                 for k, v in sorted(stages.items(), key=lambda kv: -kv[1])}
    for k, b in breakdown.items():
        try:  # each stage's fraction of the HBM peak in its algorithmic bytes
            ab = stage_mix(k, counts, N, M, conf, live)[0]
        except KeyError:
            continue
        b["frac"] = round(ab / (b["ms_total"] / b["launches"] * 1e-3) / 1e9 / peak, 3)
    cic = cic_fractions(breakdown, counts, N, M, conf, live, peak)
    learned = None
    wpath = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pmpp_b200", "data", "learned_green_c3.npy")
    if world == 1 and not args.no_learned and os.path.exists(wpath):
        # second half of the metric: learned 128^3-mesh run vs plain 384^3-mesh run
        # (128^3 particles, 256 Mpc/h, 20 KDK steps), committed weights trained by
        # `python -m pmpp_b200.learned`, evaluated on held-out seeds 64..79
        from pmpp_b200 import learned as pl
        learned = pl.evaluate(wpath)
    cpu = None
    if not args.no_cpu_baseline:
        r, dt, sample = cpu_sample_rate(args.cpu_ptcl, args.mesh, 1, full_ptcl=args.ptcl)
        cpu = {"value": r, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port", "sample": sample}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": arm_config(args, world),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": (traffic_pp * N if traffic_pp is not None and M == 8 * N else None),
                     "traffic_source": "ncu captures at 256^3/512^3 (each launch variant) scaled by particles",
                     "algorithmic_bytes_per_launch": alg, "ms_per_launch": per_launch_ms, "launch_mix": mix},
        "breakdown": breakdown,
        "cic_roofline": cic,
        "cpu_baseline": cpu,
        "e2e": {"value": world * N * args.nsteps / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "learned": learned,
    }
    print(json.dumps(line), flush=True)
    replicas.teardown(world)


def self_launch(args):
    """With --gpus N > 1 outside torchrun, re-run this command as N local ranks
    (one process per GPU, rendezvous on 127.0.0.1) and return their exit code;
    None when this process is already a rank (or N == 1)."""
    if args.gpus <= 1 or "WORLD_SIZE" in os.environ:
        return None
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    rc = self_launch(args)
    if rc is not None:
        sys.exit(rc)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
