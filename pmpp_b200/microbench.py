"""PM stage microbenchmark: 256^3 particles on a 512^3 mesh, unit masses.

Two position sets:

* U -- uniform random positions in the box (numpy PCG64, seed 1);
* K -- the final positions of the 64^3 / 128^3-mesh, 256 Mpc/h, sigma8 = 0.8
  run (2LPT at a = 0.1, 10 KDK steps to a = 1, noise seed 0) tiled 4 x 4 x 4
  onto the 256^3 lattice (clustered, same particle spacing).

Timed per stage with CUDA events on the launching stream (mean over
``reps`` launches after warm-up): row sort, density scatter, R2C, Green x
gradient, 3 x C2R, 3-channel gather, and the adjoints -- scatter VJP (position
term against an N(0,1) mesh cotangent), gather VJP (position term + 3-channel
scatter against N(0,1) particle cotangents, seed 2, the position term also
writing the cotangents in sorted order for the scatter), and the spectral adjoint
(3 x R2C, Green adjoint, C2R).  Every stage reports algorithmic bytes per
launch (pmpp_b200.roofline, with the measured count of touched cells) and
the fraction of the measured HBM copy bandwidth.

    python -m pmpp_b200.microbench --ptcl 256 --mesh 2 --reps 10
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np
import torch

from . import lpt as _lpt
from . import modes as _modes
from ._lib import call, lib
from .cic import SortedParticles
from .configuration import Configuration
from .cosmology import Cosmology
from .nbody import nbody
from .particles import Particles
from .roofline import algorithmic_bytes
from .runtime import stream_handle, workspace


def uniform_positions(conf, seed=1):
    """Set U: disp such that pmid * cell + disp is uniform in the box."""
    grid = Particles.gen_grid(conf)
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = rng.uniform(0.0, conf.box_size[0], size=(conf.ptcl_num, 3)).astype(np.float64)
    base = grid.pmid.cpu().numpy().astype(np.float64) * conf.cell_size
    disp = torch.from_numpy((pos - base).astype(np.float32)).to(grid.disp.device)
    return Particles(conf, grid.pmid, disp)


def clustered_positions(conf, seed=0):
    """Set K: the 64^3 run's final displacements tiled onto conf's lattice."""
    n1 = conf.ptcl_grid_shape[0]
    mesh = conf.mesh_shape[0] // n1
    a = np.linspace(0.1, 1.0, 11)
    small = Configuration(conf.ptcl_spacing, (64, 64, 64), mesh, a_start=0.1, a_custom=a, device=conf.device)
    cos = Cosmology.from_sigma8(small, 0.8, n_s=0.96, Omega_m=0.3, Omega_b=0.05, h=0.7)
    lin = _modes.linear_modes(_modes.white_noise_nested(seed, small), cos, small)
    out = nbody(_lpt.lpt(lin, cos, small), cos, small)
    rep = n1 // 64
    d = out.disp.reshape(64, 64, 64, 3).repeat(rep, rep, rep, 1).reshape(-1, 3).contiguous()
    grid = Particles.gen_grid(conf)
    return Particles(conf, grid.pmid, d)


def _staged(fn):
    call("pmb_set_gather_staging", 1)
    try:
        fn()
    finally:
        call("pmb_set_gather_staging", 0)


def _time(fn, reps):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_set(ptcl, conf, reps, peak):
    dev = ptcl.disp.device
    L = lib()
    s = stream_handle(dev)
    n = conf.ptcl_num
    nx, ny, nz = conf.mesh_shape
    M = conf.mesh_size
    Mc = nx * ny * (nz // 2 + 1)
    tables = conf.spectral_tables("mesh", dev, 0)
    rng = torch.Generator(device="cpu").manual_seed(2)
    acc_cot = torch.randn((n, 3), generator=rng).to(dev)
    mesh_cot = torch.randn((1, nx, ny, nz), generator=rng).to(dev)
    rho = torch.empty((1, nx, ny, nz), dtype=torch.float32, device=dev)
    F = torch.empty((3, nx, ny, nz), dtype=torch.float32, device=dev)
    F3 = torch.empty_like(F)
    spec1 = torch.empty((nx, ny, nz // 2 + 1), dtype=torch.complex64, device=dev)
    spec3 = torch.empty((3, nx, ny, nz // 2 + 1), dtype=torch.complex64, device=dev)
    acc = torch.empty((n, 3), dtype=torch.float32, device=dev)
    dcot = torch.empty((n, 3), dtype=torch.float32, device=dev)
    cot_sorted = torch.empty((n, 3), dtype=torch.float32, device=dev)
    fw = max(L.pmb_fft_work_bytes(nx, ny, nz, 3), L.pmb_fft_work_bytes(nx, ny, nz, 1))
    work = workspace(fw, dev, "micro_fft")
    sp = SortedParticles(ptcl.pmid, ptcl.disp, conf)
    vc = float(M / n)
    inv_m = float(1.0 / M)

    stages = {
        "sort": lambda: SortedParticles(ptcl.pmid, ptcl.disp, conf),
        "scatter": lambda: sp.scatter(out=rho, mode=1, src_mul=0.45),
        "fft_r2c": lambda: call("pmb_rfft3", nx, ny, nz, 1, rho.data_ptr(), spec1.data_ptr(), work.data_ptr(), s),
        "green_gradient": lambda: call("pmb_green_gradient", spec1.data_ptr(), spec3.data_ptr(), nx, ny, nz,
                                       tables.data_ptr(), int(conf.has_particle_nyquist_masks), 0, None, None, 0,
                                       inv_m, s),
        "fft_c2r_x3": lambda: call("pmb_irfft3", nx, ny, nz, 3, spec3.data_ptr(), F.data_ptr(), work.data_ptr(), s),
        "gather": lambda: sp.gather(F, out=acc),
        "scatter_adjoint": lambda: sp.interp_grad(mesh_cot, u_const=vc, disp_cot=dcot, accumulate=True),
        "gather_adjoint": lambda: sp.interp_grad(F, u=acc_cot, disp_cot=dcot, accumulate=True, u_sorted=cot_sorted),
        "scatter3": lambda: sp.scatter(val=cot_sorted, channels=3, out=F3, val_sorted=True),
        "fft_r2c_x3": lambda: call("pmb_rfft3", nx, ny, nz, 3, F3.data_ptr(), spec3.data_ptr(), work.data_ptr(), s),
        "green_gradient_adjoint": lambda: call("pmb_green_gradient_adjoint", spec3.data_ptr(), spec1.data_ptr(), nx,
                                               ny, nz, tables.data_ptr(), int(conf.has_particle_nyquist_masks), 0,
                                               None, None, 0, 0.45 * inv_m, s),
        "fft_c2r": lambda: call("pmb_irfft3", nx, ny, nz, 1, spec1.data_ptr(), rho.data_ptr(), work.data_ptr(), s),
        # the same gathers with mesh rows staged in shared memory (opt-in mode)
        "gather@staged": lambda: _staged(lambda: sp.gather(F, out=acc)),
        "gather_adjoint@staged": lambda: _staged(
            lambda: sp.interp_grad(F, u=acc_cot, disp_cot=dcot, accumulate=True, u_sorted=cot_sorted)),
    }
    # distinct touched cells: nonzero cells of the unit-mass density
    T = int((sp.scatter() != 0).sum())
    out = {"touched_cells": T}
    for name, fn in stages.items():
        ms = _time(fn, reps)
        alg = algorithmic_bytes(name.split("@")[0], n, M, Mc=Mc, R=nx * ny, T=T)
        gbs = alg / (ms * 1e-3) / 1e9
        out[name] = {"ms": round(ms, 4), "algorithmic_bytes": alg, "GB/s": round(gbs, 1), "frac_hbm": round(gbs / peak, 4)}
    return out


def pmfft_stages(conf, reps, peak, only=None):
    """Each pass of the hand-written FFT chain (pmfft.cu) on random inputs."""
    dev = conf.device
    L = lib()
    s = stream_handle(dev)
    nx, ny, nz = conf.mesh_shape
    if not L.pmb_pmfft_supported(nx, ny, nz):
        return {}
    M = conf.mesh_size
    Mc = nx * ny * (nz // 2 + 1)
    C = L.pmb_pmfft_channel_elems(nx, ny, nz)
    tables = conf.spectral_tables("mesh", dev, 0).data_ptr()
    masks = int(conf.has_particle_nyquist_masks)
    g = torch.Generator(device="cpu").manual_seed(5)
    real3 = torch.randn((3, nx, ny, nz), generator=g).to(dev)
    real3b = torch.empty_like(real3)
    pa = torch.zeros(3 * C, dtype=torch.complex64, device=dev)
    pb_ = torch.zeros(3 * C, dtype=torch.complex64, device=dev)
    a, b = pa.data_ptr(), pb_.data_ptr()
    C8 = 8 * C
    inv_m = float(1.0 / M)
    col = lambda mode, ch_off, i, o, post=1.0: call("pmb_pmfft_col", nx, ny, nz, mode, 1, ch_off, i, o, tables, masks,
                                                    None, None, 0, post, s)
    call("pmb_pmfft_z", nx, ny, nz, 0, 3, real3.data_ptr(), a, s)
    stages = {
        "fft_z_r2c": lambda: call("pmb_pmfft_z", nx, ny, nz, 0, 1, real3.data_ptr(), b, s),
        "fft_z_r2c3": lambda: call("pmb_pmfft_z", nx, ny, nz, 0, 3, real3.data_ptr(), b, s),
        "fft_y": lambda: col(0, 0, a, b),
        "fft_y_yz": lambda: col(3, 1, a, b),
        "fft_x_green": lambda: col(6, 0, a, b, inv_m),
        "fft_x_green_adj": lambda: col(7, 0, a, b, inv_m),
        "fft_x_adj": lambda: col(8, 0, a, b, inv_m),
        "fft_x_inv": lambda: col(5, 0, a, b),
        "fft_y_inv": lambda: col(1, 0, a, b),
        "fft_y_inv_yz": lambda: col(2, 0, a, b),
        "fft_z_c2r": lambda: call("pmb_pmfft_z", nx, ny, nz, 1, 1, a, real3b.data_ptr(), s),
        "fft_z_c2r3": lambda: call("pmb_pmfft_z", nx, ny, nz, 1, 3, a, real3b.data_ptr(), s),
    }
    # the same passes as stages of a force chain pruned to the particle-Nyquist
    # box (what pmb_force runs when the mesh is finer than the particle grid)
    live = None
    if masks:
        my, mz = conf.particle_nyquist_masks()[1:]
        live = (float((my != 0).sum()) / len(my), float((mz != 0).sum()) / len(mz))
        col2 = lambda mode, ch_off, i, o, post=1.0: call("pmb_pmfft_col2", nx, ny, nz, mode, 1, ch_off, i, o, tables,
                                                         masks, None, None, 0, post, 1, s)
        stages.update({
            "fft_y_pruned": lambda: col2(0, 0, a, b),
            "fft_y_yz_pruned": lambda: col2(3, 1, a, b),
            "fft_x_green_pruned": lambda: col2(6, 0, a, b, inv_m),
            "fft_x_green_adj_pruned": lambda: col2(7, 0, a, b, inv_m),
            "fft_y_inv_pruned": lambda: col2(1, 0, a, b),
            "fft_y_inv_yz_pruned": lambda: col2(2, 0, a, b),
            "fft_z_c2r_pruned": lambda: call("pmb_pmfft_z2", nx, ny, nz, 1, 1, a, real3b.data_ptr(), tables, masks, 1,
                                             s),
            "fft_z_c2r3_pruned": lambda: call("pmb_pmfft_z2", nx, ny, nz, 1, 3, a, real3b.data_ptr(), tables, masks,
                                              1, s),
        })
    out = {}
    for name, fn in stages.items():
        if only and name.replace("_pruned", "") not in only:
            continue
        ms = _time(fn, reps)
        base = name.replace("_pruned", "")
        alg = algorithmic_bytes(base, 0, M, Mc=Mc, R=nx * ny, live=live if name.endswith("_pruned") else None)
        gbs = alg / (ms * 1e-3) / 1e9
        out[name] = {"ms": round(ms, 4), "algorithmic_bytes": alg, "GB/s": round(gbs, 1), "frac_hbm": round(gbs / peak, 4)}
    return out


def load_peak():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ptcl", type=int, default=256)
    ap.add_argument("--mesh", type=int, default=2)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--sets", default="U,K")
    ap.add_argument("--pmfft-shape", type=int, nargs=3, default=None,
                    help="time only the FFT pass chain on this mesh shape")
    ap.add_argument("--stages", default=None, help="comma-separated pass names (with --pmfft-shape)")
    ap.add_argument("--col-ctas", type=int, default=None, help="resident CTAs per SM of the column passes")
    args = ap.parse_args(argv)
    if args.col_ctas is not None:
        call("pmb_pmfft_set_col_ctas", args.col_ctas)
    if args.pmfft_shape is not None:
        nx, ny, nz = args.pmfft_shape
        conf = Configuration(4.0, (nx // 2, ny // 2, nz // 2), 2, a_start=0.1, device="cuda")
        peak, kind = load_peak()
        only = args.stages.split(",") if args.stages else None
        res = {"config": {"mesh_shape": [nx, ny, nz], "reps": args.reps}, "peak_gbs": peak, "peak_kind": kind,
               "pmfft": pmfft_stages(conf, args.reps, peak, only)}
        print(json.dumps(res))
        return res
    if args.ptcl % 64:
        raise ValueError("--ptcl must be a multiple of 64 (set K tiles the 64^3 run)")
    conf = Configuration(4.0, (args.ptcl, ) * 3, args.mesh, a_start=0.1, device="cuda")
    peak, kind = load_peak()
    res = {"config": {"particles": conf.ptcl_num, "mesh": conf.mesh_size, "box": conf.box_size[0], "reps": args.reps},
           "peak_gbs": peak, "peak_kind": kind}
    for name in args.sets.split(","):
        ptcl = uniform_positions(conf) if name == "U" else clustered_positions(conf)
        res[name] = run_set(ptcl, conf, args.reps, peak)
        del ptcl
        torch.cuda.empty_cache()
    res["pmfft"] = pmfft_stages(conf, args.reps, peak)
    torch.cuda.empty_cache()
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()
