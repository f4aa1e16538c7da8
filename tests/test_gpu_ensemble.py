"""Ensembles of uneven simulations against single-simulation runs.

With one member per mesh shape every batched FFT is a batch-1 plan, so an
ensemble run must equal NBodyRun.forward of every member bit for bit; with
several members per shape the batched cuFFT plans may round differently, so
members agree within float32 round-off carried over a few steps.  Members on
power-of-two meshes (the hand-written FFT pass chain) are bitwise in every case.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _members(specs, nsteps=4):
    import pmpp_b200 as pb
    from pmpp_b200 import lpt as pl, modes as pm
    a = np.geomspace(0.1, 1.0, nsteps + 1)
    confs, coss, ics = [], [], []
    for k, (n, mesh, box, om) in enumerate(specs):
        conf = pb.Configuration(box / n, (n, ) * 3, mesh, a_start=0.1, a_custom=a, device="cuda")
        cos = pb.boltzmann(pb.SimpleLCDM(conf, Omega_m=om))
        ic = pl.lpt(pm.linear_modes(pm.white_noise_nested(k, conf), cos, conf), cos, conf)
        confs.append(conf)
        coss.append(cos)
        ics.append(ic)
    return confs, coss, ics


@pytest.mark.parametrize("graph", [False, True])
def test_one_member_per_shape_is_bitwise_single_runs(graph):
    import pmpp_b200 as pb
    from pmpp_b200.ensemble import Ensemble
    confs, coss, ics = _members([(16, 2, 64.0, 0.3), (24, 2, 100.0, 0.27), (8, 2, 50.0, 0.33), (12, 1, 80.0, 0.31)])
    ens = Ensemble(confs, coss)
    outs = ens.forward(ics, graph=graph)
    for conf, cos, ic, out in zip(confs, coss, ics, outs):
        ref = pb.NBodyRun(conf, cos).forward(ic)
        for name in ("disp", "vel", "acc"):
            assert torch.equal(getattr(out, name), getattr(ref, name)), name


def test_batched_shapes_autotune_and_replay():
    import pmpp_b200 as pb
    from pmpp_b200.ensemble import Ensemble
    specs = [(16, 2, 64.0, 0.3), (16, 2, 90.0, 0.26), (8, 2, 40.0, 0.34), (16, 2, 70.0, 0.29), (8, 2, 60.0, 0.3)]
    confs, coss, ics = _members(specs)
    ens = Ensemble(confs, coss)
    first = ens.forward(ics, graph=False)
    tuning = ens.autotune(reps=2)
    assert set(tuning["tiles"]) == {str((32, 32, 32)), str((16, 16, 16))}
    again = ens.forward(ics, graph=True)
    replay = ens.forward(ics, graph=True)
    for a, b, c in zip(first, again, replay):
        # tile and launch shapes change no arithmetic; graph replays are deterministic
        assert torch.equal(a.disp, b.disp) and torch.equal(b.disp, c.disp)
    for conf, cos, ic, out in zip(confs, coss, ics, first):
        ref = pb.NBodyRun(conf, cos).forward(ic)
        scale = float(ref.disp.abs().max())
        assert float((out.disp - ref.disp).abs().max()) < 1e-4 * scale


@pytest.mark.parametrize("graph", [False, True])
def test_ensemble_initial_conditions_bitwise(graph):
    """Batched 2LPT initial conditions equal the per-member sequence bit for bit."""
    import pmpp_b200 as pb
    from pmpp_b200 import lpt as pl, modes as pm
    from pmpp_b200.ensemble import Ensemble
    confs, coss, _ = _members([(16, 2, 64.0, 0.3), (8, 2, 50.0, 0.33), (16, 1, 90.0, 0.27)])
    seeds = [5, 9, 13]
    ens = Ensemble(confs, coss)
    for _ in range(2):  # the second call replays the captured sequence
        ens.initial_conditions(seeds, graph=graph)
    for i, (conf, cos, seed) in enumerate(zip(confs, coss, seeds)):
        ref = pl.lpt(pm.linear_modes(pm.white_noise_nested(seed, conf), cos, conf), cos, conf)
        got = ens.particles(i)
        assert torch.equal(got.disp, ref.disp) and torch.equal(got.vel, ref.vel)
        assert torch.equal(got.pmid, ref.pmid)
    outs = ens.run(seeds, graph=graph)
    ref = pb.NBodyRun(confs[0], coss[0]).forward(
        pl.lpt(pm.linear_modes(pm.white_noise_nested(seeds[0], confs[0]), coss[0], confs[0]), coss[0], confs[0]))
    assert torch.equal(outs[0].disp, ref.disp)


@pytest.mark.parametrize("graph", [False, True])
def test_fft_chain_members_are_bitwise_single_runs(graph):
    """Members on power-of-two meshes run the hand-written FFT pass chain one
    after another (the same kernels as a single run), so even several members
    of one mesh shape equal their single runs bit for bit."""
    import pmpp_b200 as pb
    from pmpp_b200 import _lib
    from pmpp_b200.ensemble import Ensemble
    confs, coss, ics = _members([(32, 4, 128.0, 0.3), (64, 2, 256.0, 0.28), (32, 4, 160.0, 0.31),
                                 (16, 2, 64.0, 0.3)], nsteps=3)
    assert _lib.pmfft_active(*confs[0].mesh_shape) and not _lib.pmfft_active(*confs[3].mesh_shape)
    ens = Ensemble(confs, coss)
    outs = ens.forward(ics, graph=graph)
    for conf, cos, ic, out in zip(confs, coss, ics, outs):
        ref = pb.NBodyRun(conf, cos).forward(ic)
        for name in ("disp", "vel", "acc"):
            assert torch.equal(getattr(out, name), getattr(ref, name)), name
    assert _lib.pmfft_timeouts() == 0
