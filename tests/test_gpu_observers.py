"""Forward observers, saved maps, segmented runs and checkpoints on the GPU
(nbody/observers.py:18-126, nbody/solver.py:21-227, 645-679), following the
reference's tests/test_deep_observers_solver.py cases, plus windowed
projections of a random density against numpy sums of the oracle's deposit
(1e-6 of the map maximum) and a checkpointed run bitwise equal to an
uninterrupted one."""
import numpy as np
import pytest
import torch

from oracle import pm as opm
from tests.helpers import random_particles, rel_err

pytestmark = pytest.mark.gpu


def _short_conf(**changes):
    import pmpp_b200 as pb
    kw = dict(a_start=0.5, a_stop=0.51, a_custom=(0.5, 0.51), device="cuda")
    kw.update(changes)
    return pb, pb.Configuration(1.0, (2, 2, 2), 1, **kw)


def test_density_projection_observer_uniform_lattice():
    pb, conf = _short_conf()
    ptcl = pb.Particles.gen_grid(conf, vel=True)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    for axis in range(3):
        raw = pb.density_projection_observer(axis)(0.5, ptcl, cos, conf)
        nrm = pb.density_projection_observer(axis, normalize=True)(0.5, ptcl, cos, conf)
        assert tuple(raw.shape) == tuple(s for i, s in enumerate(conf.mesh_shape) if i != axis)
        np.testing.assert_allclose(raw.cpu().numpy(), 2.0, atol=2e-6)
        np.testing.assert_allclose(nrm.cpu().numpy(), 1.0, atol=2e-6)
        np.testing.assert_allclose(float(raw.sum()), conf.mesh_size, atol=2e-6)


def test_nbody_observe_start_end_and_final_state():
    pb, conf = _short_conf()
    ptcl = pb.Particles.gen_grid(conf, vel=True)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))

    def observer(a, p, _cos, _conf):
        return {"a": a, "mean_disp": p.disp.double().mean(0), "mass": float(len(p))}

    final, obs = pb.nbody_observe(ptcl, cos, conf, observer, include_start=True, return_final=True)
    direct = pb.nbody(ptcl, cos, conf)
    np.testing.assert_allclose(obs["a"].numpy(), [0.5, 0.51], rtol=1e-7)
    np.testing.assert_allclose(obs["mass"].numpy(), conf.ptcl_num)
    np.testing.assert_allclose(obs["mean_disp"].cpu().numpy(), 0, atol=2e-6)
    for x, y in ((final.disp, direct.disp), (final.vel, direct.vel), (final.acc, direct.acc)):
        np.testing.assert_allclose(x.cpu().numpy(), y.cpu().numpy(), rtol=2e-6, atol=2e-6)
    rev = pb.nbody_observe(ptcl, cos, conf, observer, reverse=True)
    np.testing.assert_allclose(rev["a"].numpy(), [0.5], rtol=1e-7)


def test_nbody_collect_state_and_final_particles():
    pb, conf = _short_conf()
    ptcl = pb.Particles.gen_grid(conf, vel=True)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))

    def collector(state, a_prev, a_next, p, _cos, _conf):
        return state + torch.tensor([a_prev, a_next, float((p.disp.double()**2).sum()), float(len(p))],
                                    dtype=torch.float64)

    init = torch.zeros(4, dtype=torch.float64)
    final, state = pb.nbody_collect(ptcl, cos, conf, collector, init, return_final=True)
    only = pb.nbody_collect(ptcl, cos, conf, collector, init)
    np.testing.assert_allclose(state.numpy(), [0.5, 0.51, 0.0, conf.ptcl_num], atol=2e-6)
    np.testing.assert_allclose(only.numpy(), state.numpy(), atol=2e-6)
    assert isinstance(final, pb.Particles) and final.acc is not None


def test_nbody_kappa_saved_maps():
    pb, conf = _short_conf(to_save_a=[0.51], slice_to_save=[0, 2], max_slice_width=2)
    ptcl = pb.Particles.gen_grid(conf, vel=True)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    maps = pb.nbody_kappa(ptcl, cos, conf)
    assert tuple(maps.shape) == (1, 3, 2, 2)
    np.testing.assert_allclose(maps.cpu().numpy(), 2.0, atol=3e-6)
    for axis in range(3):
        np.testing.assert_allclose(float(maps[0, axis].sum()), conf.mesh_size, atol=3e-6)
    pb2, c2 = _short_conf(to_save_a=None)
    assert isinstance(pb.nbody_kappa(pb.Particles.gen_grid(c2, vel=True), pb.boltzmann(pb.SimpleLCDM(c2)), c2),
                      pb.Particles)


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("start,stop,width", [(0, None, None), (5, 12, None), (-3, 4, None), (10, 40, 9),
                                              (7, 7, None), (30, 38, 100)])
def test_windowed_projection_matches_numpy(axis, start, stop, width):
    import pmpp_b200 as pb
    from pmpp_b200.observers import project
    shape = (32, 24, 40)
    co = opm.Conf(2.0, (16, 12, 20), mesh_shape=2)
    conf = pb.Configuration(2.0, (16, 12, 20), 2, device="cuda")
    pmid, disp = random_particles(co, 3, 2.0)
    ptcl = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    dens = pb.scatter(ptcl, conf)
    n = shape[axis]
    stop_ = n if stop is None else stop
    got = project(dens, axis, start, stop_, width).cpu().numpy()
    count = max(0, min(stop_ - start, width if width is not None else stop_ - start))
    idx = (start + np.arange(count)) % n
    d = dens.cpu().numpy().astype(np.float64)
    ref = np.take(d, idx, axis=axis).sum(axis=axis) if count else np.zeros(got.shape)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= 1e-6 * max(np.abs(ref).max(), 1.0)
    # against the oracle's float64 deposit too
    if stop is None:
        assert rel_err(got, opm.scatter(pmid, disp, co).sum(axis=axis)) < 1e-6


def test_checkpointed_segments_equal_one_run(tmp_path):
    """A run stopped at a = 0.4, saved, loaded and resumed equals the
    uninterrupted run bitwise; nbody_scheduled chains the two segments."""
    import pmpp_b200 as pb
    a1, a2 = np.linspace(0.1, 0.4, 4), np.linspace(0.4, 1.0, 5)
    mk = lambda a: pb.Configuration(4.0, (16, 16, 16), 2, a_start=float(a[0]), a_stop=float(a[-1]), a_custom=a,
                                    device="cuda")
    c1, c2 = mk(a1), mk(a2)
    co = opm.Conf(4.0, (16, 16, 16), mesh_shape=2)
    pmid, disp = random_particles(co, 8, 1.0)
    vel = np.random.default_rng(9).normal(0, 0.3, disp.shape).astype(np.float32)
    p0 = pb.Particles(c1, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(), torch.from_numpy(vel).cuda())
    cos = pb.boltzmann(pb.SimpleLCDM(c1))
    mid = pb.nbody(p0, cos, c1)
    path = tmp_path / "state.npz"
    pb.save_state(path, mid, float(a1[-1]), c1)
    loaded, a = pb.load_state(path, c2)
    assert a == pytest.approx(0.4)
    for x, y in ((loaded.disp, mid.disp), (loaded.vel, mid.vel), (loaded.acc, mid.acc), (loaded.pmid, mid.pmid)):
        assert torch.equal(x, y)
    resumed = pb.nbody(loaded, cos, c2)
    chained = pb.nbody_scheduled(p0, cos, [c1, c2])
    for x, y in ((resumed.disp, chained.disp), (resumed.vel, chained.vel), (resumed.acc, chained.acc)):
        assert torch.equal(x, y)
