"""The memory-lean forward path (nbody/gravity.py:643-658 gravity_streamed,
nbody/solver.py:559-602 nbody_low_memory): one force component at a time
through one real mesh.

Bars: the streamed force within 1e-6 of the fused force's cuFFT route (the same
arithmetic per component) and 1e-5 of the oracle; a 3-step forward run within
1e-4 of the oracle's (the bar of the fused run); the streamed force's device
memory peak below 70% of the fused force's; reverse runs and corrections
rejected as in the reference."""
import numpy as np
import pytest
import torch

from oracle import cosmology as ocos
from oracle import pm as opm
from tests.helpers import random_particles, rel_err

pytestmark = pytest.mark.gpu


def _confs(shape=(32, 32, 32), mesh=2, a_custom=None):
    import pmpp_b200 as pb
    co = opm.Conf(4.0, shape, mesh_shape=mesh, a_start=0.1, a_custom=a_custom)
    c = pb.Configuration(4.0, shape, mesh, a_start=0.1, a_custom=a_custom, device="cuda")
    return pb, co, c


def test_streamed_force_matches_fused_and_oracle():
    from pmpp_b200 import _lib
    pb, co, conf = _confs()
    pmid, disp = random_particles(co, seed=3, spread=2.0)
    p = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda())
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    acc_s = pb.gravity_streamed(1.0, p, cos, conf).cpu().numpy()
    _lib.set_pmfft(False)
    try:
        acc_f = pb.gravity(1.0, p, cos, conf).cpu().numpy()
    finally:
        _lib.set_pmfft(True)
    assert rel_err(acc_s, acc_f) < 1e-6
    assert rel_err(acc_s, opm.gravity(pmid, disp, co, 0.3)) < 1e-5
    with pytest.raises(ValueError):
        pb.gravity_streamed(1.0, p, cos, conf, correction=object())


def test_low_memory_run_matches_oracle():
    a = np.linspace(0.1, 1.0, 4)
    pb, co, conf = _confs(shape=(16, 16, 16), a_custom=a)
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    oc = opm.boltzmann(ocos.Cosmo(), co)
    pmid, disp = random_particles(co, seed=21, spread=1.0)
    vel = np.random.default_rng(22).normal(0, 0.5, size=disp.shape).astype(np.float32)
    p = pb.Particles(conf, torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda(), torch.from_numpy(vel).cuda())
    out = pb.nbody_low_memory(p, cos, conf)
    rd, rv, ra = opm.nbody(pmid, disp, vel, co, oc)
    assert rel_err(out.disp.cpu().numpy(), rd) < 1e-4
    assert rel_err(out.vel.cpu().numpy(), rv) < 1e-4
    assert rel_err(out.acc.cpu().numpy(), ra) < 1e-4
    with pytest.raises(ValueError):
        pb.nbody_low_memory(p, cos, conf, reverse=True)


def test_streamed_force_memory_peak():
    from pmpp_b200 import runtime
    from pmpp_b200.gravity import force, force_streamed
    pb, co, conf = _confs(shape=(128, 128, 128), mesh=2)
    p = pb.Particles.gen_grid(conf)
    disp = p.disp + 0.1
    om = 0.3
    peaks = {}
    for name, fn in (("fused", lambda: force(p.pmid, disp.clone(), conf, om)),
                     ("streamed", lambda: force_streamed(p.pmid, disp.clone(), conf, om))):
        runtime.release_workspaces()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        base = torch.cuda.memory_allocated()
        torch.cuda.reset_peak_memory_stats()
        out = fn()
        torch.cuda.synchronize()
        peaks[name] = torch.cuda.max_memory_allocated() - base
        del out
    runtime.release_workspaces()
    print(f"force memory peak at 128^3 / 256^3: fused {peaks['fused'] / 2**20:.0f} MiB, "
          f"streamed {peaks['streamed'] / 2**20:.0f} MiB")
    assert peaks["streamed"] < 0.7 * peaks["fused"]
