"""Golden fixtures (tests/golden/pm_small.npz, made by tests/golden/make_golden.py).

CPU: the oracle still reproduces the committed fixtures (regression guard).
GPU: every hot-path stage of libpmb200 against the committed numbers.
"""
import os

import numpy as np
import pytest
import torch

from oracle import cosmology as ocos
from oracle import pm as opm
from tests.golden.make_golden import A, conf as oconf
from tests.helpers import rel_err

G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pm_small.npz"))


def test_oracle_reproduces_fixtures():
    co = oconf()
    assert np.array_equal(opm.sort_by_cell(G["pmid"], G["disp"], co)[1], G["perm"])
    np.testing.assert_array_equal(opm.scatter(G["pmid"], G["disp"], co).astype(np.float32), G["density"])
    np.testing.assert_allclose(opm.gravity(G["pmid"], G["disp"], co, 0.3), G["acc"], rtol=1e-6, atol=1e-7)
    assert np.array_equal(opm.white_noise_nested(1234, co).view(np.uint32), G["noise"].view(np.uint32))


def _gpu():
    import pmpp_b200 as pb
    conf = pb.Configuration(16.0, (8, 8, 8), 2, a_start=0.1, a_custom=A, device="cuda")
    ptcl = pb.Particles(conf, torch.from_numpy(G["pmid"]).cuda(), torch.from_numpy(G["disp"]).cuda(),
                        torch.from_numpy(G["vel"]).cuda())
    return pb, conf, ptcl


@pytest.mark.gpu
def test_gpu_cic_and_sort_against_fixtures():
    pb, conf, ptcl = _gpu()
    from pmpp_b200 import sort as ps
    keys, perm = ps.sort_by_cell(ptcl, conf)
    assert np.array_equal(perm.cpu().numpy(), G["perm"])
    assert rel_err(pb.scatter(ptcl, conf).cpu().numpy(), G["density"]) < 2e-6
    m3 = torch.from_numpy(np.moveaxis(G["mesh3"], 0, -1).copy()).cuda()
    assert rel_err(pb.gather(ptcl, conf, m3).cpu().numpy(), G["gather3"]) < 2e-6
    dc, _ = pb.scatter_vjp(ptcl, conf, torch.from_numpy(G["mcot"]).cuda())
    assert rel_err(dc.cpu().numpy(), G["scatter_vjp_disp"]) < 5e-6
    dc, mc = pb.gather_vjp(ptcl, conf, m3, torch.from_numpy(G["vcot"]).cuda())
    assert rel_err(dc.cpu().numpy(), G["gather_vjp_disp"]) < 5e-6
    assert rel_err(np.moveaxis(mc.cpu().numpy(), -1, 0), G["gather_vjp_mesh"]) < 2e-6


@pytest.mark.gpu
def test_gpu_force_nbody_ic_pk_against_fixtures():
    pb, conf, ptcl = _gpu()
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    assert rel_err(pb.gravity(1.0, ptcl, cos, conf).cpu().numpy(), G["acc"]) < 2e-5
    dc, _ = pb.gravity_vjp(1.0, ptcl, cos, conf, torch.from_numpy(G["vcot"]).cuda())
    assert rel_err(dc.cpu().numpy(), G["gravity_vjp_disp"]) < 2e-5
    out = pb.nbody(ptcl, cos, conf)
    assert rel_err(out.disp.cpu().numpy(), G["nbody_disp"]) < 1e-4
    assert rel_err(out.vel.cpu().numpy(), G["nbody_vel"]) < 1e-4
    from pmpp_b200 import lpt as pl, modes as pm, power_spectrum as pps
    noise = pm.white_noise_nested(1234, conf).cpu().numpy()
    assert np.abs(noise - G["noise"]).max() < 5e-6 * np.abs(G["noise"]).max()
    lin = pm.linear_modes(torch.from_numpy(G["noise"]).cuda(), cos, conf)
    assert np.abs(lin.cpu().numpy() - G["linear_modes"]).max() < 2e-5 * np.abs(G["linear_modes"]).max()
    lp = pl.lpt(torch.from_numpy(G["linear_modes"]).cuda(), cos, conf)
    assert rel_err(lp.disp.cpu().numpy(), G["lpt_disp"]) < 2e-5
    assert rel_err(lp.vel.cpu().numpy(), G["lpt_vel"]) < 2e-5
    p = pb.Particles(conf, ptcl.pmid, torch.from_numpy(G["nbody_disp"]).cuda())
    k, pk, n = pps.particles_to_pk(p, conf)
    assert np.array_equal(n, G["pk_nmodes"])
    np.testing.assert_allclose(pk, G["pk"], rtol=2e-5)
