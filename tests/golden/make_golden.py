"""Generate the golden fixtures in this folder from the CPU oracle.

    python tests/golden/make_golden.py

The fixtures freeze small float32 cases of every hot-path stage (inputs and the oracle's
outputs) so the GPU parity tests compare against committed numbers, not only against a
live oracle run.  The oracle restates PM++ (see oracle/pm.py); it is pinned against the
reference test suite's closed-form checks in tests/test_oracle_pins.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import cosmology as ocos  # noqa: E402
from oracle import pm as opm  # noqa: E402

A = np.linspace(0.1, 1.0, 4)


def conf():
    return opm.Conf(16.0, (8, 8, 8), mesh_shape=2, a_start=0.1, a_custom=A)


def make():
    co = conf()
    cosmo = opm.boltzmann(ocos.Cosmo(), co)
    rng = np.random.default_rng(2024)
    pmid, disp = opm.gen_grid(co)
    disp = (disp + rng.normal(0, 1.5 * co.cell_size, size=disp.shape)).astype(np.float32)
    vel = rng.normal(0, 0.5, size=disp.shape).astype(np.float32)
    mesh3 = rng.normal(size=(3, ) + co.mesh_shape).astype(np.float32)
    vcot = rng.normal(size=disp.shape).astype(np.float32)
    mcot = rng.normal(size=co.mesh_shape).astype(np.float32)
    out = {"pmid": pmid, "disp": disp, "vel": vel, "mesh3": mesh3, "vcot": vcot, "mcot": mcot}
    out["keys"], out["perm"] = opm.sort_by_cell(pmid, disp, co)
    out["density"] = opm.scatter(pmid, disp, co).astype(np.float32)
    out["gather3"] = opm.gather(pmid, disp, co, mesh3.astype(np.float64)).astype(np.float32)
    out["scatter_vjp_disp"] = opm.scatter_vjp(pmid, disp, co, mcot.astype(np.float64))[0].astype(np.float32)
    gd, gm = opm.gather_vjp(pmid, disp, co, mesh3.astype(np.float64), vcot)
    out["gather_vjp_disp"] = gd.astype(np.float32)
    out["gather_vjp_mesh"] = gm.astype(np.float32)
    out["acc"] = opm.gravity(pmid, disp, co, 0.3).astype(np.float32)
    out["gravity_vjp_disp"] = opm.gravity_vjp(pmid, disp, co, 0.3, vcot)[0].astype(np.float32)
    d, v, a = opm.nbody(pmid, disp, vel, co, cosmo)
    out["nbody_disp"], out["nbody_vel"], out["nbody_acc"] = d, v, a
    noise = opm.white_noise_nested(1234, co)
    out["noise"] = noise
    lin = opm.linear_modes(noise, cosmo, co)
    out["linear_modes"] = lin
    _, ld, lv = opm.lpt(lin, cosmo, co)
    out["lpt_disp"], out["lpt_vel"] = ld, lv
    rho = opm.scatter(pmid, d, co)
    k, pk, n = opm.density_to_pk(rho, co)
    out["pk_k"], out["pk"], out["pk_nmodes"] = k, pk, n
    np.savez_compressed(os.path.join(HERE, "pm_small.npz"), **out)


if __name__ == "__main__":
    make()
    print("wrote", os.path.join(HERE, "pm_small.npz"))
