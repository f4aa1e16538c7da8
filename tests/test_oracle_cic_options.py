"""CPU checks of the oracle's CIC options (offset, explicit cell size, unused
slots) against properties the reference's own formulas imply: an explicit cell
size equal to the particle cell reproduces the common-grid path, every
particle's mass lands on the target mesh when it covers the box, a whole-cell
offset is an index shift, and unused slots contribute nothing."""
import numpy as np

from oracle import pm as opm
from tests.helpers import random_particles


def _conf():
    co = opm.Conf(2.0, (12, 12, 12), mesh_shape=2)
    pmid, disp = random_particles(co, 3, 3.0)
    return co, pmid, disp


def test_explicit_cell_equal_to_particle_cell_matches_common_path():
    co, pmid, disp = _conf()
    a = opm.scatter(pmid, disp, co)
    b = opm.scatter(pmid, disp, co, cell_size=co.cell_size)
    assert np.abs(a - b).max() < 1e-5 * np.abs(a).max()


def test_explicit_coarse_mesh_conserves_mass_and_gather_of_constant():
    co, pmid, disp = _conf()
    shape = tuple(s // 2 for s in co.mesh_shape)
    m = opm.scatter(pmid, disp, co, val=1.0, mesh_shape=shape, cell_size=2 * co.cell_size, offset=0.3)
    np.testing.assert_allclose(m.sum(), len(pmid), rtol=1e-6)
    g = opm.gather(pmid, disp, co, np.ones(shape), cell_size=2 * co.cell_size, offset=0.3)
    np.testing.assert_allclose(g, 1.0, rtol=1e-6)


def test_whole_cell_offset_is_index_shift_and_mask_drops_particles():
    co, pmid, disp = _conf()
    base = opm.scatter(pmid, disp, co)
    sh = opm.scatter(pmid, disp, co, offset=[co.cell_size, 0.0, -2 * co.cell_size])
    np.testing.assert_array_equal(sh, np.roll(base, (-1, 0, 2), axis=(0, 1, 2)))
    valid = np.arange(len(pmid)) % 3 != 0
    a = opm.scatter(pmid, disp, co, valid=valid)
    b = opm.scatter(pmid[valid], disp[valid], co, val=opm.default_val(co))
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-12)
    dc, vc = opm.scatter_vjp(pmid, disp, co, np.random.default_rng(0).normal(size=co.mesh_shape), valid=valid)
    assert np.all(dc[~valid] == 0)
