"""Host-side particle constructors (no GPU): from_pos / from_ordered_pos
against the reference's ordered-initialisation test (restated from
tests/test_particles_ordered_init.py:9-29) and against numpy restatements of
particles.py:441-479 and :497-545 in float32; gen_grid against the oracle."""
import numpy as np
import torch

import pmpp_b200 as pb


def _raveled(pmid, conf):
    return pb.pmid_to_idx(pmid, conf).numpy()


def _lattice(conf):
    axes = [np.arange(n, dtype=np.float32) * np.float32(conf.ptcl_spacing) for n in conf.ptcl_grid_shape]
    return np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)


def test_from_ordered_pos_keeps_unique_anchors_under_collisions():
    conf = pb.Configuration(1.0, (4, 4, 4), 1, device="cpu")
    pos = _lattice(conf)
    # particles 0 and 16 share y, z; moving both to x = 0.6 makes them round to the same cell
    pos[0, 0] = np.float32(0.6)
    pos[16, 0] = np.float32(0.6)
    colliding = pb.Particles.from_pos(conf, torch.from_numpy(pos))
    assert np.unique(_raveled(colliding.pmid, conf)).size < conf.ptcl_num
    ordered = pb.Particles.from_ordered_pos(conf, torch.from_numpy(pos))
    assert np.unique(_raveled(ordered.pmid, conf)).size == conf.ptcl_num
    np.testing.assert_allclose(ordered.pos(dtype=torch.float32).numpy(), pos, atol=1e-6, rtol=1e-6)


def _scattered_positions(conf, seed):
    rng = np.random.default_rng(seed)
    base = _lattice(conf).astype(np.float64)
    box = np.asarray(conf.box_size, dtype=np.float64)
    return ((base + rng.normal(0, 2.0 * conf.cell_size, size=base.shape)) % box).astype(np.float32)


def test_from_ordered_pos_matches_nearest_image_restatement():
    for shape, mesh in (((8, 8, 8), 2), ((4, 8, 16), 1), ((6, 4, 8), 2)):
        conf = pb.Configuration(1.5, shape, mesh, device="cpu")
        pos = _scattered_positions(conf, seed=sum(shape))
        got = pb.Particles.from_ordered_pos(conf, torch.from_numpy(pos))
        grid = pb.Particles.gen_grid(conf)
        assert torch.equal(got.pmid, grid.pmid)
        anchor = grid.pmid.numpy().astype(np.float32) * np.float32(conf.cell_size)
        box = np.asarray(conf.box_size, dtype=np.float32)
        ref = (pos - anchor + np.float32(0.5) * box) % box - np.float32(0.5) * box
        np.testing.assert_array_equal(got.disp.numpy(), ref)
        # positions come back to within float32 rounding of the box
        back = got.pos(dtype=torch.float64).numpy()
        d = (back - pos.astype(np.float64) + box / 2) % box - box / 2
        assert np.abs(d).max() < 1e-4


def test_from_pos_matches_rint_restatement():
    conf = pb.Configuration(1.5, (8, 8, 8), 2, device="cpu")
    pos = _scattered_positions(conf, seed=4)
    got = pb.Particles.from_pos(conf, torch.from_numpy(pos))
    c = np.float32(conf.cell_size)
    pm = np.rint(pos / c)
    disp = pos - pm * c
    pm = np.mod(pm.astype(np.int16), np.asarray(conf.mesh_shape, dtype=np.int16))
    np.testing.assert_array_equal(got.pmid.numpy(), pm)
    np.testing.assert_array_equal(got.disp.numpy(), disp.astype(np.float32))


def test_from_ordered_pos_rejects_partial_arrays():
    conf = pb.Configuration(1.0, (4, 4, 4), 1, device="cpu")
    pos = torch.from_numpy(_lattice(conf)[:10])
    try:
        pb.Particles.from_ordered_pos(conf, pos)
    except ValueError as e:
        assert "expected 64 particles, got 10" in str(e)
    else:
        raise AssertionError("partial array accepted")


def test_gen_grid_matches_oracle_bitwise():
    """Lattice anchors and displacements of gen_grid (particles.py:615-727),
    including mesh / particle ratios that are not integers, where the anchors
    come from rounding."""
    from oracle import pm as opm
    for shape, mesh in (((4, 4, 4), 1), ((8, 8, 8), 2), ((6, 4, 10), (9, 6, 15)), ((16, 16, 16), 1.5),
                        ((12, 12, 12), (20, 20, 20))):
        co = opm.Conf(2.0, shape, mesh_shape=mesh)
        conf = pb.Configuration(2.0, shape, mesh, device="cpu")
        pmid, disp = opm.gen_grid(co)
        g = pb.Particles.gen_grid(conf)
        np.testing.assert_array_equal(g.pmid.numpy(), pmid)
        np.testing.assert_array_equal(g.disp.numpy(), disp.astype(np.float32))


def _small_conf(shape=(3, 2, 2), mesh=2):
    return pb.Configuration(0.75, shape, mesh, device="cpu")


def test_coordinate_conversions_keep_subcell_offsets_and_periodicity():
    """Restated from the reference's tests/test_deep_particles.py:39-60."""
    conf = _small_conf()
    box = np.asarray(conf.box_size, dtype=np.float32)
    pos = torch.tensor([[-0.03, 0.11, 0.73], [0.38, 0.77, 1.51], [2.26, -0.01, 0.05]], dtype=torch.float32)
    unwrapped = pb.Particles.from_pos(conf, pos, wrap=False)
    wrapped = pb.Particles.from_pos_sharded(conf, pos, wrap=True)
    expected = np.mod(pos.numpy(), box)
    np.testing.assert_allclose(unwrapped.pos(dtype=torch.float32, wrap=False).numpy(), pos.numpy(), atol=2e-7)
    np.testing.assert_allclose(wrapped.pos(dtype=torch.float32).numpy(), expected, atol=2e-7)
    assert bool((unwrapped.pmid != wrapped.pmid).any()) and bool((wrapped.pmid >= 0).all())
    pmid, disp = pb.Particles.pos_to_pmid(pos, conf)
    np.testing.assert_allclose(pb.Particles.pmid_to_pos(pmid, disp, conf).numpy(), expected, atol=2e-7)
    assert torch.equal(pmid, wrapped.pmid)
    np.testing.assert_allclose(disp.numpy(), wrapped.disp.numpy(), atol=1e-7)
    jac = torch.autograd.functional.jacobian(
        lambda x: pb.Particles.from_pos(conf, x, wrap=False).pos(dtype=torch.float32, wrap=False), pos)
    np.testing.assert_allclose(jac.reshape(pos.numel(), pos.numel()).numpy(), np.eye(pos.numel()), atol=2e-6)


def test_ids_indexing_attributes_and_ordered_initialisation():
    """Restated from the reference's tests/test_deep_particles.py:63-92."""
    conf = _small_conf(shape=(2, 2, 2), mesh=2)
    grid = pb.Particles.gen_grid(conf, vel=True, acc=True)
    assert len(grid) == conf.ptcl_num
    assert grid.pmid.dtype == torch.int16 and grid.disp.dtype == conf.float_dtype
    assert float(grid.vel.abs().max()) == 0 and float(grid.acc.abs().max()) == 0
    expected = np.ravel_multi_index(tuple(grid.pmid.numpy().astype(np.int64).T), conf.mesh_shape)
    np.testing.assert_array_equal(grid.raveled_id().numpy(), expected)
    first = grid[0]
    assert tuple(first.pmid.shape) == (3, ) and torch.equal(first.pmid, grid.pmid[0])
    attr = {"mass": np.arange(conf.ptcl_num, dtype=np.float64), "tag": np.ones((conf.ptcl_num, 2))}
    attributed = pb.Particles(conf, grid.pmid, grid.disp, attr=attr)
    assert attributed.attr["mass"].dtype == conf.float_dtype and attributed.attr["tag"].dtype == conf.float_dtype
    np.testing.assert_array_equal(attributed[:2].attr["mass"].numpy(), [0, 1])
    shifted = grid.pos(dtype=torch.float32).clone()
    shifted[:, 0] += np.float32(0.37)
    ordered = pb.Particles.from_ordered_pos(conf, shifted, vel=torch.ones_like(shifted),
                                            acc=2 * torch.ones_like(shifted))
    assert torch.equal(ordered.pmid, grid.pmid)
    np.testing.assert_allclose(ordered.pos(dtype=torch.float32).numpy(), shifted.numpy(), atol=2e-7)
    import pytest
    with pytest.raises(ValueError, match="full particle-grid ordered"):
        pb.Particles.from_ordered_pos(conf, shifted[:-1])


def test_raveled_ids_and_copies_wrap_only_when_requested():
    """Restated from the reference's tests/test_deep_particles.py:95-109."""
    conf = _small_conf(shape=(2, 2, 2), mesh=1)
    pmid = torch.tensor([[-1, 0, 0], [0, 1, 1], [2, 0, 0]], dtype=torch.int16)
    disp = torch.zeros((3, 3), dtype=torch.float32)
    original = pb.Particles.from_pmid(conf, pmid, disp, vel=torch.ones_like(disp), acc=2 * torch.ones_like(disp))
    np.testing.assert_array_equal(original.raveled_id(dtype=torch.int32, wrap=True).numpy(), [4, 3, 0])
    np.testing.assert_array_equal(original.raveled_id(dtype=torch.int32, wrap=False).numpy(), [-4, 3, 8])
    copied = pb.Particles.from_ptcl(original)
    unwrapped = pb.Particles.from_ptcl(original, conf=conf, wrap=False)
    np.testing.assert_array_equal(copied.pmid.numpy(), [[1, 0, 0], [0, 1, 1], [0, 0, 0]])
    assert torch.equal(unwrapped.pmid, pmid)
    assert float(copied.vel.min()) == 1 and float(copied.acc.min()) == 2
    import pytest
    with pytest.raises(TypeError):
        original.raveled_id(dtype=torch.float32)


def test_pmid_to_idx_wraps_and_masks():
    """core/utils.py:292-326: int32 keys, anchors wrapped, unused slots -1."""
    conf = _small_conf(shape=(2, 2, 2), mesh=1)
    pmid = torch.tensor([[-1, 0, 0], [0, 1, 1], [2, 0, 0], [1, 1, 1]], dtype=torch.int16)
    idx = pb.pmid_to_idx(pmid, conf)
    assert idx.dtype == torch.int32
    np.testing.assert_array_equal(idx.numpy(), [4, 3, 0, 7])
    masked = pb.pmid_to_idx(pmid, conf, unused_index=torch.tensor([False, True, False, False]))
    np.testing.assert_array_equal(masked.numpy(), [4, -1, 0, 7])


def test_large_meshes_keep_exact_sizes_and_ids_fail_closed():
    """Restated from the reference's tests/test_lpt_large_index.py:46-60:
    2048^3 sizes stay exact integers; raveled ids refuse a dtype that cannot
    hold every mesh index."""
    import pytest
    conf = pb.Configuration(1.0, (2048, 2048, 2048), 1, device="cpu")
    assert conf.ptcl_num == 8_589_934_592 and conf.mesh_size == 8_589_934_592
    p = pb.Particles(conf, torch.tensor([[2047, 2047, 2047]], dtype=torch.int16), torch.zeros((1, 3)))
    with pytest.raises(OverflowError):
        p.raveled_id(dtype=torch.int32)
    assert int(p.raveled_id()[0]) == 8_589_934_591
