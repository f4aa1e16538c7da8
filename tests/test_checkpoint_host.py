"""Checkpoint files, saved-map configuration fields and segment ordering on
the host (no GPU): the state round-trips bitwise, a geometry or format
mismatch is refused, to_save_z converts to to_save_a (core/configuration.py:
311-318) and nbody_scheduled runs segments in order, reversed with reverse
(nbody/solver.py:645-679)."""
import numpy as np
import pytest
import torch


def _conf(**kw):
    import pmpp_b200 as pb
    return pb, pb.Configuration(2.0, (4, 4, 4), 2, device="cpu", **kw)


def test_state_round_trip_and_geometry_check(tmp_path):
    pb, conf = _conf()
    g = torch.Generator().manual_seed(0)
    n = conf.ptcl_num
    unused = torch.zeros(n, dtype=torch.bool)
    unused[-5:] = True
    p = pb.Particles(conf, torch.randint(0, 8, (n, 3), dtype=torch.int16, generator=g),
                     torch.randn((n, 3), generator=g), torch.randn((n, 3), generator=g), None, unused_index=unused)
    path = tmp_path / "s.npz"
    pb.save_state(path, p, 0.25, conf)
    q, a = pb.load_state(path, conf)
    assert a == 0.25 and q.acc is None
    for x, y in ((q.pmid, p.pmid), (q.disp, p.disp), (q.vel, p.vel), (q.unused_index, p.unused_index)):
        assert torch.equal(x, y)
    _, other = _conf()
    other.mesh_shape = (16, 16, 16)
    with pytest.raises(ValueError, match="geometry"):
        pb.load_state(path, other)
    with np.load(path) as z:
        d = dict(z)
    d["format_version"] = np.int64(99)
    np.savez(tmp_path / "bad.npz", **d)
    with pytest.raises(ValueError, match="format"):
        pb.load_state(tmp_path / "bad.npz", conf)


def test_save_fields_and_scheduled_order(monkeypatch):
    pb, conf = _conf(to_save_z=[1.0, 3.0], slice_to_save=[0, 4, 8], max_slice_width=4)
    np.testing.assert_allclose(conf.to_save_a, [0.5, 0.25])
    assert conf.nMesh == 8 and conf.max_slice_width == 4
    import importlib
    nb = importlib.import_module("pmpp_b200.nbody")
    calls = []

    def fake(state, cosmo, c, reverse=False, correction=None):
        calls.append((c, reverse))
        return state * 10 + c

    monkeypatch.setattr(nb, "nbody", fake)
    assert nb.nbody_scheduled(0, object(), [1, 2, 3]) == 123
    assert calls == [(1, False), (2, False), (3, False)]
    calls.clear()
    assert nb.nbody_static_halo_scheduled(0, object(), [1, 2, 3], reverse=True) == 321
    assert calls == [(3, True), (2, True), (1, True)]


def test_observation_trees_stack():
    from pmpp_b200.nbody import _stack_tree
    obs = [{"a": 0.5, "m": torch.ones(2), "t": (torch.zeros(1), 1)}, {"a": 0.6, "m": torch.zeros(2),
                                                                       "t": (torch.ones(1), 2)}]
    s = _stack_tree(obs)
    np.testing.assert_allclose(s["a"].numpy(), [0.5, 0.6])
    assert s["m"].shape == (2, 2) and s["t"][0].shape == (2, 1)
    np.testing.assert_array_equal(s["t"][1].numpy(), [1, 2])
