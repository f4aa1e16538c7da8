"""CUDA-graph-captured forward runs and the committed learned-correction weights."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pmpp_b200", "data",
                       "learned_green_c3.npy")


def test_graph_replay_equals_eager_run_bitwise():
    import pmpp_b200 as pb
    from pmpp_b200.graphs import GraphedForward
    from pmpp_b200 import lpt as pl, modes as pm
    a = np.geomspace(0.1, 1.0, 6)
    conf = pb.Configuration(4.0, (16, 16, 16), 2, a_start=0.1, a_custom=a, device="cuda")
    cos = pb.boltzmann(pb.SimpleLCDM(conf))
    ptcl = pl.lpt(pm.linear_modes(pm.white_noise_nested(2, conf), cos, conf), cos, conf)
    eager = pb.NBodyRun(conf, cos).forward(ptcl)
    g = GraphedForward(conf, cos, ptcl)
    out = g()
    for name in ("disp", "vel", "acc"):
        assert torch.equal(getattr(out, name), getattr(eager, name)), name
    disp2 = ptcl.disp * 1.01
    out2 = g(disp2, ptcl.vel)
    eager2 = pb.NBodyRun(conf, cos).forward(pb.Particles(conf, ptcl.pmid, disp2, ptcl.vel))
    assert torch.equal(out2.disp, eager2.disp)


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="trained weights not committed")
def test_committed_learned_weights_beat_plain_coarse_mesh():
    from pmpp_b200 import learned
    res = learned.evaluate(WEIGHTS, test_seeds=range(64, 66))
    assert res["max_pk_err_learned_128"] < 0.01
    assert res["max_pk_err_learned_128"] < 0.5 * res["max_pk_err_plain_128"]
