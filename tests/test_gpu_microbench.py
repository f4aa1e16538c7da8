"""The PM stage microbenchmark runs on both position sets at a small size."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_microbench_small():
    from pmpp_b200 import microbench
    res = microbench.main(["--ptcl", "64", "--mesh", "2", "--reps", "2"])
    for s in ("U", "K"):
        stages = {k: v for k, v in res[s].items() if k != "touched_cells"}
        assert set(stages) == {"sort", "scatter", "fft_r2c", "green_gradient", "fft_c2r_x3", "gather", "scatter_adjoint",
                               "gather_adjoint", "scatter3", "fft_r2c_x3", "green_gradient_adjoint", "fft_c2r",
                               "gather@staged", "gather_adjoint@staged"}
        assert all(v["ms"] > 0 for v in stages.values())
        assert 0 < res[s]["touched_cells"] <= 128**3


def test_position_sets_conserve_mass():
    import pmpp_b200 as pb
    from pmpp_b200 import microbench
    from pmpp_b200.cic import SortedParticles
    conf = pb.Configuration(4.0, (64, 64, 64), 2, a_start=0.1, device="cuda")
    for p in (microbench.uniform_positions(conf), microbench.clustered_positions(conf)):
        rho = SortedParticles(p.pmid, p.disp, conf).scatter()[0]
        assert abs(float(rho.double().sum()) / conf.mesh_size - 1.0) < 1e-6
