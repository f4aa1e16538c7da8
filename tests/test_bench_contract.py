"""CPU checks of bench.py's output contract: the reference arm's JSON line (a
tiny oracle sample), the workload config both arms share, and the byte models
the roofline divides by."""
import importlib.util
import json
import os
import subprocess
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--cpu-ptcl", "16"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    b = _bench()
    args = types.SimpleNamespace(ptcl=512, mesh=2, nsteps=32, gpus=1)
    assert d["config"] == b.arm_config(args, 1)
    assert d["metric"] == b.METRIC and d["unit"] == b.UNIT


def test_roofline_byte_models():
    from pmpp_b200.roofline import algorithmic_bytes
    N, M = 256**3, 512**3
    assert algorithmic_bytes("gather_kick", N, M) - algorithmic_bytes("gather", N, M) == 24 * N
    assert algorithmic_bytes("gather_kick", N, M) - algorithmic_bytes("gather_kick_only", N, M) == 12 * N
    b = _bench()
    # measured traffic per launch stays within a few percent of the algorithmic bytes
    for name in ("gather", "gather_kick"):
        ratio = b.MEASURED_TRAFFIC_PER_PARTICLE[name] * N / algorithmic_bytes(name, N, M)
        assert 0.95 < ratio < 1.05, (name, ratio)
    assert b.STAGE_VARIANTS["gather"] == ("gather_kick", "gather_kick_only")
    # a stage's bytes are the launch-weighted mean over the variants the timer counted
    conf = types.SimpleNamespace(mesh_shape=(512, 512, 512))
    counts = {"gather": 10, "gather_kick": 3, "gather_kick_only": 5}
    alg, _, mix = b.stage_mix("gather", counts, N, M, conf, None)
    want = (3 * algorithmic_bytes("gather_kick", N, M) + 5 * algorithmic_bytes("gather_kick_only", N, M)
            + 2 * algorithmic_bytes("gather", N, M)) / 10
    assert abs(alg - want) < 1 and mix == {"gather_kick": 3, "gather_kick_only": 5, "gather": 2}
    # combined fraction of a CIC group: total bytes over total time
    bd = {"scatter": {"ms_total": 2.0, "launches": 2}, "gather": {"ms_total": 5.0, "launches": 10}}
    peak = 1000.0
    fr = b.cic_fractions(bd, dict(counts, scatter=2), N, M, conf, None, peak)
    tot = 2 * algorithmic_bytes("scatter", N, M) + 10 * want
    assert abs(fr["scatter+gather"] - round(tot / 7e-3 / 1e9 / peak, 3)) < 1e-9 and "adjoint" not in fr


def test_pruned_byte_models():
    """Live fractions of the 512^3 / 1024^3 chain and the pruned pass bytes."""
    import pmpp_b200 as pb
    from pmpp_b200.roofline import algorithmic_bytes
    b = _bench()
    conf = pb.Configuration(2.0, (512,) * 3, 2, device="cpu")
    fy, fz = b.live_fractions(conf)
    assert fy == 513 / 1024 and fz == 257 / 513
    M, Mc = 1024 ** 3, 1024 * 1024 * 513
    full = algorithmic_bytes("fft_x_green", 0, M, Mc=Mc)
    assert algorithmic_bytes("fft_x_green", 0, M, Mc=Mc, live=(fy, fz)) == full * fy * fz
    assert algorithmic_bytes("fft_y", 0, M, Mc=Mc, live=(fy, fz)) == 8 * Mc * fz * (1 + fy)
    assert algorithmic_bytes("gather", 512 ** 3, M, live=(fy, fz)) == algorithmic_bytes("gather", 512 ** 3, M)
    assert b.live_fractions(pb.Configuration(2.0, (64,) * 3, 1, device="cpu")) is None


def test_gpus_flag_self_launches_ranks():
    """`bench.py --gpus 2` outside torchrun re-runs itself as two local ranks
    (torch.distributed.run, rendezvous on 127.0.0.1); exactly one line, from rank
    0, reports the job's two ranks.  The reference arm runs here (no GPU)."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "0", "--cpu-ptcl", "16"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["config"]["parallelism"] == "replicas x2"
    assert "sub-volume" in d["cpu_baseline"]["sample"]
