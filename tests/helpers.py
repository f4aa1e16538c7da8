"""Shared fixtures for the parity tests: seeded particle sets and configs."""
import numpy as np

from oracle import pm as opm


def random_particles(conf_o, seed=0, spread=3.0, lattice=True):
    """Lattice (gen_grid) particles with seeded random displacements of a few cells."""
    rng = np.random.default_rng(seed)
    pmid, disp = opm.gen_grid(conf_o)
    disp = (disp + rng.normal(0, spread * conf_o.cell_size, size=disp.shape)).astype(np.float32)
    if not lattice:
        pmid = rng.integers(0, min(conf_o.mesh_shape), size=pmid.shape).astype(np.int16)
    return pmid, disp


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def fixed_point_scatter(pmid, disp, conf_o, val):
    """Bit-exact restatement of the GPU deposit's arithmetic (mode 0).

    float32 corner weights as the reference enmesh forms them, contributions
    c = float32(val * w), q = round_half_even(float64(c) * scale) summed exactly
    in int64 per cell, result float32(float64(sum) / scale), with the power of
    two scale = 2^e / 2^ceil(log2 max|val|) and e = min(62 - ceil(log2(n + 1)), 52)."""
    mesh_shape = conf_o.mesh_shape
    cell, d, fl = opm.enmesh(pmid, disp, conf_o)
    w, _ = opm.corner_weights(d, fl, np.float32)
    idx = opm.corner_index(cell, mesh_shape)
    n = len(pmid)
    lg = 0
    while (1 << lg) < n + 1:
        lg += 1
    e = min(62 - lg, 52)
    val = np.asarray(val, np.float32)
    m, x = np.frexp(float(np.abs(val).max()))
    scale = np.ldexp(1.0, e - (int(x) - 1 if m == 0.5 else int(x)))
    M = int(np.prod(mesh_shape))
    chans = [val] if val.ndim <= 1 else [val[:, c] for c in range(val.shape[1])]
    outs = []
    for v in chans:
        contrib = (v[:, None] if v.ndim == 1 else v) * w
        q = np.rint(contrib.astype(np.float64) * scale).astype(np.int64)
        acc = np.zeros(M, np.int64)
        np.add.at(acc, idx.ravel(), q.ravel())
        outs.append((acc.astype(np.float64) * (1.0 / scale)).astype(np.float32).reshape(mesh_shape))
    return outs[0] if val.ndim <= 1 else np.stack(outs)
