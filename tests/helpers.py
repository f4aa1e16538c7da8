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


def fixed_point_scatter(pmid, disp, conf_o, val, offset=0, valid=None, cell_size=None, mesh_shape=None,
                        n_total=None):
    """Bit-exact restatement of the GPU deposit's arithmetic (mode 0).

    float32 corner weights as the reference enmesh forms them, contributions
    c = float32(val * w), q = round_half_even(float64(c) * scale) summed exactly
    in int64 per cell, result float32(float64(sum) / scale), with the power of
    two scale = 2^e / 2^ceil(log2 max|val|) and e = min(62 - ceil(log2(n + 1)), 52)
    (n counts every particle, masked ones included; n_total when pmid is a
    subset of the particles the device deposited)."""
    mesh_shape = conf_o.mesh_shape if mesh_shape is None else mesh_shape
    idx, w, _, _ = opm.corners(pmid, disp, conf_o, mesh_shape, offset, cell_size, valid)
    keep = idx >= 0
    n = len(pmid) if n_total is None else int(n_total)
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
        contrib = np.broadcast_to((v[:, None] if v.ndim == 1 else v) * w, idx.shape)
        q = np.rint(contrib.astype(np.float64) * scale)[keep]
        # integer sums in float64 are exact (any order) while every partial sum
        # stays below 2^53, which the sum of |q| per cell bounds; else int64
        bound = np.bincount(idx[keep], weights=np.abs(q), minlength=M)
        if bound.max() < 2.0**53:
            acc = np.bincount(idx[keep], weights=q, minlength=M)
        else:
            acc = np.zeros(M, np.int64)
            np.add.at(acc, idx[keep], q.astype(np.int64))
            acc = acc.astype(np.float64)
        outs.append((acc * (1.0 / scale)).astype(np.float32).reshape(mesh_shape))
    return outs[0] if val.ndim <= 1 else np.stack(outs)
