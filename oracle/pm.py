"""CPU oracle -- test infrastructure only, never part of the product path.

NumPy restatement of PM++'s single-GPU particle-mesh step, used as the checker
for the CUDA kernels.  It runs in float64 (the reference's x64 build) or in
float32 (reproducing the reference's float32 binning and weight arithmetic).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import it.

Each function cites the reference file:line it restates (paths relative to
the PM++ source tree ``src/pmpp``).  Parity status: partially pinned -- the
reference (JAX) cannot be imported here, so the restatement is pinned against
the reference's own closed-form known-answer tests (see tests/test_oracle_*.py),
not against outputs of the reference itself.
"""
from __future__ import annotations

import math

import numpy as np

from . import cosmology as cos

# Corner order of enmesh.py:98 / pallas.py:166: bit a of the corner index
# selects +1 along axis a.
NEIGHBORS = ((np.arange(8)[:, None] >> np.arange(3)) & 1).astype(np.int64)


class _FFT:
    """numpy.fft by default; scipy.fft with worker threads for the timed CPU baseline."""
    workers = 1

    def rfftn(self, x):
        if self.workers > 1:
            import scipy.fft
            return scipy.fft.rfftn(x, workers=self.workers)
        return np.fft.rfftn(x)

    def irfftn(self, x, s):
        if self.workers > 1:
            import scipy.fft
            return scipy.fft.irfftn(x, s=s, workers=self.workers)
        return np.fft.irfftn(x, s=s)


_fft = _FFT()


def set_fft_workers(n):
    """Threads for the FFTs and the particle loops of the CIC functions (the
    timed CPU baseline); 1 (the default, used by the tests) is plain serial
    NumPy."""
    _fft.workers = int(n)


def _chunks(n, partial_bytes=0):
    """Particle ranges of the threaded CIC (None: run serially).  At most 16
    chunks, and few enough that the partial meshes of a deposit (partial_bytes
    each, all in flight at once) stay within 8 GB."""
    w = min(_fft.workers, 16)
    if partial_bytes > 0:
        w = min(w, max(1, int(8e9 // partial_bytes)))
    if w <= 1 or n < 65536:
        return None
    b = np.linspace(0, n, w + 1).astype(np.int64)
    return [(int(b[i]), int(b[i + 1])) for i in range(w) if b[i + 1] > b[i]]


def _pmap(fn, ranges):
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(len(ranges)) as ex:
        return list(ex.map(lambda r: fn(*r), ranges))


def _psum(fn, ranges):
    """Sum of fn over the chunks, in chunk order, keeping one running total."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(len(ranges)) as ex:
        it = ex.map(lambda r: fn(*r), ranges)
        total = next(it)
        for part in it:
            total = total + part
        return total


def _rows(x, lo, hi):
    """Particle slice of a per-particle array (scalars pass through)."""
    x = np.asarray(x) if x is not None else None
    return x if x is None or x.ndim == 0 else x[lo:hi]


class Conf:
    """Configuration fields the hot path reads (core/configuration.py:172-575)."""

    def __init__(self, ptcl_spacing, ptcl_grid_shape, mesh_shape=1, float_dtype=np.float32, a_start=1 / 64,
                 a_stop=1.0, a_lpt_maxstep=1 / 128, a_nbody_maxstep=1 / 64, a_custom=None,
                 symp_splits=((0, 0.5), (1, 0.5)), lpt_order=2, transfer_lgk_min=-4, transfer_lgk_max=3,
                 transfer_lgk_maxstep=1 / 128):
        self.ptcl_spacing = float(ptcl_spacing)
        self.ptcl_grid_shape = tuple(int(s) for s in ptcl_grid_shape)
        if isinstance(mesh_shape, (int, float)):
            mesh_shape = tuple(round(s * mesh_shape) for s in self.ptcl_grid_shape)  # configuration.py:249-252
        self.mesh_shape = tuple(int(s) for s in mesh_shape)
        self.float_dtype = np.dtype(float_dtype)
        self.complex_dtype = np.dtype(np.complex64 if self.float_dtype == np.float32 else np.complex128)
        self.a_start = float(a_start)
        self.a_stop = float(a_stop)
        self.a_lpt_maxstep = a_lpt_maxstep
        self.a_nbody_maxstep = a_nbody_maxstep
        self.a_custom = None if a_custom is None else tuple(float(a) for a in a_custom)
        self.symp_splits = symp_splits
        self.lpt_order = lpt_order
        self.transfer_lgk_min = transfer_lgk_min
        self.transfer_lgk_max = transfer_lgk_max
        self.transfer_lgk_maxstep = transfer_lgk_maxstep
        self.kvec = fftfreq(self.mesh_shape, self.cell_size, self.float_dtype)
        self.kvec_spacing = fftfreq(self.ptcl_grid_shape, self.ptcl_spacing, self.float_dtype)
        self.neg_ik = tuple(self._neg_k(k) for k in self.kvec)

    def fastpm_neg_k(self, k):
        """Real factor c with neg_ik = i*c for FastPM's 4-point derivative,
        (8 sin(k dx) - sin(2 k dx)) / (6 dx) (gravity.py:385-387), in the float dtype."""
        f = self.float_dtype.type
        phase = (k * f(self.cell_size)).astype(self.float_dtype)
        d = ((f(8.0) * np.sin(phase)).astype(self.float_dtype) - np.sin(f(2.0) * phase)).astype(self.float_dtype)
        return (-(d / f(6.0 * self.cell_size))).astype(self.float_dtype)

    def derivative_factors(self, gradient="spectral"):
        if gradient == "spectral":
            return self.neg_ik
        if gradient == "fastpm_4point":
            return tuple(self.fastpm_neg_k(k) for k in self.kvec)
        raise ValueError(f"Unsupported force-gradient kernel {gradient!r}.")

    def _neg_k(self, k):
        """Real factor c with neg_ik = i*c (configuration.py:370-376)."""
        f = self.float_dtype.type
        nyquist = f(np.pi / self.cell_size)
        eps = nyquist * np.finfo(self.float_dtype).eps
        return np.where(np.abs(np.abs(k) - nyquist) <= eps, f(0), -k).astype(self.float_dtype)

    # derived quantities, configuration.py:437-563
    @property
    def dim(self):
        return len(self.ptcl_grid_shape)

    @property
    def ptcl_num(self):
        return math.prod(self.ptcl_grid_shape)

    @property
    def mesh_size(self):
        return math.prod(self.mesh_shape)

    @property
    def cell_size(self):
        return self.ptcl_spacing * self.ptcl_grid_shape[0] / self.mesh_shape[0]

    @property
    def ptcl_cell_vol(self):
        return self.ptcl_spacing**self.dim

    @property
    def box_size(self):
        return tuple(self.ptcl_spacing * s for s in self.ptcl_grid_shape)

    @property
    def box_vol(self):
        return float(np.prod(self.box_size))

    @property
    def transfer_k_num(self):
        return 1 + math.ceil((self.transfer_lgk_max - self.transfer_lgk_min) / self.transfer_lgk_maxstep) + 1

    @property
    def transfer_k(self):
        k = np.logspace(self.transfer_lgk_min, self.transfer_lgk_max, num=self.transfer_k_num - 1)
        return np.concatenate(([0.0], k))

    @property
    def a_lpt_num(self):
        return math.ceil(self.a_start / self.a_lpt_maxstep)

    @property
    def a_lpt_step(self):
        return self.a_start / self.a_lpt_num

    @property
    def a_nbody_num(self):
        return math.ceil((self.a_stop - self.a_start) / self.a_nbody_maxstep)

    @property
    def a_lpt(self):
        return np.linspace(0, self.a_start, num=self.a_lpt_num + 1)

    @property
    def a_nbody(self):
        if self.a_custom is not None:
            return np.array(self.a_custom, dtype=np.float64)
        return np.linspace(self.a_start, self.a_stop, num=1 + self.a_nbody_num)

    @property
    def growth_a(self):
        return np.concatenate((self.a_lpt, self.a_nbody[1:]))

    @property
    def particle_nyquist_masks(self):
        """core/utils.py:15-37 (empty when the mesh equals the particle grid)."""
        if self.mesh_shape == self.ptcl_grid_shape:
            return ()
        f = self.float_dtype.type
        kn = f(np.pi / self.ptcl_spacing)
        limit = kn + kn * f(8 * np.finfo(self.float_dtype).eps)
        return tuple((np.abs(k) <= limit).astype(self.float_dtype) for k in self.kvec)


def fftfreq(shape, spacing, dtype):
    """Angular wavevectors, numerics/fft.py:4-44 (1-D per axis; rfft last)."""
    period = 2 * np.pi / spacing
    ks = [(np.fft.fftfreq(s) * period).astype(dtype) for s in shape[:-1]]
    ks.append((np.fft.rfftfreq(shape[-1]) * period).astype(dtype))
    return tuple(ks)


def boltzmann(cosmo, conf):
    """Transfer + growth tables, cosmology/boltzmann.py:358-398 (varlin via quadrature)."""
    cosmo.transfer = cos.transfer_fit(conf.transfer_k, cosmo)
    cosmo.growth = cos.growth_integ(cosmo, conf.growth_a, conf.a_lpt_step)
    return cosmo


def cosmo_from_sigma8(conf, sigma8, **kw):
    """Cosmology.from_sigma8, cosmology/models.py:183-203."""
    c1 = boltzmann(cos.Cosmo(A_s_1e9=1.0, **kw), conf)
    A = (sigma8 / sigma8_of(c1, conf))**2
    return boltzmann(cos.Cosmo(A_s_1e9=A, **kw), conf)


def sigma8_of(cosmo, conf):
    """Cosmology.sigma8 = sqrt(varlin(8 Mpc/h, a=1)), models.py:249-254 + boltzmann.py:314-355."""
    return cos.sigma8(cosmo, conf.transfer_k) * float(cos.growth(1.0, cosmo, conf.growth_a))


# --------------------------------------------------------------------------
# Particles
# --------------------------------------------------------------------------
def gen_grid(conf):
    """Lagrangian lattice (nbody/particles.py:615-727), single device."""
    pmid, disp = [], []
    for sp, sm in zip(conf.ptcl_grid_shape, conf.mesh_shape):
        p = np.rint(np.linspace(0, sm, num=sp, endpoint=False)).astype(np.int16)
        d = (np.arange(sp) * sm - p.astype(np.int64) * sp) * (conf.cell_size / sp)
        pmid.append(p)
        disp.append(d.astype(conf.float_dtype))
    pmid = np.stack(np.meshgrid(*pmid, indexing='ij'), axis=-1).reshape(-1, 3)
    disp = np.stack(np.meshgrid(*disp, indexing='ij'), axis=-1).reshape(-1, 3)
    return pmid, disp


def positions(pmid, disp, conf):
    """Particles.pos, particles.py:773-798 (float64, wrapped)."""
    pos = pmid.astype(np.float64) * conf.cell_size + disp.astype(np.float64)
    return pos % np.array(conf.box_size)


# --------------------------------------------------------------------------
# CIC binning, cic/enmesh.py:34-165 (a2=None branch) and pallas.py:225-256
# --------------------------------------------------------------------------
def offset_shift(offset, cell, dtype):
    """Mesh origin offset as whole cells q = floor(o / cell) and the remainder
    o - q * cell rounded once to the float dtype (the common-grid offset path,
    cic/pallas.py:225-238, cic/enmesh.py:128-147).  The offset itself is first
    rounded to the float dtype, as the reference casts it (pallas.py:108-111)."""
    o = np.broadcast_to(np.asarray(offset, dtype=dtype).astype(np.float64), (3, ))
    q = np.floor(o / float(cell))
    return q.astype(np.int64), (o - q * float(cell)).astype(dtype)


def enmesh(pmid, disp, conf, mesh_shape=None, offset=0):
    """Return lower-corner cells (N,3) int64, normalised fractions (N,3).

    The float arithmetic follows enmesh.py:139-143 in ``conf.float_dtype``:
    d = (disp - r) / cell, i = floor(d), f = d - i, with the neighbour deltas
    d - (i + b) formed later in :func:`corner_weights`; the offset's whole
    cells q shift the anchor (r = q = 0 without an offset)."""
    mesh_shape = conf.mesh_shape if mesh_shape is None else mesh_shape
    ft = conf.float_dtype.type
    q, r = offset_shift(offset, conf.cell_size, conf.float_dtype)
    d = (disp.astype(conf.float_dtype) - r) / ft(conf.cell_size)
    fl = np.floor(d)
    cell = (pmid.astype(np.int64) - q + fl.astype(np.int64)) % np.array(mesh_shape)
    return cell, d, fl


def corner_weights(d, fl, dtype):
    """Per-corner weights (N,8) and weight gradients (N,8,3), enmesh.py:149-162.

    delta = d - (floor(d) + b); w_axis = 1 - |delta|;
    w = (w0*w1)*w2; grad_i = sign(-delta_i) * w_{i+1} * w_{i+2}."""
    ft = np.dtype(dtype).type
    w = np.empty((d.shape[0], 8), dtype=dtype)
    g = np.empty((d.shape[0], 8, 3), dtype=dtype)
    for c in range(8):
        b = NEIGHBORS[c]
        delta = (d - (fl + b.astype(dtype))).astype(dtype)
        wa = (ft(1) - np.abs(delta)).astype(dtype)
        sg = np.where(delta < 0, ft(1), np.where(delta > 0, ft(-1), ft(0))).astype(dtype)
        w[:, c] = (wa[:, 0] * wa[:, 1]) * wa[:, 2]
        for i in range(3):
            g[:, c, i] = (sg[:, i] * wa[:, (i + 1) % 3]) * wa[:, (i + 2) % 3]
    return w, g


def corner_index(cell, mesh_shape):
    """Raveled indices of the 8 corners (N,8)."""
    M = np.array(mesh_shape)
    idx = np.empty((cell.shape[0], 8), dtype=np.int64)
    for c in range(8):
        cc = (cell + NEIGHBORS[c]) % M
        idx[:, c] = (cc[:, 0] * M[1] + cc[:, 1]) * M[2] + cc[:, 2]
    return idx


def _fmod_floor(x, y):
    r = np.fmod(x, y)
    return np.where((r != 0) & ((r < 0) != (y < 0)), r + y, r).astype(x.dtype)


def explicit_corners(pmid, disp, conf, offset, cell2, mesh_shape):
    """CIC onto a mesh of cell size cell2 (the explicit cell_size branch,
    cic/pallas.py:192-222, cic/enmesh.py:108-127), in the float dtype: per
    axis p = mod((pmid a1 + disp) - o, L a1); for bit b, i_b = floor(mod(p +
    b a2, L a1) / a2), delta = p - i_b a2 folded into the half period; weight
    1 - |delta / a2|.  Returns idx (N,8) with -1 for corners outside the
    target mesh, w (N,8) and the weight gradients g (N,8,3) (before / a2)."""
    dt = conf.float_dtype
    ft = dt.type
    a1, a2 = ft(conf.cell_size), ft(cell2)
    o = np.broadcast_to(np.asarray(offset, dtype=dt), (3, ))
    n = pmid.shape[0]
    ia, wa, sa = np.empty((n, 3, 2), np.int64), np.empty((n, 3, 2), dt), np.empty((n, 3, 2), dt)
    for ax in range(3):
        period = (ft(conf.mesh_shape[ax]) * a1).astype(dt)
        p = ((pmid[:, ax].astype(dt) * a1).astype(dt) + disp[:, ax].astype(dt)).astype(dt)
        p = _fmod_floor((p - o[ax]).astype(dt), period)
        for b in range(2):
            npos = _fmod_floor((p + ft(b) * a2).astype(dt), period)
            i = np.floor((npos / a2).astype(dt)).astype(np.int64)
            delta = (p - (i.astype(dt) * a2).astype(dt)).astype(dt)
            half = (ft(0.5) * period).astype(dt)
            delta = np.where(delta > half, delta - period, delta).astype(dt)
            delta = np.where(delta < -half, delta + period, delta).astype(dt)
            q = (delta / a2).astype(dt)
            wa[:, ax, b] = (ft(1) - np.abs(q)).astype(dt)
            sa[:, ax, b] = np.where(q < 0, ft(1), np.where(q > 0, ft(-1), ft(0)))
            ia[:, ax, b] = np.where((i >= 0) & (i < mesh_shape[ax]), i, -1)
    idx = np.empty((n, 8), np.int64)
    w = np.empty((n, 8), dt)
    g = np.empty((n, 8, 3), dt)
    for c in range(8):
        b = NEIGHBORS[c]
        ix, iy, iz = ia[:, 0, b[0]], ia[:, 1, b[1]], ia[:, 2, b[2]]
        wx, wy, wz = wa[:, 0, b[0]], wa[:, 1, b[1]], wa[:, 2, b[2]]
        sx, sy, sz = sa[:, 0, b[0]], sa[:, 1, b[1]], sa[:, 2, b[2]]
        ok = (ix >= 0) & (iy >= 0) & (iz >= 0)
        idx[:, c] = np.where(ok, (ix * mesh_shape[1] + iy) * mesh_shape[2] + iz, -1)
        w[:, c] = (wx * wy) * wz
        g[:, c, 0] = (sx * wy) * wz
        g[:, c, 1] = (sy * wz) * wx
        g[:, c, 2] = (sz * wx) * wy
    return idx, w, g


def corners(pmid, disp, conf, mesh_shape, offset=0, cell_size=None, valid=None):
    """Raveled corner indices (N,8; -1 = dropped), weights, weight gradients and
    the cell size the gradients divide by, for either grid path; particles with
    valid == False drop every corner (cic/pallas.py:133-141)."""
    if cell_size is None:
        cell, d, fl = enmesh(pmid, disp, conf, mesh_shape, offset)
        w, g = corner_weights(d, fl, conf.float_dtype)
        idx, a = corner_index(cell, mesh_shape), conf.cell_size
    else:
        idx, w, g = explicit_corners(pmid, disp, conf, offset, cell_size, mesh_shape)
        a = cell_size
    if valid is not None:
        idx = np.where(np.asarray(valid, dtype=bool)[:, None], idx, -1)
    return idx, w, g, a


def _take(chan, idx):
    """chan[idx] with dropped corners (-1) reading 0."""
    return np.where(idx >= 0, chan[np.maximum(idx, 0)], 0.0)


def cell_key(pmid, disp, conf):
    """Raveled lower-corner cell key ((x*My)+y)*Mz+z (core/utils.py:292-326)."""
    cell, _, _ = enmesh(pmid, disp, conf)
    M = conf.mesh_shape
    return (cell[:, 0] * M[1] + cell[:, 1]) * M[2] + cell[:, 2]


def sort_by_cell(pmid, disp, conf):
    """Stable per-cell order: keys ascending, ties keep source order."""
    key = cell_key(pmid, disp, conf)
    perm = np.argsort(key, kind='stable')
    return key, perm


def default_val(conf):
    """scatter.py:259-265: mesh_size / ptcl_num per valid particle."""
    return conf.float_dtype.type(conf.mesh_size / conf.ptcl_num)


def scatter(pmid, disp, conf, val=None, mesh_shape=None, offset=0, cell_size=None, valid=None):
    """CIC deposit, cic/scatter.py:315-338.  val: scalar, (N,) or (N,C).

    Returns a float64 mesh (M...) or (C, M...) accumulated exactly in float64
    from float-dtype weights (the reference accumulates with unordered
    float atomics; the difference is below the dtype's rounding)."""
    mesh_shape = conf.mesh_shape if mesh_shape is None else mesh_shape
    kw = dict(offset=offset, cell_size=cell_size)
    nch = 1 if val is None or np.ndim(val) <= 1 else np.shape(val)[1]
    ranges = _chunks(pmid.shape[0], 8 * math.prod(mesh_shape) * nch)
    if ranges is not None:
        # threaded: partial meshes of particle chunks, summed in chunk order
        if val is None:
            val = default_val(conf)
        return _psum(lambda lo, hi: _scatter1(pmid[lo:hi], disp[lo:hi], conf, _rows(val, lo, hi), mesh_shape,
                                              valid=_rows(valid, lo, hi), **kw), ranges)
    return _scatter1(pmid, disp, conf, val, mesh_shape, valid=valid, **kw)


def _scatter1(pmid, disp, conf, val, mesh_shape, offset=0, cell_size=None, valid=None):
    idx, w, _, _ = corners(pmid, disp, conf, mesh_shape, offset, cell_size, valid)
    keep = idx >= 0
    M = math.prod(mesh_shape)
    if val is None:
        val = default_val(conf)
    val = np.asarray(val, dtype=conf.float_dtype)
    if val.ndim <= 1:
        vw = (val[:, None] if val.ndim == 1 else val) * w
        vw = np.broadcast_to(vw, idx.shape)
        out = np.bincount(idx[keep], weights=vw[keep].astype(np.float64), minlength=M)
        return out.reshape(mesh_shape)
    outs = []
    for c in range(val.shape[1]):
        vw = val[:, c, None] * w
        outs.append(np.bincount(idx[keep], weights=vw[keep].astype(np.float64), minlength=M).reshape(mesh_shape))
    return np.stack(outs)


def gather(pmid, disp, conf, mesh, offset=0, cell_size=None, valid=None):
    """CIC interpolation, cic/gather.py:452-472.  mesh: (M...) or (C, M...)."""
    kw = dict(offset=offset, cell_size=cell_size)
    ranges = _chunks(pmid.shape[0])
    if ranges is not None:
        return np.concatenate(_pmap(lambda lo, hi: _gather1(pmid[lo:hi], disp[lo:hi], conf, mesh,
                                                            valid=_rows(valid, lo, hi), **kw), ranges))
    return _gather1(pmid, disp, conf, mesh, valid=valid, **kw)


def _gather1(pmid, disp, conf, mesh, offset=0, cell_size=None, valid=None):
    mesh_shape = mesh.shape[-3:]
    idx, w, _, _ = corners(pmid, disp, conf, mesh_shape, offset, cell_size, valid)
    chans = mesh.reshape(-1, math.prod(mesh_shape)) if mesh.ndim == 4 else mesh.reshape(1, -1)
    out = np.empty((pmid.shape[0], chans.shape[0]), dtype=np.float64)
    for c in range(chans.shape[0]):
        out[:, c] = (_take(chans[c], idx) * w).sum(axis=1)
    return out if mesh.ndim == 4 else out[:, 0]


def scatter_vjp(pmid, disp, conf, mesh_cot, val=None, offset=0, cell_size=None, valid=None):
    """cic/scatter.py:341-437: disp_cot = sum_b mesh_cot[i_b] val grad_b / cell,
    val_cot = sum_b mesh_cot[i_b] w_b (summed over particles for scalar val)."""
    kw = dict(offset=offset, cell_size=cell_size)
    ranges = _chunks(pmid.shape[0])
    if ranges is not None:
        parts = _pmap(lambda lo, hi: _scatter_vjp1(pmid[lo:hi], disp[lo:hi], conf, mesh_cot, _rows(val, lo, hi),
                                                   valid=_rows(valid, lo, hi), **kw), ranges)
        dc = np.concatenate([p[0] for p in parts])
        vcs = [p[1] for p in parts]
        return dc, (sum(vcs[1:], vcs[0]) if np.ndim(vcs[0]) == 0 else np.concatenate(vcs))
    return _scatter_vjp1(pmid, disp, conf, mesh_cot, val, valid=valid, **kw)


def _scatter_vjp1(pmid, disp, conf, mesh_cot, val, offset=0, cell_size=None, valid=None):
    mesh_shape = mesh_cot.shape[-3:]
    idx, w, g, a = corners(pmid, disp, conf, mesh_shape, offset, cell_size, valid)
    if val is None:
        val = default_val(conf)
    val = np.asarray(val, dtype=np.float64)
    chans = mesh_cot.reshape(-1, math.prod(mesh_shape)) if mesh_cot.ndim == 4 else mesh_cot.reshape(1, -1)
    vals = val.reshape(-1, 1) if val.ndim == 1 else (val if val.ndim == 2 else np.full((1, 1), float(val)))
    inner = np.zeros(idx.shape, dtype=np.float64)
    val_cot = np.zeros((pmid.shape[0], chans.shape[0]))
    for c in range(chans.shape[0]):
        mc = _take(chans[c], idx)
        inner += mc * vals[:, min(c, vals.shape[1] - 1)][:, None]
        val_cot[:, c] = (mc * w).sum(axis=1)
    disp_cot = (inner[..., None] * g).sum(axis=1) / a
    if val.ndim == 0:
        val_cot = val_cot.sum()
    elif val.ndim == 1:
        val_cot = val_cot[:, 0]
    return disp_cot, val_cot


def gather_vjp(pmid, disp, conf, mesh, val_cot, offset=0, cell_size=None, valid=None):
    """cic/gather.py:475-548: disp_cot = sum_b (sum_c val_cot mesh_c[i_b]) grad_b / cell,
    mesh_cot_c = scatter of val_cot_c w_b."""
    kw = dict(offset=offset, cell_size=cell_size)
    ranges = _chunks(pmid.shape[0], 8 * mesh.size)
    if ranges is not None:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(len(ranges)) as ex:
            it = ex.map(lambda r: _gather_vjp1(pmid[r[0]:r[1]], disp[r[0]:r[1]], conf, mesh, val_cot[r[0]:r[1]],
                                               valid=_rows(valid, r[0], r[1]), **kw), ranges)
            dcs, mesh_cot = [], None
            for dc, mc in it:  # chunk order; one running mesh total
                dcs.append(dc)
                mesh_cot = mc if mesh_cot is None else mesh_cot + mc
        return np.concatenate(dcs), mesh_cot
    return _gather_vjp1(pmid, disp, conf, mesh, val_cot, valid=valid, **kw)


def _gather_vjp1(pmid, disp, conf, mesh, val_cot, offset=0, cell_size=None, valid=None):
    mesh_shape = mesh.shape[-3:]
    idx, w, g, a = corners(pmid, disp, conf, mesh_shape, offset, cell_size, valid)
    keep = idx >= 0
    chans = mesh.reshape(-1, math.prod(mesh_shape)) if mesh.ndim == 4 else mesh.reshape(1, -1)
    vc = val_cot.reshape(pmid.shape[0], -1).astype(np.float64)
    inner = np.zeros(idx.shape, dtype=np.float64)
    M = math.prod(mesh_shape)
    mesh_cot = []
    for c in range(chans.shape[0]):
        inner += vc[:, c, None] * _take(chans[c], idx)
        wc = vc[:, c, None] * w
        mesh_cot.append(np.bincount(idx[keep], weights=wc[keep], minlength=M).reshape(mesh_shape))
    disp_cot = (inner[..., None] * g).sum(axis=1) / a
    mesh_cot = np.stack(mesh_cot) if mesh.ndim == 4 else mesh_cot[0]
    return disp_cot, mesh_cot


# --------------------------------------------------------------------------
# Spectral operators, nbody/gravity.py
# --------------------------------------------------------------------------
def k_squared(kvec, dtype):
    """gravity.py:74-119 (float-dtype sum of squares)."""
    kx, ky, kz = kvec
    return ((kx[:, None, None]**2 + ky[None, :, None]**2).astype(dtype) + kz[None, None, :]**2).astype(dtype)


def discrete_k_squared(kvec, cell, dtype):
    """gravity.py:122-171 (2 sin(k dx/2)/dx per axis)."""
    c = np.dtype(dtype).type(cell)
    ke = [(2 * np.sin(k * c / 2) / c).astype(dtype) for k in kvec]
    return k_squared(ke, dtype)


def green(conf, kernel="continuum", kvec=None):
    """Real Green's function G(k) with G=0 where k^2 == 0 (gravity.py:283-352)."""
    kvec = conf.kvec if kvec is None else kvec
    dt = conf.float_dtype
    k2 = k_squared(kvec, dt) if kernel == "continuum" else discrete_k_squared(kvec, conf.cell_size, dt)
    with np.errstate(divide='ignore'):
        return np.where(k2 != 0, -1.0 / k2.astype(np.float64), 0.0)


def nyquist_filter(conf):
    """Product of the per-axis particle-Nyquist masks (gravity.py:174-196)."""
    masks = conf.particle_nyquist_masks
    if not masks:
        return None
    return masks[0][:, None, None] * masks[1][None, :, None] * masks[2][None, None, :]


def window_gain(conf, alpha=0.48, max_gain=4.0, assignment_order=2, windows=2, taper_start=0.75, taper_stop=1.0):
    """CIC-window compensation transfer, corrections/window.py:229-265."""
    kx, ky, kz = [k.astype(np.float64) for k in conf.kvec]
    cell = conf.cell_size
    kn = np.pi / conf.ptcl_spacing
    sx = np.sinc(kx * cell / (2 * np.pi))[:, None, None]
    sy = np.sinc(ky * cell / (2 * np.pi))[None, :, None]
    sz = np.sinc(kz * cell / (2 * np.pi))[None, None, :]
    base = np.maximum(np.abs(sx * sy * sz), 1e-6)
    gain = base**(-(assignment_order * windows * alpha))
    if max_gain is not None and max_gain > 0:
        gain = np.minimum(gain, max_gain)
    if taper_stop > taper_start:
        q = np.maximum(np.maximum(np.abs(kx)[:, None, None], np.abs(ky)[None, :, None]), np.abs(kz)[None, None, :]) / kn
        t = np.clip((q - taper_start) / (taper_stop - taper_start), 0.0, 1.0)
        gain = 1.0 + (gain - 1.0) * (1.0 - t * t * (3.0 - 2.0 * t))
    return gain


def pgd_transfer(conf, a, alpha0=0.1, A=0.0, B=0.0, kl=0.1, ks=1.0):
    """1 - alpha(a) exp(-kl^2/k^2 - k^4/ks^4), 0 band at k = 0 (corrections/pgd.py:154-237)."""
    kx, ky, kz = [k.astype(np.float64) for k in conf.kvec]
    k2 = kx[:, None, None]**2 + ky[None, :, None]**2 + kz[None, None, :]**2
    safe = np.where(k2 > 0, k2, 1.0)
    band = np.where(k2 > 0, np.exp(-kl**2 / safe - safe**2 / ks**4), 0.0)
    return 1.0 - alpha0 * 10.0**(A * a**2 - B * a) * band


def softening_transfer(conf, strength=0.0, start=0.7, stop=1.0, mode="smoothstep"):
    """max(1 - strength taper(max_i |k_i| / k_Ny), 0) (corrections/softening.py:49-80)."""
    kn = np.pi / conf.ptcl_spacing
    ka = [np.abs(k.astype(np.float64)) / kn for k in conf.kvec]
    q = np.maximum(np.maximum(ka[0][:, None, None], ka[1][None, :, None]), ka[2][None, None, :])
    t = np.clip((q - start) / max(stop - start, 1e-6), 0.0, 1.0)
    taper = t * t * (3.0 - 2.0 * t) if mode == "smoothstep" else t
    return np.maximum(1.0 - strength * taper, 0.0)


def _gelu(x):
    """jax.nn.gelu (approximate=True)."""
    return 0.5 * x * (1.0 + np.tanh(np.sqrt(2.0 / np.pi) * (x + 0.044715 * x**3)))


def periodic_conv3d(x, w, b):
    """haiku Conv3D after periodic padding by one cell ('VALID'),
    corrections/mesh_cnn.py:54-64: x (Cin, nx, ny, nz), w (3, 3, 3, Cin, Cout)."""
    out = np.zeros((w.shape[4], ) + x.shape[1:])
    for kd in range(3):
        for kh in range(3):
            for kw in range(3):
                xs = np.roll(x, shift=(-(kd - 1), -(kh - 1), -(kw - 1)), axis=(1, 2, 3))
                out += np.einsum("cxyz,co->oxyz", xs, w[kd, kh, kw])
    return out + np.asarray(b)[:, None, None, None]


def mesh_cnn_residual(params, S, phi, a, omega_m, sigma8, depth=4, max_residual=0.1):
    """MeshResidualPotentialCorrection.__call__ (corrections/mesh_cnn.py:80-109)
    in float64: params maps haiku names to arrays."""
    P = {k: np.asarray(v, np.float64) for k, v in params.items()}
    sS = np.sqrt(np.mean(S**2) + 1e-6)
    sP = np.sqrt(np.mean(phi**2) + 1e-6)
    feat = np.array([a, omega_m, sigma8], np.float64)
    const = [np.full(S.shape, v) for v in feat]
    x = np.stack([S / sS, phi / sP] + const)
    h = _gelu(periodic_conv3d(x, P["stem/w"], P["stem/b"]))
    for i in range(max(depth - 1, 0)):
        r = h
        t = _gelu(periodic_conv3d(h, P[f"block_{i}_conv1/w"], P[f"block_{i}_conv1/b"]))
        h = _gelu(periodic_conv3d(t, P[f"block_{i}_conv2/w"], P[f"block_{i}_conv2/b"]) + r)
    o = periodic_conv3d(h, P["out/w"], P["out/b"])[0]
    conv_res = max_residual * np.tanh(o) * sP
    g = max_residual * np.tanh(feat @ P["direct_gain/w"][:, 0] + P["direct_gain/b"][0])
    return g * phi + conv_res


def force_meshes_cnn(rho, conf, Omega_m, params, a, sigma8, kernel=None, depth=4, max_residual=0.1):
    """force_meshes with the mesh-CNN residual added to the potential spectrum
    (corrections/core.py:321-331): pot += rfft(R(S, irfft(pot)))."""
    kernel = potential_kernel(conf) if kernel is None else kernel
    cs = conf.derivative_factors("spectral")
    om = float(np.float32(Omega_m)) if conf.float_dtype == np.float32 else float(Omega_m)
    S = (rho - 1.0) * (1.5 * om)
    pot = _fft.rfftn(S) * kernel
    phi = _fft.irfftn(pot, s=conf.mesh_shape)
    pot = pot + _fft.rfftn(mesh_cnn_residual(params, S, phi, a, om, sigma8, depth, max_residual))
    out = []
    for d in range(3):
        c = cs[d].astype(np.float64)
        shape = [1, 1, 1]
        shape[d] = -1
        out.append(_fft.irfftn(1j * c.reshape(shape) * pot, s=conf.mesh_shape))
    return np.stack(out)


def gravity_cnn(pmid, disp, conf, Omega_m, params, a, sigma8, kernel=None, depth=4, max_residual=0.1):
    """gravity() with a mesh-CNN correction (gravity.py:786-814 via
    _gravity_potential_from_density, :626-633)."""
    rho = scatter(pmid, disp, conf)
    F = force_meshes_cnn(rho, conf, Omega_m, params, a, sigma8, kernel, depth, max_residual)
    return gather(pmid, disp, conf, F)


def potential_kernel(conf, green_kernel="continuum", transfer=None):
    """Real multiplier from density-hat to potential-hat: G * nyquist * transfer."""
    G = green(conf, green_kernel)
    nf = nyquist_filter(conf)
    if nf is not None:
        G = G * nf
    if transfer is not None:
        G = G * transfer
    return G


def interlacing_phase(conf):
    """exp(-i (kx + ky + kz) cell / 2) on the half spectrum (gravity.py:440-443)."""
    kx, ky, kz = [k.astype(np.float64) for k in conf.kvec]
    ksum = kx[:, None, None] + ky[None, :, None] + kz[None, None, :]
    return np.exp(-1j * ksum * (conf.cell_size / 2))


def interlaced_density(pmid, disp, conf, val=None):
    """The regular deposit and the one shifted by half a cell on every axis
    (gravity.py:446-463: scatter(..., offset=cell/2))."""
    return scatter(pmid, disp, conf, val), scatter(pmid, disp, conf, val, offset=conf.cell_size / 2)


def force_meshes(rho, conf, Omega_m, kernel=None, gradient="spectral", rho_shifted=None):
    """Density (M) -> 3 real force meshes, gravity.py:626-633 + 506-543;
    gradient "fastpm_4point" takes FastPM's derivative (gravity.py:355-391).
    With rho_shifted (the half-cell-shifted deposit) the source spectrum is the
    interlaced average 0.5 (rfft(S) + rfft(S_shifted) P) (gravity.py:446-463)."""
    kernel = potential_kernel(conf) if kernel is None else kernel
    cs = conf.derivative_factors(gradient)
    om = float(np.float32(Omega_m)) if conf.float_dtype == np.float32 else float(Omega_m)
    S = (rho - 1.0) * (1.5 * om)
    Sh = _fft.rfftn(S)
    if rho_shifted is not None:
        Sh = 0.5 * (Sh + _fft.rfftn((rho_shifted - 1.0) * (1.5 * om)) * interlacing_phase(conf))
    pot = Sh * kernel
    out = []
    for d in range(3):
        c = cs[d].astype(np.float64)
        shape = [1, 1, 1]
        shape[d] = -1
        out.append(_fft.irfftn(1j * c.reshape(shape) * pot, s=conf.mesh_shape))
    return np.stack(out)


def gravity(pmid, disp, conf, Omega_m, kernel=None, gradient="spectral", interlacing=False):
    """gravity(), gravity.py:786-814, uncorrected (or fixed real transfer);
    interlacing averages the regular and half-cell-shifted deposits
    (gravity.py:809-811, 446-463)."""
    if interlacing:
        rho, rho1 = interlaced_density(pmid, disp, conf)
    else:
        rho, rho1 = scatter(pmid, disp, conf), None
    F = force_meshes(rho, conf, Omega_m, kernel, gradient, rho1)
    return gather(pmid, disp, conf, F)


def gravity_vjp(pmid, disp, conf, Omega_m, acc_cot, kernel=None, val=None, gradient="spectral", interlacing=False):
    """Transpose of gravity w.r.t. disp and Omega_m.

    The map S -> A_d is the real convolution irfft(H_d rfft(S)) with
    H_d = i c_d K(k) Hermitian, so its transpose is irfft(conj(H_d) rfft(.)).
    With interlacing the shifted source enters through H_d P / 2 and the
    regular one through H_d / 2 (Hermitian wherever K is non-zero once the
    mesh Nyquist planes are masked), so their transposes are
    irfft(conj(P) conj(H_d) rfft(.)) / 2 and irfft(conj(H_d) rfft(.)) / 2.
    Returns (disp_cot, Omega_m_cot)."""
    kernel = potential_kernel(conf) if kernel is None else kernel
    om = float(np.float32(Omega_m)) if conf.float_dtype == np.float32 else float(Omega_m)
    if interlacing:
        rho, rho1 = interlaced_density(pmid, disp, conf, val)
    else:
        rho, rho1 = scatter(pmid, disp, conf, val), None
    F = force_meshes(rho, conf, Omega_m, kernel, gradient, rho1)
    dc_gather, A_cot = gather_vjp(pmid, disp, conf, F, acc_cot)
    cs = conf.derivative_factors(gradient)
    spec = 0
    for d in range(3):
        c = cs[d].astype(np.float64)
        shape = [1, 1, 1]
        shape[d] = -1
        spec = spec + (-1j) * c.reshape(shape) * _fft.rfftn(A_cot[d])
    spec = spec * kernel
    if rho1 is None:
        S_cot = _fft.irfftn(spec, s=conf.mesh_shape)
        dc_scatter, _ = scatter_vjp(pmid, disp, conf, S_cot * (1.5 * om), val)
        om_cot = 1.5 * float(((rho - 1.0) * S_cot).sum())
        return dc_gather + dc_scatter, om_cot
    S_cot = 0.5 * _fft.irfftn(spec, s=conf.mesh_shape)
    S1_cot = 0.5 * _fft.irfftn(spec * np.conj(interlacing_phase(conf)), s=conf.mesh_shape)
    dc0, _ = scatter_vjp(pmid, disp, conf, S_cot * (1.5 * om), val)
    dc1, _ = scatter_vjp(pmid, disp, conf, S1_cot * (1.5 * om), val, offset=conf.cell_size / 2)
    om_cot = 1.5 * float(((rho - 1.0) * S_cot).sum() + ((rho1 - 1.0) * S1_cot).sum())
    return dc_gather + dc0 + dc1, om_cot


# --------------------------------------------------------------------------
# Time integration, nbody/integrator.py
# --------------------------------------------------------------------------
def _G_D(a, cosmo, conf):
    """integrator.py:114-116."""
    return a**2 * np.sqrt(cos.E2(a, cosmo)) * cos.growth(a, cosmo, conf.growth_a, deriv=1)


def _G_K(a, cosmo, conf):
    """integrator.py:119-122."""
    ga = conf.growth_a
    return a**3 * cos.E2(a, cosmo) * (cos.growth(a, cosmo, ga, deriv=2) +
                                      (2 + cos.H_deriv(a, cosmo)) * cos.growth(a, cosmo, ga, deriv=1))


def drift_factor(a_vel, a_prev, a_next, cosmo, conf):
    """integrator.py:125-146."""
    return (cos.growth(a_next, cosmo, conf.growth_a) - cos.growth(a_prev, cosmo, conf.growth_a)) / _G_D(
        a_vel, cosmo, conf)


def kick_factor(a_acc, a_prev, a_next, cosmo, conf):
    """integrator.py:149-170."""
    return (_G_D(a_next, cosmo, conf) - _G_D(a_prev, cosmo, conf)) / _G_K(a_acc, cosmo, conf)


def stage_schedule(a_prev, a_next, conf):
    """integrator.py:689-778: ('drift', a_vel, a_prev, a_next, a_acc_in) / ('kick', a_acc, a_prev, a_next)."""
    D = K = 0
    a_disp = a_vel = a_acc = a_prev
    stages = []
    for d, k in conf.symp_splits:
        if d != 0:
            D += d
            a_disp_next = a_prev * (1 - D) + a_next * D
            stages.append(("drift", a_vel, a_disp, a_disp_next, a_acc))
            a_disp = a_disp_next
            a_acc = a_disp
        if k != 0:
            K += k
            a_vel_next = a_prev * (1 - K) + a_next * K
            stages.append(("kick", a_acc, a_vel, a_vel_next))
            a_vel = a_vel_next
    return stages


def nbody(pmid, disp, vel, conf, cosmo, kernel=None, acc=None, interlacing=False):
    """nbody/solver.py:253-273 forward (init force + scan of integrate)."""
    ft = conf.float_dtype
    a = conf.a_nbody
    K = kernel if callable(kernel) else (lambda _a: kernel)
    disp = disp.astype(ft).copy()
    vel = vel.astype(ft).copy()
    acc = gravity(pmid, disp, conf, cosmo.Omega_m, K(a[0]), interlacing=interlacing).astype(ft)
    for a_prev, a_next in zip(a[:-1], a[1:]):
        for st in stage_schedule(a_prev, a_next, conf):
            if st[0] == "drift":
                f = ft.type(drift_factor(st[1], st[2], st[3], cosmo, conf))
                disp = (disp + vel * f).astype(ft)
                acc = gravity(pmid, disp, conf, cosmo.Omega_m, K(st[3]), interlacing=interlacing).astype(ft)
            else:
                f = ft.type(kick_factor(st[1], st[2], st[3], cosmo, conf))
                vel = (vel + acc * f).astype(ft)
    return disp, vel, acc


def _factor_dOm(fn, args, cosmo, conf, h=1e-4):
    """d factor / d Omega_m by a central difference of the FP64 host tables.

    h = 1e-4 keeps the adaptive-step noise (~1e-10 in the tables) well below
    the O(h^2) truncation error."""
    vals = []
    for s in (+1, -1):
        c = cosmo.replace(Omega_m=cosmo.Omega_m + s * h)
        c.growth = cos.growth_integ(c, conf.growth_a, conf.a_lpt_step)
        vals.append(fn(*args, c, conf))
    return (vals[0] - vals[1]) / (2 * h)


def nbody_adj(pmid, disp, vel, acc, disp_cot, vel_cot, acc_cot, conf, cosmo, kernel=None, om_grads=True,
              interlacing=False, om_terms=None):
    """Reverse sweep, nbody/solver.py:385-444 + integrator.py:541-582, 429-509,
    620-686, 781-837.  States are rebuilt algebraically (disp -= vel*D,
    vel -= acc*K) and the force at the earlier time is recomputed.

    Returns (disp, vel, disp_cot, vel_cot, Omega_m_cot) at the initial time;
    om_terms (a list) receives every term of the Omega_m cotangent's sum (the
    sum can cancel to far below its terms).  A callable kernel is evaluated
    at the scale factor of the positions each force sees, as force_adj(a, ...)
    does (integrator.py:620-686)."""
    om_terms = [] if om_terms is None else om_terms
    ft = conf.float_dtype
    a = conf.a_nbody
    K = kernel if callable(kernel) else (lambda _a: kernel)
    disp, vel, acc = disp.astype(ft).copy(), vel.astype(ft).copy(), acc.astype(ft).copy()
    dc = disp_cot.astype(np.float64).copy()
    vc = vel_cot.astype(np.float64).copy()
    ac = acc_cot.astype(np.float64).copy()
    om_cot = 0.0
    for a_prev, a_next in zip(a[:-1][::-1], a[1:][::-1]):
        for st in reversed(stage_schedule(a_prev, a_next, conf)):
            if st[0] == "kick":
                f64 = kick_factor(st[1], st[2], st[3], cosmo, conf)
                f = ft.type(f64)
                vel = (vel - acc * f).astype(ft)
                ac = ac + vc * float(f)
                if om_grads:
                    om_terms.append(_factor_dOm(kick_factor, st[1:], cosmo, conf) * float((vc * acc).sum()))
                    om_cot += om_terms[-1]
                continue
            _, a_vel, a_dp, a_dn, a_acc_in = st
            g, oc = gravity_vjp(pmid, disp, conf, cosmo.Omega_m, ac, K(a_dn), interlacing=interlacing)
            dc = dc + g
            om_cot += oc
            om_terms.append(oc)
            ac = np.zeros_like(ac)
            f64 = drift_factor(a_vel, a_dp, a_dn, cosmo, conf)
            f = ft.type(f64)
            disp = (disp - vel * f).astype(ft)
            vc = vc + dc * float(f)
            if om_grads:
                om_terms.append(_factor_dOm(drift_factor, (a_vel, a_dp, a_dn), cosmo, conf) * float((dc * vel).sum()))
                om_cot += om_terms[-1]
            acc = gravity(pmid, disp, conf, cosmo.Omega_m, K(a_dp), interlacing=interlacing).astype(ft)
    g, oc = gravity_vjp(pmid, disp, conf, cosmo.Omega_m, ac, K(a[0]), interlacing=interlacing)
    dc = dc + g
    om_cot += oc
    om_terms.append(oc)
    return disp, vel, dc, vc, om_cot


# --------------------------------------------------------------------------
# Initial conditions
# --------------------------------------------------------------------------
def _mix32(x):
    """lowbias32 finaliser, initial_conditions/modes.py:92-111."""
    x = np.array(x, dtype=np.uint32, ndmin=1)
    with np.errstate(over='ignore'):
        x = x ^ (x >> np.uint32(16))
        x = x * np.uint32(0x7FEB352D)
        x = x ^ (x >> np.uint32(15))
        x = x * np.uint32(0x846CA68B)
        x = x ^ (x >> np.uint32(16))
    return x


def hash_mode(seed, kx, ky, kz, salt):
    """modes.py:114-129 (kx, ky, kz wrap to uint32)."""
    u = lambda v: np.asarray(v).astype(np.int64).astype(np.uint32)
    h = _mix32(np.uint32(seed & 0xFFFFFFFF) ^ np.uint32(salt))
    h = _mix32(h ^ _mix32((u(kx) + np.uint32(0x9E3779B9)).astype(np.uint32)))
    h = _mix32(h ^ _mix32((u(ky) + np.uint32(0x85EBCA6B)).astype(np.uint32)))
    h = _mix32(h ^ _mix32((u(kz) + np.uint32(0xC2B2AE35)).astype(np.uint32)))
    return h


def _self_inverse(k, size):
    m = k == 0
    if size % 2 == 0:
        m = m | (k == -(size // 2))
    return m


def white_noise_nested(seed, conf, dtype=None):
    """Hermitian-consistent hashed Gaussian modes, modes.py:75-268."""
    dtype = conf.float_dtype if dtype is None else np.dtype(dtype)
    ft = dtype.type
    n0, n1, n2 = conf.ptcl_grid_shape
    mode = lambda n: np.where(np.arange(n) < (n + 1) // 2, np.arange(n), np.arange(n) - n)
    kx = mode(n0)[:, None, None]
    ky = mode(n1)[None, :, None]
    kz = np.arange(n2 // 2 + 1)[None, None, :]
    plane = kz == 0
    if n2 % 2 == 0:
        plane = plane | (kz == n2 // 2)
    px = np.where(_self_inverse(kx, n0), kx, -kx)
    py = np.where(_self_inverse(ky, n1), ky, -ky)
    keep = (kx < px) | ((kx == px) & (ky <= py))
    rx = np.where(keep, kx, px)
    ry = np.where(keep, ky, py)
    self_point = _self_inverse(kx, n0) & _self_inverse(ky, n1)
    hx = np.where(plane, rx, kx)
    hy = np.where(plane, ry, ky)
    hx, hy, hz = np.broadcast_arrays(hx, hy, kz)
    hr = hash_mode(seed, hx, hy, hz, 0xA24BAED4)
    hi = hash_mode(seed, hx, hy, hz, 0x9FB21C65)
    scale = ft(2.3283064365386963e-10)
    u1 = (hr.astype(dtype) + ft(0.5)) * scale
    u2 = (hi.astype(dtype) + ft(0.5)) * scale
    r = np.sqrt(ft(-2.0) * np.log(u1)).astype(dtype)
    th = (ft(2 * np.pi) * u2).astype(dtype)
    gr = (r * np.cos(th)).astype(dtype)
    gi = (r * np.sin(th)).astype(dtype)
    sq = ft(0.7071067811865476)
    coeff = (gr * sq) + 1j * (gi * sq)
    selfc = np.where(self_point, gr + 0j, coeff)
    need_conj = ~keep
    plane_c = np.where(need_conj, np.conj(selfc), selfc)
    out = np.where(plane, plane_c, coeff)
    return out.astype(np.complex64 if dtype == np.float32 else np.complex128)


def linear_modes(modes, cosmo, conf, a=None):
    """delta(k) = omega(k) sqrt(V P_lin(k)), modes.py:397-454 (Fourier input)."""
    kx, ky, kz = conf.kvec_spacing
    dt = conf.float_dtype
    k = np.sqrt(k_squared((kx, ky, kz), dt)).astype(dt)
    P = cos.linear_power(k.astype(np.float64), a, cosmo, conf.transfer_k, growth_a=conf.growth_a).astype(dt)
    amp = np.sqrt((P * dt.type(conf.box_vol)).astype(dt)).astype(dt)
    return modes * amp


def _strain_ops(conf):
    """-k_i k_j multipliers on the particle grid, lpt.py:17-43."""
    ks = conf.kvec_spacing
    dt = conf.float_dtype
    nyq = np.pi / conf.ptcl_spacing
    eps = nyq * np.finfo(dt).eps
    kz_ = [k.astype(np.float64) for k in ks]
    kzero = [np.where(np.abs(np.abs(k) - nyq) <= eps, 0.0, k) for k in kz_]
    shp = lambda i: tuple(-1 if j == i else 1 for j in range(3))
    ops = {}
    for i in range(3):
        for j in range(i, 3):
            if i == j:
                ops[(i, j)] = -(kz_[i].reshape(shp(i))**2)
            else:
                ops[(i, j)] = -(kzero[i].reshape(shp(i)) * kzero[j].reshape(shp(j)))
    return ops


def lpt_source(pot_m, conf, pot_n=None):
    """Quadratic LPT source, lpt.py:239-301:
    sum_{i<j} phi_ii psi_jj (symmetrised when pot_n is given) - phi_ij psi_ji."""
    shape = conf.ptcl_grid_shape
    ops = _strain_ops(conf)
    same = pot_n is None
    pot_n = pot_m if same else pot_n
    dm = [np.fft.irfftn(ops[(i, i)] * pot_m, s=shape) for i in range(3)]
    dn = dm if same else [np.fft.irfftn(ops[(i, i)] * pot_n, s=shape) for i in range(3)]
    L = np.zeros(shape)
    for i in range(3):
        for j in range(2, i, -1):
            L += dm[i] * dn[j]
        if not same:
            for j in range(i - 1, -1, -1):
                L += dm[i] * dn[j]
    if not same:
        L *= 0.5
    for i in range(2):
        for j in range(i + 1, 3):
            sm = np.fft.irfftn(ops[(i, j)] * pot_m, s=shape)
            sn = sm if same else np.fft.irfftn(ops[(i, j)] * pot_n, s=shape)
            L -= sm * sn
    return L


def lpt_fields(modes, cosmo, conf):
    """1LPT/2LPT gradient fields on the particle grid, lpt.py:239-449.

    Returns (g1, g2), each (3, N) float64: -grad phi_m sampled per particle."""
    shape = conf.ptcl_grid_shape
    G = green(conf, "continuum", conf.kvec_spacing)
    pot1 = modes.astype(np.complex128) / conf.ptcl_cell_vol * G
    L = lpt_source(pot1, conf)
    pot2 = np.fft.rfftn(L) * G
    c = [np.where(np.abs(np.abs(k.astype(np.float64)) - np.pi / conf.ptcl_spacing) <= np.pi / conf.ptcl_spacing *
                  np.finfo(conf.float_dtype).eps, 0.0, -k.astype(np.float64)) for k in conf.kvec_spacing]
    out = []
    for pot in (pot1, pot2):
        g = []
        for d in range(3):
            shp = tuple(-1 if j == d else 1 for j in range(3))
            g.append(np.fft.irfftn(1j * c[d].reshape(shp) * pot, s=shape).reshape(-1))
        out.append(np.stack(g))
    return out


def lpt_factors(cosmo, conf):
    """(D_m, a^2 H dD_m/dlna) at a_start for m = 1, 2, lpt.py:412-417."""
    a = conf.a_start
    out = []
    for order in (1, 2):
        D = cos.growth(a, cosmo, conf.growth_a, order=order)
        dD = cos.growth(a, cosmo, conf.growth_a, order=order, deriv=1)
        out.append((float(D), float(a**2 * np.sqrt(cos.E2(a, cosmo)) * dD)))
    return out


def lpt(modes, cosmo, conf):
    """lpt(), lpt.py:337-449 on the gen_grid lattice.  Returns (pmid, disp, vel)."""
    pmid, disp = gen_grid(conf)
    ft = conf.float_dtype
    vel = np.zeros_like(disp)
    g = lpt_fields(modes, cosmo, conf)
    facs = lpt_factors(cosmo, conf)
    for order in range(conf.lpt_order):
        D, V = facs[order]
        for i in range(3):
            gi = g[order][i].astype(ft)
            disp[:, i] = (disp[:, i] + ft.type(D) * gi).astype(ft)
            vel[:, i] = (vel[:, i] + ft.type(V) * gi).astype(ft)
    return pmid, disp, vel


# --------------------------------------------------------------------------
# Power spectrum, analysis/power_spectrum.py
# --------------------------------------------------------------------------
def shell_statistics(mesh_shape, cell_size):
    """power_spectrum.py:46-74: shell k centres and mode counts (shells >= 1)."""
    mx = np.fft.fftfreq(mesh_shape[0]) * mesh_shape[0]
    my = np.fft.fftfreq(mesh_shape[1]) * mesh_shape[1]
    mz = np.fft.rfftfreq(mesh_shape[2]) * mesh_shape[2]
    X, Y, Z = np.meshgrid(mx, my, mz, indexing="ij")
    mag = np.sqrt(X**2 + Y**2 + Z**2)
    shell = np.floor(mag + 1e-6).astype(np.int64)
    mult = np.full(shell.shape, 2)
    mult[..., 0] = 1
    if mesh_shape[2] % 2 == 0:
        mult[..., -1] = 1
    n = int(shell.max()) + 1
    nmodes = np.bincount(shell.ravel(), weights=mult.ravel(), minlength=n).astype(np.int64)
    ksum = np.bincount(shell.ravel(), weights=(mag * mult).ravel(), minlength=n)
    k = ksum / np.maximum(nmodes, 1) * (2 * np.pi / (mesh_shape[0] * cell_size))
    return k[1:], nmodes[1:]


def shell_sums(spec, mesh_shape, mas_power=2, dtype=np.float64):
    """power_spectrum.py:120-143: sum |d|^2 * mult * sinc^(-2p) per integer shell."""
    mx = np.fft.fftfreq(mesh_shape[0]) * mesh_shape[0]
    my = np.fft.fftfreq(mesh_shape[1]) * mesh_shape[1]
    mz = np.arange(mesh_shape[2] // 2 + 1)
    num_shells = math.floor(math.sqrt(3) * (mesh_shape[0] // 2)) + 1
    sq = (mx[:, None, None].astype(np.int64)**2 + my[None, :, None].astype(np.int64)**2 + mz[None, None, :]**2)
    shell = np.clip(np.floor(np.sqrt(sq.astype(np.float64)) + 1e-9).astype(np.int64), 0, num_shells - 1)
    mult = np.full(spec.shape, 2.0)
    mult[..., 0] = 1
    if mesh_shape[2] % 2 == 0:
        mult[..., -1] = 1
    power = (spec.real**2 + spec.imag**2)
    if mas_power > 0:
        w = (np.sinc(mx / mesh_shape[0])[:, None, None] * np.sinc(my / mesh_shape[1])[None, :, None] *
             np.sinc(mz / mesh_shape[2])[None, None, :])
        power = power * w**(-2 * mas_power)
    return np.bincount(shell.ravel(), weights=(power * mult).ravel(), minlength=num_shells), shell, mult


def delta_to_pk(delta, conf, mas_power=2):
    """power_spectrum.py:277-305.  Returns (k, P, nmodes) over shells 1..n-1."""
    spec = np.fft.rfftn(delta)
    psum, _, _ = shell_sums(spec, conf.mesh_shape, mas_power)
    k, nmodes = shell_statistics(conf.mesh_shape, conf.cell_size)
    nsh = len(psum) - 1
    k, nmodes = k[:nsh], nmodes[:nsh]
    pk = psum[1:] / nmodes * (conf.cell_size**3 / conf.mesh_size)
    return k, pk, nmodes


def density_to_pk(density, conf, mas_power=2):
    """power_spectrum.py:348-374."""
    return delta_to_pk(density / density.mean() - 1, conf, mas_power)


def delta_to_cross_correlation(da, db, conf, mas_power=2, eps=1e-30):
    """power_spectrum.py:146-176, 259-267, 308-345: (k, r, P_ab, P_aa, P_bb, nmodes)."""
    sa, sb = np.fft.rfftn(da), np.fft.rfftn(db)
    k, pa, n = delta_to_pk(da, conf, mas_power)
    _, pb, _ = delta_to_pk(db, conf, mas_power)
    cross = (sa * np.conj(sb)).real
    mx = np.fft.fftfreq(conf.mesh_shape[0]) * conf.mesh_shape[0]
    my = np.fft.fftfreq(conf.mesh_shape[1]) * conf.mesh_shape[1]
    mz = np.arange(conf.mesh_shape[2] // 2 + 1)
    _, shell, mult = shell_sums(sa, conf.mesh_shape, mas_power)
    w = (np.sinc(mx / conf.mesh_shape[0])[:, None, None] * np.sinc(my / conf.mesh_shape[1])[None, :, None] *
         np.sinc(mz / conf.mesh_shape[2])[None, None, :])**(-2 * mas_power)
    xs = np.bincount(shell.ravel(), weights=(cross * w * mult).ravel(), minlength=len(pa) + 1)
    px = xs[1:len(pa) + 1] / n * (conf.cell_size**3 / conf.mesh_size)
    r = px / np.sqrt(np.maximum(pa * pb, eps))
    return k, r, px, pa, pb, n


# --------------------------------------------------------------------------
# Learned Green's-function correction (test reference for csrc/mlp.cu)
# --------------------------------------------------------------------------
def bf16_round(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def mlp_unpack(w, b, H=64):
    w = np.asarray(w, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    W1 = w[:4 * H].reshape(H, 4)
    W2 = w[4 * H:4 * H + H * H].reshape(H, H)
    W3 = w[4 * H + H * H:4 * H + 2 * H * H].reshape(H, H)
    W4 = w[4 * H + 2 * H * H:]
    return W1, W2, W3, W4, b[:H], b[H:2 * H], b[2 * H:3 * H], b[3 * H]


def mlp_table(w, b, kscale, a, om, s8, length):
    """T[n2] = 1 + f(sqrt(n2) kscale, a, Om, s8), T[0] = 1 (width-64 sin-MLP)."""
    W1, W2, W3, W4, b1, b2, b3, b4 = mlp_unpack(w, b)
    n2 = np.arange(length, dtype=np.float64)
    x = np.stack([np.sqrt(n2) * kscale, np.full_like(n2, a), np.full_like(n2, om), np.full_like(n2, s8)], 1)
    h = np.sin(x @ W1.T + b1)
    h = np.sin(h @ W2.T + b2)
    h = np.sin(h @ W3.T + b3)
    T = 1.0 + h @ W4 + b4
    T[0] = 1.0
    return T


def radial_transfer(table, conf):
    """Expand a |n|^2-indexed table onto the half spectrum (cubic mesh)."""
    mx = np.fft.fftfreq(conf.mesh_shape[0]) * conf.mesh_shape[0]
    my = np.fft.fftfreq(conf.mesh_shape[1]) * conf.mesh_shape[1]
    mz = np.arange(conf.mesh_shape[2] // 2 + 1)
    n2 = (mx[:, None, None]**2 + my[None, :, None]**2 + mz[None, None, :]**2).astype(np.int64)
    return np.asarray(table)[n2]


def log_bins(k, pk, nmodes, nbins=32, kmin=None, kmax=None):
    """Mode-count-weighted rebinning of integer shells into log-spaced bins.

    An extension, not reference behaviour: the reference only reports
    integer-radius shells."""
    kmin = k[0] if kmin is None else kmin
    kmax = k[-1] * (1 + 1e-9) if kmax is None else kmax
    edges = np.geomspace(kmin, kmax, nbins + 1)
    b = np.clip(np.searchsorted(edges, k, side='right') - 1, 0, nbins - 1)
    w = np.bincount(b, weights=nmodes, minlength=nbins)
    kb = np.bincount(b, weights=k * nmodes, minlength=nbins) / np.maximum(w, 1)
    pb = np.bincount(b, weights=pk * nmodes, minlength=nbins) / np.maximum(w, 1)
    return kb, pb, w
