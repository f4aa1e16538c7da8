"""Run configuration (the fields of PM++'s ``Configuration`` the PM path reads).

Mirrors core/configuration.py:172-575: geometry (ptcl_spacing,
ptcl_grid_shape, mesh_shape as a scale or a shape), time schedules (a_start,
a_stop, a_custom, symp_splits), LPT order, growth-ODE tolerances and the
transfer-function k grid.  The cached spectral operators (kvec, the
Nyquist-zeroed derivative factors and the particle-Nyquist masks) are built
here once with the reference formulas and uploaded as one device table.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _fftfreq(shape, spacing, dtype=np.float32):
    """Angular wavevectors per axis (numerics/fft.py:4-44) in the working precision."""
    period = 2 * np.pi / spacing
    ks = [(np.fft.fftfreq(s) * period).astype(dtype) for s in shape[:-1]]
    ks.append((np.fft.rfftfreq(shape[-1]) * period).astype(dtype))
    return ks


class Configuration:
    """PM configuration; see core/configuration.py:22-243 for field meanings."""

    # SI constants and the code units [L] = Mpc/h, [T] = 1/H_0, [M] = 1e10 Msun/h
    # (configuration.py:198-209; the values must agree for the time factors)
    M_sun_SI = 1.98847e30
    Mpc_SI = 3.0856775815e22
    H_0_SI = 1e5 / Mpc_SI
    c_SI = 299792458
    G_SI = 6.67430e-11
    M = 1e10 * M_sun_SI
    L = Mpc_SI
    T = 1 / H_0_SI
    # the reference's multi-GPU attributes at their single-device values
    use_mGPU = False
    mesh_halo_width = 0
    ptcl_halo_width = 0

    def __init__(self, ptcl_spacing, ptcl_grid_shape, mesh_shape=1, *, a_start=1 / 64, a_stop=1.0,
                 a_lpt_maxstep=1 / 128, a_nbody_maxstep=1 / 64, a_custom=None, growth_a_custom=None,
                 symp_splits=((0, 0.5), (1, 0.5)), lpt_order=2, growth_rtol=None, growth_atol=None,
                 growth_inistep=(1, None), transfer_fit=True, transfer_fit_nowiggle=False, transfer_lgk_min=-4,
                 transfer_lgk_max=3, transfer_lgk_maxstep=1 / 128, T_cmb=2.7255, k_pivot_Mpc=0.05,
                 float_dtype="float32", device=None, to_save_z=None, to_save_a=None, slice_to_save=None,
                 max_slice_width=None):
        self.ptcl_spacing = float(ptcl_spacing)
        self.ptcl_grid_shape = tuple(int(s) for s in ptcl_grid_shape)
        if isinstance(mesh_shape, (int, float)):
            mesh_shape = tuple(round(s * mesh_shape) for s in self.ptcl_grid_shape)
        self.mesh_shape = tuple(int(s) for s in mesh_shape)
        if len(self.ptcl_grid_shape) != len(self.mesh_shape):
            raise ValueError('particle and mesh grid dimensions differ')
        if len(self.ptcl_grid_shape) != 3:
            raise ValueError("only three spatial dimensions are supported")
        if any(sm < sp for sp, sm in zip(self.ptcl_grid_shape, self.mesh_shape)):
            raise ValueError('mesh grid cannot be smaller than particle grid')
        if any(self.ptcl_grid_shape[0] * sm != self.mesh_shape[0] * sp
               for sp, sm in zip(self.ptcl_grid_shape[1:], self.mesh_shape[1:])):
            raise ValueError('particle and mesh grid aspect ratios differ')
        name = str(np.dtype(str(float_dtype).replace("torch.", "")))
        if name not in ("float32", "float64"):
            raise NotImplementedError("float32 (optimised kernels) and float64 (x64 build) are supported")
        # float32: the optimised kernels; float64: the x64 build (forward path only)
        self.float_dtype = torch.float32 if name == "float32" else torch.float64
        self.np_dtype = np.dtype(name)
        self.a_start = float(a_start)
        self.a_stop = float(a_stop)
        self.a_lpt_maxstep = a_lpt_maxstep
        self.a_nbody_maxstep = a_nbody_maxstep
        self.a_custom = None if a_custom is None else tuple(float(a) for a in np.asarray(a_custom).tolist())
        self.growth_a_custom = (None if growth_a_custom is None else
                                tuple(float(a) for a in np.asarray(growth_a_custom).tolist()))
        if any(len(s) != 2 for s in symp_splits):
            raise ValueError(f'symp_splits={symp_splits} not supported')
        if tuple(sum(s) for s in zip(*symp_splits)) != (1, 1):
            raise ValueError('sum of symplectic splits != (1, 1)')
        self.symp_splits = tuple(tuple(s) for s in symp_splits)
        if lpt_order not in (0, 1, 2):
            raise ValueError(f'lpt_order={lpt_order} not supported')
        self.lpt_order = lpt_order
        tol = math.sqrt(np.finfo(np.float64).eps)
        self.growth_rtol = tol if growth_rtol is None else growth_rtol
        self.growth_atol = tol if growth_atol is None else growth_atol
        self.growth_inistep = growth_inistep
        if not transfer_fit:
            raise NotImplementedError('only the Eisenstein-Hu transfer fit is available')
        self.transfer_fit_nowiggle = bool(transfer_fit_nowiggle)
        self.transfer_lgk_min = transfer_lgk_min
        self.transfer_lgk_max = transfer_lgk_max
        self.transfer_lgk_maxstep = transfer_lgk_maxstep
        self.T_cmb = T_cmb
        self.k_pivot_Mpc = k_pivot_Mpc
        self.device = torch.device(device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu"))
        # saved-map controls of the forward observers (configuration.py:235-238, 311-318)
        self.to_save_z = None if to_save_z is None else list(to_save_z)
        if to_save_a is None and to_save_z is not None:
            to_save_a = [1 / (1 + z) for z in to_save_z]
        self.to_save_a = None if to_save_a is None else list(to_save_a)
        self.slice_to_save = None if slice_to_save is None else [int(i) for i in slice_to_save]
        self.max_slice_width = None if max_slice_width is None else int(max_slice_width)
        # cached spectral operators (configuration.py:301-307, 365-376)
        self.kvec = _fftfreq(self.mesh_shape, self.cell_size, self.np_dtype)
        self.kvec_spacing = _fftfreq(self.ptcl_grid_shape, self.ptcl_spacing, self.np_dtype)
        self.neg_k = tuple(self._neg_k(k, self.cell_size) for k in self.kvec)
        self._tables = {}

    @staticmethod
    def _neg_k(k, spacing):
        f = k.dtype.type
        nyquist = f(np.pi / spacing)
        eps = nyquist * np.finfo(k.dtype).eps
        return np.where(np.abs(np.abs(k) - nyquist) <= eps, f(0), -k).astype(k.dtype)

    # ---- derived quantities (configuration.py:437-563) ----
    @property
    def dim(self):
        return 3

    @property
    def nMesh(self):
        return self.mesh_shape[0]

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
        return self.ptcl_spacing**3

    @property
    def box_size(self):
        return tuple(self.ptcl_spacing * s for s in self.ptcl_grid_shape)

    @property
    def box_vol(self):
        return float(np.prod(self.box_size))

    @property
    def disp_size(self):
        """Inverse mesh-cell size (displacements in cell units)."""
        return 1 / self.cell_size

    @property
    def local_mesh_shape(self):
        return self.mesh_shape

    @property
    def local_mesh_with_halo_shape(self):
        return self.mesh_shape

    @property
    def local_mesh_size(self):
        return self.mesh_size

    # ---- units (configuration.py:483-506) ----
    @property
    def V(self):
        return self.L / self.T

    @property
    def H_0(self):
        return self.H_0_SI * self.T

    @property
    def c(self):
        return self.c_SI / self.V

    @property
    def G(self):
        return self.G_SI * self.M / (self.L * self.V**2)

    @property
    def rho_crit(self):
        return 3 * self.H_0**2 / (8 * np.pi * self.G)

    @property
    def transfer_k_num(self):
        return 1 + math.ceil((self.transfer_lgk_max - self.transfer_lgk_min) / self.transfer_lgk_maxstep) + 1

    @property
    def transfer_lgk_step(self):
        return (self.transfer_lgk_max - self.transfer_lgk_min) / (self.transfer_k_num - 2)

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
    def a_nbody_step(self):
        return (self.a_stop - self.a_start) / self.a_nbody_num

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
        """Growth-table scale factors: growth_a_custom, else a_lpt then a_nbody[1:]
        (configuration.py:559-563)."""
        if self.growth_a_custom is not None:
            return np.array(self.growth_a_custom, dtype=np.float64)
        return np.concatenate((self.a_lpt, self.a_nbody[1:]))

    @property
    def has_particle_nyquist_masks(self):
        return self.mesh_shape != self.ptcl_grid_shape

    def particle_nyquist_masks(self):
        """Per-axis masks of modes resolvable on the particle grid (core/utils.py:15-37)."""
        f = self.np_dtype.type
        kn = f(np.pi / self.ptcl_spacing)
        limit = kn + kn * f(8 * np.finfo(self.np_dtype).eps)
        return tuple((np.abs(k) <= limit).astype(self.np_dtype) for k in self.kvec)

    @staticmethod
    def _fastpm_neg_k(k, spacing):
        """Derivative factor c (neg_ik = i c) of FastPM's 4-point gradient,
        (8 sin(k dx) - sin(2 k dx)) / (6 dx) (gravity.py:355-391), in k's dtype."""
        f = k.dtype.type
        phase = (k * f(spacing)).astype(k.dtype)
        d = ((f(8.0) * np.sin(phase)).astype(k.dtype) - np.sin(f(2.0) * phase)).astype(k.dtype)
        return (-(d / f(6.0 * spacing))).astype(k.dtype)

    def spectral_tables(self, which="mesh", device=None, green_kernel=0, gradient_kernel=0):
        """Device table [kx ky kz cx cy cz (mx my mz)] for pmb_green_gradient.

        which="mesh" uses the force mesh (kvec, cell_size); "particle" the
        particle grid (kvec_spacing, ptcl_spacing).  green_kernel=1 replaces
        k by the discrete-Laplacian wavenumber 2 sin(k dx/2)/dx
        (gravity.py:122-171); gradient_kernel=1 takes FastPM's 4-point
        derivative for c instead of the spectral -k (gravity.py:355-391)."""
        device = self.device if device is None else torch.device(device)
        key = (which, str(device), green_kernel, gradient_kernel)
        if key not in self._tables:
            if which == "mesh":
                ks, spacing, masks = self.kvec, self.cell_size, (self.particle_nyquist_masks()
                                                                 if self.has_particle_nyquist_masks else ())
            else:
                ks, spacing, masks = self.kvec_spacing, self.ptcl_spacing, ()
            cs = [(self._fastpm_neg_k(k, spacing) if gradient_kernel == 1 else self._neg_k(k, spacing)) for k in ks]
            if green_kernel == 1:
                f = self.np_dtype.type
                c = f(spacing)
                ks = [(f(2) * np.sin(k * c / f(2)) / c).astype(self.np_dtype) for k in ks]
            parts = list(ks) + cs + list(masks)
            self._tables[key] = torch.from_numpy(np.concatenate(parts).astype(self.np_dtype)).to(device)
        return self._tables[key]
