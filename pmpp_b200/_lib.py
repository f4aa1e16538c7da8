"""ctypes binding of libpmb200.so (include/pmb200.h).

The library must have been built in-tree (``python -m pmpp_b200.build``); a
missing library is an error, never a silent fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpmb200.so")

c_int, c_i64, c_f, c_d, c_p = ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_void_p

_SIGS = {
    "pmb_abi_version": (c_int, []),
    "pmb_last_error": (ctypes.c_char_p, []),
    "pmb_sorted_bytes": (c_i64, [c_i64, c_int, c_int, c_int]),
    "pmb_sort_scratch_bytes": (c_i64, [c_i64, c_int, c_int, c_int]),
    "pmb_sort_rows": (c_int, [c_p, c_p, c_p, c_f, c_i64, c_int, c_int, c_int, c_f, c_p, c_p, c_i64, c_p]),
    "pmb_sort_rows_ex": (c_int, [c_p, c_p, c_p, c_f, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_f, c_p, c_p, c_p,
                                 c_i64, c_p]),
    "pmb_sort_by_cell": (c_int, [c_p, c_p, c_i64, c_int, c_int, c_int, c_f, c_p, c_p, c_p, c_i64, c_p]),
    "pmb_cic_general_scratch_bytes": (c_i64, [c_int, c_int, c_int, c_int]),
    "pmb_cic_general_scatter": (c_int, [c_p, c_p, c_p, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_f, c_f, c_int,
                                        c_int, c_int, c_int, c_p, c_f, c_p, c_p, c_i64, c_p]),
    "pmb_cic_general_gather": (c_int, [c_p, c_p, c_p, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_f, c_f, c_int,
                                       c_int, c_int, c_int, c_p, c_p, c_p]),
    "pmb_cic_general_interp_grad": (c_int, [c_p, c_p, c_p, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_f, c_f,
                                            c_int, c_int, c_int, c_int, c_p, c_p, c_f, c_p, c_p, c_p]),
    "pmb_sort_by_cell_scratch_bytes": (c_i64, [c_i64, c_int, c_int, c_int]),
    "pmb_scatter_rows": (c_int, [c_p, c_i64, c_int, c_int, c_int, c_int, c_p, c_int, c_f, c_int, c_f, c_p, c_p, c_p]),
    "pmb_gather_rows": (c_int, [c_p, c_i64, c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_f, c_p]),
    "pmb_gather_rows2": (c_int, [c_p, c_i64, c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_f, c_f, c_p]),
    "pmb_interp_grad_rows": (c_int, [c_p, c_i64, c_int, c_int, c_int, c_int, c_p, c_p, c_f, c_f, c_int, c_p, c_p,
                                     c_p, c_p]),
    "pmb_wait_timeouts": (c_int, [c_p]),
    "pmb_set_wait_limit": (c_int, [c_i64]),
    "pmb_sorted_status": (c_int, [c_p, c_i64, c_int, c_int, c_int, c_p, c_p]),
    "pmb_device_status": (c_int, [c_p]),
    "pmb_set_gather_staging": (c_int, [c_int]),
    "pmb_fft_work_bytes": (c_i64, [c_int, c_int, c_int, c_int]),
    "pmb_set_pmfft": (c_int, [c_int]),
    "pmb_pmfft_supported": (c_int, [c_int, c_int, c_int]),
    "pmb_pmfft_channel_elems": (c_i64, [c_int, c_int, c_int]),
    "pmb_pmfft_z": (c_int, [c_int, c_int, c_int, c_int, c_int, c_p, c_p, c_p]),
    "pmb_pmfft_col": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_int, c_p, c_p, c_int, c_f,
                              c_p]),
    "pmb_pmfft_z2": (c_int, [c_int, c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_int, c_int, c_p]),
    "pmb_pmfft_col2": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_int, c_p, c_p, c_int, c_f,
                               c_int, c_p]),
    "pmb_pmfft_timeouts": (c_int, [c_p]),
    "pmb_pmfft_set_col_ctas": (c_int, [c_int]),
    "pmb_rfft3": (c_int, [c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_p]),
    "pmb_irfft3": (c_int, [c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_p]),
    "pmb_green_gradient": (c_int, [c_p, c_p, c_int, c_int, c_int, c_p, c_int, c_int, c_p, c_p, c_int, c_f, c_p]),
    "pmb_interlace_spectra": (c_int, [c_p, c_p, c_int, c_int, c_int, c_int, c_p]),
    "pmb_project_density": (c_int, [c_p, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_p, c_p]),
    "pmb_cnn_conv3d": (c_int, [c_p, c_int, c_p, c_p, c_p, c_p, c_int, c_p, c_p, c_int, c_int, c_int, c_int, c_int, c_p]),
    "pmb_cnn_conv3d_wgrad": (c_int, [c_p, c_int, c_p, c_int, c_int, c_int, c_int, c_p, c_p, c_p]),
    "pmb_cnn_stem_input": (c_int, [c_p, c_p, c_i64, c_f, c_f, c_p, c_p]),
    "pmb_cnn_residual": (c_int, [c_p, c_p, c_i64, c_f, c_f, c_p, c_p]),
    "pmb_cnn_residual_adjoint": (c_int, [c_p, c_p, c_p, c_i64, c_f, c_f, c_p, c_p, c_p, c_p]),
    "pmb_cnn_norm_adjoint": (c_int, [c_p, c_p, c_p, c_i64, c_f, c_f, c_f, c_f, c_p, c_p, c_p]),
    "pmb_green_potential": (c_int, [c_p, c_p, c_int, c_int, c_int, c_p, c_int, c_int, c_p, c_p, c_int, c_f, c_p]),
    "pmb_gradient_spectra": (c_int, [c_p, c_p, c_f, c_p, c_int, c_int, c_int, c_p, c_f, c_p]),
    "pmb_gradient_adjoint_plain": (c_int, [c_p, c_p, c_int, c_int, c_int, c_p, c_f, c_p]),
    "pmb_green_gradient_adjoint": (c_int, [c_p, c_p, c_int, c_int, c_int, c_p, c_int, c_int, c_p, c_p, c_int, c_f,
                                           c_p]),
    "pmb_force_workspace_bytes": (c_i64, [c_i64, c_int, c_int, c_int]),
    "pmb_force": (c_int, [c_p, c_p, c_p, c_f, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_p, c_int, c_int, c_p, c_p,
                          c_int, c_p, c_p, c_p, c_f, c_p, c_i64, c_p]),
    "pmb_force2": (c_int, [c_p, c_p, c_p, c_f, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_p, c_int, c_int, c_p, c_p,
                          c_int, c_p, c_p, c_p, c_f, c_f, c_p, c_i64, c_p]),
    "pmb_force_streamed_workspace_bytes": (c_i64, [c_i64, c_int, c_int, c_int]),
    "pmb_force_streamed": (c_int, [c_p, c_p, c_p, c_f, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_p, c_int, c_int,
                                   c_p, c_p, c_int, c_p, c_p, c_i64, c_p]),
    "pmb_force_vjp_workspace_bytes": (c_i64, [c_i64, c_int, c_int, c_int]),
    "pmb_force_vjp": (c_int, [c_p, c_p, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_p, c_int, c_int, c_p, c_p, c_int,
                              c_p, c_p, c_p, c_p, c_i64, c_p]),
    "pmb_force_vjp_presorted": (c_int, [c_p, c_i64, c_int, c_int, c_int, c_f, c_f, c_f, c_p, c_int, c_int, c_p, c_p,
                                        c_int, c_p, c_p, c_p, c_p, c_i64, c_p]),
    "pmb_axpy": (c_int, [c_p, c_p, c_i64, c_f, c_p]),
    "pmb_kick_adj": (c_int, [c_p, c_p, c_p, c_p, c_i64, c_f, c_p, c_p]),
    "pmb_kick_adj2": (c_int, [c_p, c_p, c_p, c_p, c_i64, c_f, c_f, c_int, c_int, c_p, c_p, c_p, c_p]),
    "pmb_kick_adj3": (c_int, [c_p, c_p, c_p, c_p, c_i64, c_f, c_f, c_int, c_int, c_p, c_p, c_p, c_p, c_f, c_p, c_p]),
    "pmb_drift_cot_adj": (c_int, [c_p, c_p, c_p, c_i64, c_f, c_p, c_p]),
    "pmb_drift_adj": (c_int, [c_p, c_p, c_p, c_p, c_i64, c_f, c_p, c_p]),
    "pmb_dot": (c_int, [c_p, c_p, c_i64, c_p, c_p]),
    "pmb_sum": (c_int, [c_p, c_i64, c_p, c_p]),
    "pmb_white_noise_nested": (c_int, [ctypes.c_uint32, c_int, c_int, c_int, c_p, c_p, c_p]),
    "pmb_linear_modes": (c_int, [c_p, c_p, c_p, c_int, c_int, c_int, c_p, c_p, c_p, c_int, c_d, c_d, c_d, c_d, c_d,
                                 c_d, c_p]),
    "pmb_lpt_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_lpt": (c_int, [c_p, c_int, c_int, c_int, c_f, c_f, c_p, c_int, c_f, c_f, c_f, c_f, c_p, c_p, c_p, c_i64, c_f,
                        c_p, c_p, c_p, c_i64, c_p]),
    "pmb_lpt_vjp_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_lpt_vjp": (c_int, [c_p, c_int, c_int, c_int, c_f, c_p, c_int, c_f, c_f, c_f, c_f, c_p, c_p, c_p, c_p, c_i64,
                            c_p, c_p, c_p, c_p, c_i64, c_p]),
    "pmb_pk_shells": (c_int, [c_p, c_int, c_int, c_int, c_p, c_int, c_int, c_p, c_p, c_p, c_p, c_p]),
    "pmb_shell_stats": (c_int, [c_int, c_int, c_int, c_int, c_p, c_p, c_p]),
    "pmb_pk_shells_adjoint": (c_int, [c_p, c_int, c_int, c_int, c_p, c_int, c_int, c_p, c_f, c_p, c_p]),
    "pmb_overdensity": (c_int, [c_p, c_p, c_i64, c_p, c_p]),
    "pmb_scatter_density_noalloc": (c_int, [c_p, c_p, c_i64, c_int, c_int, c_int, c_f, c_f, c_p, c_p]),
    "pmb_mlp_param_counts": (c_int, [c_p, c_p]),
    "pmb_mlp_table": (c_int, [c_p, c_p, c_f, c_f, c_f, c_f, c_int, c_p, c_p]),
    "pmb_mlp_backward": (c_int, [c_p, c_p, c_f, c_f, c_f, c_f, c_int, c_p, c_p, c_p]),
    "pmb_transfer_cot": (c_int, [c_p, c_p, c_int, c_int, c_int, c_p, c_int, c_int, c_p, c_p]),
    "pmb_growth_table": (c_int, [c_d, c_d, c_d, c_d, c_p, c_int, c_d, c_d, c_d, c_d, c_p, c_p]),
    "pmb_time_factor": (c_int, [c_int, c_d, c_d, c_d, c_d, c_d, c_d, c_d, c_p, c_int, c_p, c_p, c_p, c_p]),
    "pmb_lpt_factors": (c_int, [c_d, c_d, c_d, c_d, c_d, c_p, c_int, c_p, c_p, c_p, c_p]),
    "pmb_transfer_fit": (c_int, [c_p, c_i64, c_d, c_d, c_d, c_d, c_int, c_p]),
    "pmb_linear_power": (c_int, [c_p, c_i64, c_p, c_p, c_int, c_d, c_d, c_d, c_d, c_d, c_p]),
    "pmb_force64_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_force64": (c_int, [c_p, c_p, c_p, c_d, c_i64, c_int, c_int, c_int, c_d, c_d, c_d, c_p, c_int, c_p, c_p, c_p,
                            c_p, c_d, c_p, c_i64, c_p]),
    "pmb_deposit64": (c_int, [c_p, c_p, c_i64, c_int, c_int, c_int, c_d, c_d, c_p, c_p]),
    "pmb_axpy64": (c_int, [c_p, c_p, c_i64, c_d, c_p]),
    "pmb_sum64": (c_int, [c_p, c_i64, c_p, c_p]),
    "pmb_force_vjp64_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_force_vjp64": (c_int, [c_p, c_p, c_i64, c_int, c_int, c_int, c_d, c_d, c_d, c_p, c_int, c_p, c_p, c_p, c_p,
                                c_p, c_i64, c_p]),
    "pmb_force64_interlaced_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_force64_interlaced": (c_int, [c_p, c_p, c_p, c_d, c_i64, c_int, c_int, c_int, c_d, c_d, c_d, c_p, c_int,
                                       c_p, c_p, c_p, c_p, c_d, c_p, c_i64, c_p]),
    "pmb_force_vjp64_interlaced_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_force_vjp64_interlaced": (c_int, [c_p, c_p, c_i64, c_int, c_int, c_int, c_d, c_d, c_d, c_p, c_int, c_p,
                                           c_p, c_p, c_p, c_p, c_i64, c_p]),
    "pmb_dot64": (c_int, [c_p, c_p, c_i64, c_p, c_p]),
    "pmb_lpt64_ex": (c_int, [c_p, c_int, c_int, c_int, c_d, c_d, c_p, c_int, c_d, c_d, c_d, c_d, c_p, c_p, c_p, c_i64,
                             c_d, c_p, c_p, c_p, c_i64, c_p]),
    "pmb_lpt_vjp64_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_lpt_vjp64": (c_int, [c_p, c_int, c_int, c_int, c_d, c_p, c_int, c_d, c_d, c_d, c_d, c_p, c_p, c_p, c_p, c_i64,
                              c_p, c_p, c_p, c_p, c_i64, c_p]),
    "pmb_scatter_vjp64": (c_int, [c_p, c_p, c_i64, c_int, c_int, c_int, c_d, c_d, c_p, c_p, c_p]),
    "pmb_fft64_work_bytes": (c_i64, [c_int, c_int, c_int, c_int]),
    "pmb_rfft3_64": (c_int, [c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_p]),
    "pmb_irfft3_64": (c_int, [c_int, c_int, c_int, c_int, c_p, c_p, c_p, c_p]),
    "pmb_white_noise_nested64": (c_int, [ctypes.c_uint32, c_int, c_int, c_int, c_p, c_p]),
    "pmb_linear_modes64": (c_int, [c_p, c_p, c_int, c_int, c_int, c_p, c_p, c_p, c_int, c_d, c_d, c_d, c_d, c_d, c_d,
                                   c_p]),
    "pmb_lpt64_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_lpt64": (c_int, [c_p, c_int, c_int, c_int, c_d, c_d, c_p, c_int, c_d, c_d, c_d, c_d, c_p, c_p, c_p, c_i64, c_d,
                          c_p, c_p, c_i64, c_p]),
    "pmb_pk_shells64": (c_int, [c_p, c_int, c_int, c_int, c_p, c_int, c_int, c_p, c_p]),
    "pmb_pk_shells_adjoint64": (c_int, [c_p, c_int, c_int, c_int, c_p, c_int, c_int, c_p, c_d, c_p, c_p]),
    "pmb_overdensity64": (c_int, [c_p, c_p, c_i64, c_p, c_p]),
    "pmb_ens_create": (c_int, [c_int, c_p, c_p, c_p, c_p, c_p, c_p, c_int, c_p]),
    "pmb_ens_destroy": (c_int, [c_p]),
    "pmb_ens_workspace_bytes": (c_i64, [c_p]),
    "pmb_ens_size": (c_i64, [c_p, c_int]),
    "pmb_ens_bind": (c_int, [c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_p]),
    "pmb_ens_set_tiles": (c_int, [c_p, c_p, c_p]),
    "pmb_ens_set_launch": (c_int, [c_p, c_int, c_int, c_int]),
    "pmb_ens_set_factors": (c_int, [c_p, c_int, c_p, c_p]),
    "pmb_ens_set_step": (c_int, [c_p, c_int, c_p]),
    "pmb_ens_stage": (c_int, [c_p, c_int, c_int, c_int, c_p]),
    "pmb_ens_force": (c_int, [c_p, c_int, c_int, c_p]),
    "pmb_ens_step": (c_int, [c_p, c_p]),
}

_lib = None


class PMBError(RuntimeError):
    """A libpmb200 entry point returned a non-zero status."""


def lib():
    """Load libpmb200.so once; raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pmpp_b200.build`")
        L = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return sorted(_SIGS)


def check(status, what):
    if status != 0:
        msg = lib().pmb_last_error().decode(errors="replace")
        raise PMBError(f"{what} failed with status {status}: {msg}")


# Hand-written kernels launched per entry point (cuFFT's own kernels excluded).
_KERNELS = {
    "pmb_sort_rows": 5, "pmb_sort_rows_ex": 5, "pmb_cic_general_scatter": 3, "pmb_cic_general_gather": 1,
    "pmb_cic_general_interp_grad": 1, "pmb_gather_rows": 1, "pmb_gather_rows2": 1, "pmb_interp_grad_rows": 1,
    "pmb_green_gradient": 1, "pmb_interlace_spectra": 1, "pmb_project_density": 1, "pmb_cnn_conv3d": 1,
    "pmb_cnn_conv3d_wgrad": 1, "pmb_cnn_stem_input": 1, "pmb_cnn_residual": 1, "pmb_cnn_residual_adjoint": 1,
    "pmb_cnn_norm_adjoint": 1, "pmb_green_potential": 1, "pmb_gradient_spectra": 1, "pmb_gradient_adjoint_plain": 1,
    "pmb_green_gradient_adjoint": 1, "pmb_axpy": 1,
    "pmb_kick_adj": 1, "pmb_kick_adj2": 1, "pmb_kick_adj3": 1, "pmb_drift_cot_adj": 1, "pmb_drift_adj": 1, "pmb_dot": 1,
    "pmb_force": 9, "pmb_force2": 9, "pmb_force_streamed": 14, "pmb_force_vjp": 11, "pmb_force_vjp_presorted": 6, "pmb_sum": 1,
    "pmb_white_noise_nested": 1, "pmb_linear_modes": 1,
    "pmb_lpt": 4, "pmb_lpt_vjp": 6, "pmb_pk_shells": 1, "pmb_shell_stats": 1, "pmb_pk_shells_adjoint": 1,
    "pmb_overdensity": 1, "pmb_ens_force": 7, "pmb_ens_step": 9, "pmb_ens_set_step": 1,
    "pmb_force64": 5, "pmb_force64_interlaced": 7, "pmb_force_vjp64_interlaced": 6, "pmb_deposit64": 1, "pmb_axpy64": 1, "pmb_sum64": 1, "pmb_force_vjp64": 4, "pmb_dot64": 1, "pmb_lpt64_ex": 4, "pmb_lpt_vjp64": 6,
    "pmb_scatter_vjp64": 1, "pmb_white_noise_nested64": 1,
    "pmb_linear_modes64": 1, "pmb_lpt64": 4, "pmb_pk_shells64": 1, "pmb_pk_shells_adjoint64": 1, "pmb_overdensity64": 1,
    "pmb_pmfft_z": 1, "pmb_pmfft_col": 1, "pmb_pmfft_z2": 1, "pmb_pmfft_col2": 1,
}
_pmfft = {"enabled": True}
_launches = [0]


def wait_timeouts():
    """Bounded device waits that gave up since the library was loaded."""
    v = ctypes.c_uint32()
    check(lib().pmb_wait_timeouts(ctypes.byref(v)), "pmb_wait_timeouts")
    return v.value


def device_status():
    """Device-wide flags (1 timed-out wait, 2 non-finite displacement, 4
    non-finite deposit value) since the last call, then cleared; raises
    PMBError naming the conditions when any is set.  Synchronises the device."""
    v = ctypes.c_uint32()
    check(lib().pmb_device_status(ctypes.byref(v)), "pmb_device_status")
    return v.value


def set_wait_limit(polls):
    """Poll limit of the first bounded wait of the staged / TMA-fed kernels
    (None or a negative value: the default)."""
    check(lib().pmb_set_wait_limit(-1 if polls is None else int(polls)), "pmb_set_wait_limit")


def set_pmfft(enabled):
    """Route the fused force through the hand-written FFT passes (default) or cuFFT."""
    check(lib().pmb_set_pmfft(1 if enabled else 0), "pmb_set_pmfft")
    _pmfft["enabled"] = bool(enabled)


def pmfft_active(nx, ny, nz):
    return _pmfft["enabled"] and bool(lib().pmb_pmfft_supported(int(nx), int(ny), int(nz)))


def pmfft_timeouts():
    v = ctypes.c_uint32()
    check(lib().pmb_pmfft_timeouts(ctypes.byref(v)), "pmb_pmfft_timeouts")
    return v.value


def reset_launch_count():
    _launches[0] = 0


def launch_count():
    return _launches[0]


def call(name, *args):
    """Call an entry point that returns a status and raise on failure."""
    check(getattr(lib(), name)(*args), name)
    if name == "pmb_scatter_rows":
        _launches[0] += 2 if args[6] is None else 3
    else:
        _launches[0] += _KERNELS.get(name, 0)
        # the hand-written FFT chain replaces the multiplier kernel by six passes
        if name in ("pmb_force", "pmb_force2") and pmfft_active(*args[5:8]):
            _launches[0] += 5
        elif name == "pmb_force_vjp" and pmfft_active(*args[3:6]):
            _launches[0] += 5
        elif name == "pmb_force_vjp_presorted" and pmfft_active(*args[2:5]):
            _launches[0] += 5
