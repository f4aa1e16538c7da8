"""CPU-side checks of the C ABI: the library loads and exports every symbol
include/pmb200.h declares, and the host-side FP64 cosmology agrees with the
oracle.  No device work."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pmb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pmb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from pmpp_b200 import _lib
    L = _lib.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert set(declared_symbols()) <= set(_lib.exported_symbols()) | {"pmb_last_error"}
    assert L.pmb_abi_version() == 3


def test_workspace_queries_without_device():
    from pmpp_b200 import _lib
    L = _lib.lib()
    assert L.pmb_sorted_bytes(1000, 16, 16, 16) >= 20 * 1000
    assert L.pmb_sort_scratch_bytes(1000, 16, 16, 16) > 0
    assert L.pmb_sort_by_cell_scratch_bytes(1000, 16, 16, 16) > 0


def test_invalid_arguments_fail_loudly():
    import pytest
    from pmpp_b200 import _lib
    with pytest.raises(_lib.PMBError):
        _lib.call("pmb_sort_rows", None, None, None, 0.0, 10, 0, 4, 4, 1.0, None, None, 0, None)
    assert b"unsupported mesh" in _lib.lib().pmb_last_error()


def test_ensemble_create_rejects_bad_layouts_without_device_work():
    """Descriptions are validated on the host before any CUDA call."""
    import ctypes

    import numpy as np

    from pmpp_b200 import _lib
    L = _lib.lib()

    def create(shapes, counts=None, cells=None):
        n = len(shapes)
        counts = np.array(counts or [8] * n, np.int64)
        sh = np.array(shapes, np.int32).reshape(-1)
        cells = np.array(cells or [1.0] * n, np.float32)
        vals = np.ones(n, np.float32)
        muls = np.full(n, 0.45, np.float32)
        masks = np.zeros(n, np.int32)
        h = ctypes.c_void_p()
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        return L.pmb_ens_create(n, p(counts), p(sh), p(cells), p(vals), p(muls), p(masks), 4, ctypes.byref(h)), h

    st, h = create([(8, 8, 8), (4, 4, 4), (8, 8, 8)])
    assert st == -1 and not h.value
    assert b"consecutive" in L.pmb_last_error()
    st, _ = create([(8, 8, 8)], cells=[0.0])
    assert st == -1
    st, _ = create([(8, 8, 8)], counts=[-1])
    assert st == -1
    st, _ = create([(8, 8, 0)])
    assert st == -1


def test_count_and_shape_limits_rejected_on_the_host():
    """Particle counts past the uint32 permutation (n >= 2^32 - 1) and meshes of
    2^32 cells or more (uint32 cell keys) are rejected before any device work,
    with the output pointers never touched (they are null here)."""
    from pmpp_b200 import _lib
    L = _lib.lib()
    big_n = 2**32
    calls = [
        ("pmb_sort_rows", (None, None, None, 0.0, big_n, 16, 16, 16, 1.0, None, None, 1 << 40, None)),
        ("pmb_sort_rows_ex", (None, None, None, 0.0, big_n, 16, 16, 16, 1.0, 0.0, 0.0, 0.0, None, None, None, 1 << 40,
                              None)),
        ("pmb_scatter_rows", (None, big_n, 16, 16, 16, 1, None, 0, 1.0, 0, 1.0, None, None, None)),
        ("pmb_gather_rows", (None, big_n, 16, 16, 16, 3, None, None, None, 0.0, None)),
        ("pmb_interp_grad_rows", (None, big_n, 16, 16, 16, 1, None, None, 1.0, 1.0, 0, None, None, None, None)),
        # 2048 x 2048 x 1024 = 2^32 cells
        ("pmb_sort_rows", (None, None, None, 0.0, 10, 2048, 2048, 1024, 1.0, None, None, 1 << 40, None)),
        ("pmb_scatter_rows", (None, 10, 2048, 2048, 1024, 1, None, 0, 1.0, 0, 1.0, None, None, None)),
        ("pmb_force", (None, None, None, 0.0, 10, 2048, 2048, 1024, 1.0, 1.0, 1.0, None, 0, 0, None, None, 0, None,
                       None, None, 0.0, None, 1 << 40, None)),
        ("pmb_scatter_density_noalloc", (None, None, big_n, 16, 16, 16, 1.0, 1.0, None, None)),
    ]
    for name, args in calls:
        st = getattr(L, name)(*args)
        assert st == -1, (name, st, L.pmb_last_error())
    assert L.pmb_set_wait_limit(-1) == 0
