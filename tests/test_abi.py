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
    assert L.pmb_abi_version() == 1


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
