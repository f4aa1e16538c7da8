"""pmb_scatter_density_noalloc: the density scatter for callers that may not allocate.

A framework plugin whose host program owns all device memory (and hands it no
scratch) cannot call cudaMalloc and cannot supply the workspace the regular
entry points take; this entry point keeps its scratch in a fixed device array
inside the library.  The test calls it through the C ABI twice in a row (the
second call sees the first call's leftovers in the shared array) and compares
each result with the workspace path pmb_sort_rows + pmb_scatter_rows bit for
bit (both sum the same exact fixed-point contributions), including a problem
just under the fixed scratch size; one just over it is rejected before any
work is queued.  It lives in its own file so that a run stopping at the first
failure has already run every other test.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _particles(n1, mesh, seed):
    rng = np.random.default_rng(seed)
    g = np.arange(n1) * mesh
    pmid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.int16)
    disp = rng.normal(0, 2.5, size=pmid.shape).astype(np.float32)
    return torch.from_numpy(pmid).cuda(), torch.from_numpy(disp).cuda()


def _reference_scatter(pmid, disp, dims, cell, val):
    from pmpp_b200 import _lib
    from pmpp_b200.runtime import stream_handle
    L = _lib.lib()
    n = pmid.shape[0]
    nx, ny, nz = dims
    sorted_buf = torch.empty(L.pmb_sorted_bytes(n, nx, ny, nz), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(L.pmb_sort_scratch_bytes(n, nx, ny, nz), dtype=torch.uint8, device="cuda")
    s16 = torch.empty(16, dtype=torch.uint8, device="cuda")
    out = torch.empty(dims, dtype=torch.float32, device="cuda")
    s = stream_handle()
    _lib.call("pmb_sort_rows", pmid.data_ptr(), disp.data_ptr(), None, 0.0, n, nx, ny, nz, cell,
              sorted_buf.data_ptr(), scratch.data_ptr(), scratch.numel(), s)
    _lib.call("pmb_scatter_rows", sorted_buf.data_ptr(), n, nx, ny, nz, 1, None, 0, val, 0, 1.0, out.data_ptr(),
              s16.data_ptr(), s)
    return out


def _noalloc_scatter(pmid, disp, dims, cell, val):
    from pmpp_b200 import _lib
    from pmpp_b200.runtime import stream_handle
    out = torch.full(dims, float("nan"), dtype=torch.float32, device="cuda")
    status = _lib.lib().pmb_scatter_density_noalloc(pmid.data_ptr(), disp.data_ptr(), pmid.shape[0], dims[0],
                                                    dims[1], dims[2], cell, val, out.data_ptr(), stream_handle())
    assert status == 0, _lib.lib().pmb_last_error()
    return out


def _bits(t):
    return t.cpu().numpy().view(np.uint32)


def test_noalloc_scatter_matches_workspace_path_on_consecutive_calls():
    cases = [(16, 2, 0, 4.0), (24, 2, 1, 8.0)]  # different sizes back to back reuse the shared array
    for _ in range(2):
        for n1, mesh, seed, val in cases:
            pmid, disp = _particles(n1, mesh, seed)
            dims = (n1 * mesh, ) * 3
            ref = _reference_scatter(pmid, disp, dims, 1.0, val)
            got = _noalloc_scatter(pmid, disp, dims, 1.0, val)
            torch.cuda.synchronize()
            assert np.array_equal(_bits(got), _bits(ref))
            np.testing.assert_allclose(float(got.double().sum()), val * pmid.shape[0], rtol=1e-5)


# A 128^3 mesh needs 28 B per particle plus 12 B per mesh row and 768 B for
# alignment, the scale and the status word: 28 n + 198144 bytes for n a
# multiple of 64, so 1191296 particles fill the 32 MiB (33554432 B) scratch
# exactly and 1191360 do not fit.
N_FITS, N_OVER = 1191296, 1191360


def test_noalloc_scatter_just_under_the_limit():
    rng = np.random.default_rng(4)
    pmid = torch.from_numpy(rng.integers(0, 128, size=(N_FITS, 3)).astype(np.int16)).cuda()
    disp = torch.from_numpy(rng.uniform(-2.0, 2.0, size=(N_FITS, 3)).astype(np.float32)).cuda()
    dims = (128, 128, 128)
    for _ in range(2):
        ref = _reference_scatter(pmid, disp, dims, 1.0, 0.5)
        got = _noalloc_scatter(pmid, disp, dims, 1.0, 0.5)
        torch.cuda.synchronize()
        assert np.array_equal(_bits(got), _bits(ref))


def test_noalloc_scatter_rejects_oversized_problems():
    from pmpp_b200 import _lib
    from pmpp_b200.runtime import stream_handle
    pmid, disp = _particles(8, 2, 0)
    n_too_many = 2_000_000  # 28 B per particle alone exceeds the fixed 32 MiB scratch
    status = _lib.lib().pmb_scatter_density_noalloc(pmid.data_ptr(), disp.data_ptr(), n_too_many, 16, 16, 16, 1.0,
                                                    1.0, disp.data_ptr(), stream_handle())
    assert status == -1
    assert b"32 MiB" in _lib.lib().pmb_last_error()
    # just over the limit on a 128^3 mesh: rejected, the output left untouched
    pmid = torch.zeros((N_OVER, 3), dtype=torch.int16, device="cuda")
    disp = torch.zeros((N_OVER, 3), dtype=torch.float32, device="cuda")
    out = torch.full((128, 128, 128), 7.0, device="cuda")
    status = _lib.lib().pmb_scatter_density_noalloc(pmid.data_ptr(), disp.data_ptr(), N_OVER, 128, 128, 128, 1.0,
                                                    1.0, out.data_ptr(), stream_handle())
    assert status == -1
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())
