"""ffcm_sort_cells_noalloc (cell-list sort whose scratch lives in the
library's own device image) against the handle-based sort,
ffcm_sort_particles_by_cell, through the C ABI. Kept last in collection
order so it also runs after every other GPU test in the same process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_CELLS = 1 << 21   # FFCM_NOALLOC_MAX_CELLS


def _noalloc(lib):
    f = lib.ffcm_sort_cells_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


@pytest.mark.parametrize("L,M,N,R_c", [(40.0, 64, 2000, 3.0), (275.6, 512, 500_000, 3.0),
                                       (12.0, 32, 3000, 3.0)])
def test_noalloc_sort_matches_handle_sort(ffcm, L, M, N, R_c):
    torch = pytest.importorskip("torch")
    lib = ffcm._lib.load()
    sort = _noalloc(lib)
    rng = np.random.default_rng(N)
    Y = (rng.random((N, 3)) * L).astype(np.float32)
    F = rng.standard_normal((N, 3)).astype(np.float32)
    cfg = ffcm.FFCMConfig(np.float32, L=(L, L, L), R_c=R_c, N=N, kernel_widths_ratio=2.0,
                          viscosity=1.0, num_grid_points=(M, M, M), M_G=8)
    ffcm.wrap_positions(cfg, Y)
    ffcm.assign_cells(cfg)
    ffcm.sort_particles_by_cell(cfg, F)
    key = cfg.get("CELL_HASH")
    want = [cfg.get(n) for n in ("ORIGINAL_INDEX", "CELL_START", "CELL_END")]
    ncell = want[1].size
    dkey = torch.from_numpy(key).cuda()
    outs = [torch.full((N,), -7, dtype=torch.int32, device="cuda"),
            torch.full((ncell,), -7, dtype=torch.int32, device="cuda"),
            torch.full((ncell,), -7, dtype=torch.int32, device="cuda")]
    torch.cuda.synchronize()
    for _ in range(2):            # two calls in a row: the scratch is reset by each call
        for o in outs:
            o.fill_(-7)
        torch.cuda.synchronize()
        rc = sort(dkey.data_ptr(), N, ncell, outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), None)
        assert rc == 0, ffcm._lib.last_error()
        for got, ref in zip(outs, want):
            np.testing.assert_array_equal(got.cpu().numpy(), ref)
    cfg.close()


def test_noalloc_sort_rejects_bad_sizes_and_keys(ffcm):
    torch = pytest.importorskip("torch")
    lib = ffcm._lib.load()
    sort = _noalloc(lib)
    N, ncell = 100, 27
    key = torch.arange(N, dtype=torch.int32, device="cuda") % ncell
    oi = torch.empty(N, dtype=torch.int32, device="cuda")
    cs = torch.empty(ncell, dtype=torch.int32, device="cuda")
    ce = torch.empty(ncell, dtype=torch.int32, device="cuda")
    assert sort(key.data_ptr(), N, MAX_CELLS + 1, oi.data_ptr(), cs.data_ptr(), ce.data_ptr(), None) == 1
    assert "scratch" in ffcm._lib.last_error()
    assert sort(key.data_ptr(), N, 0, oi.data_ptr(), cs.data_ptr(), ce.data_ptr(), None) == 1
    bad = key.clone()
    bad[5] = ncell            # out of range: skipped on the device, reported as an argument error
    assert sort(bad.data_ptr(), N, ncell, oi.data_ptr(), cs.data_ptr(), ce.data_ptr(), None) == 1
    assert "outside" in ffcm._lib.last_error()
    assert sort(key.data_ptr(), N, ncell, oi.data_ptr(), cs.data_ptr(), ce.data_ptr(), None) == 0
    k = key.cpu().numpy()
    order = np.argsort(k, kind="stable") + 1
    np.testing.assert_array_equal(oi.cpu().numpy(), order)
    counts = np.bincount(k, minlength=ncell)
    np.testing.assert_array_equal(ce.cpu().numpy(), np.cumsum(counts))
    np.testing.assert_array_equal(cs.cpu().numpy(), np.cumsum(counts) - counts + 1)


@pytest.mark.parametrize("N,ncell,crowd", [(50_000, 27, None), (12_000, 1000, 10_000), (4000, 5000, 33)])
def test_noalloc_sort_crowded_cells(ffcm, N, ncell, crowd):
    """Crowded cells (more than 32 particles) are put in order by a block in
    shared memory, and a cell beyond 8192 by one thread; the result is the
    stable order either way, twice in a row."""
    torch = pytest.importorskip("torch")
    lib = ffcm._lib.load()
    sort = _noalloc(lib)
    rng = np.random.default_rng(N + ncell)
    k = rng.integers(0, ncell, N).astype(np.int32)
    if crowd is not None:
        k[rng.permutation(N)[:crowd]] = 7      # one cell with `crowd` (or more) particles
    key = torch.from_numpy(k).cuda()
    outs = [torch.empty(N, dtype=torch.int32, device="cuda"), torch.empty(ncell, dtype=torch.int32, device="cuda"),
            torch.empty(ncell, dtype=torch.int32, device="cuda")]
    counts = np.bincount(k, minlength=ncell)
    for _ in range(2):
        for o in outs:
            o.fill_(-7)
        rc = sort(key.data_ptr(), N, ncell, outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), None)
        assert rc == 0, ffcm._lib.last_error()
        np.testing.assert_array_equal(outs[0].cpu().numpy(), np.argsort(k, kind="stable") + 1)
        np.testing.assert_array_equal(outs[2].cpu().numpy(), np.cumsum(counts))
        np.testing.assert_array_equal(outs[1].cpu().numpy(), np.cumsum(counts) - counts + 1)
