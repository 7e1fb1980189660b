"""The allocation-free direct sum (fmm3d_l3dpartdirect_noalloc) against the regular one.

Callers whose GPU memory is owned by another allocator, or whose service loop
forbids cudaMalloc/cudaFree after start-up, use the allocation-free entry
point; it must give the same values as fmm3d_l3dpartdirect_device (within
the direct-sum tolerance of these tests, 1e-13 relative) on consecutive calls,
since all calls share one scratch array in the library's device image.
This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _call(fn, torch, src, q, ds, dv, trg, want_src=True):
    n, m = src.shape[0], trg.shape[0]
    dev = "cuda"
    pot = torch.full((n, 2), np.nan, dtype=torch.float64, device=dev)
    fld = torch.full((n, 6), np.nan, dtype=torch.float64, device=dev)
    pt = torch.full((m, 2), np.nan, dtype=torch.float64, device=dev)
    ft = torch.full((m, 6), np.nan, dtype=torch.float64, device=dev)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ier = fn(n, P(src), 1, P(q), 1, P(ds), P(dv), int(want_src), P(pot), int(want_src), P(fld), m, P(trg), 1,
             P(pt), 1, P(ft), s)
    torch.cuda.synchronize()
    return ier, pot.cpu().numpy(), fld.cpu().numpy(), pt.cpu().numpy(), ft.cpu().numpy()


def _inputs(torch, n, m, seed):
    rng = np.random.default_rng(seed)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dv = rng.normal(size=(n, 3))
    return (d(rng.random((n, 3))), d(rng.uniform(-1, 1, (n, 2))), d(rng.uniform(-1, 1, (n, 2))), d(dv),
            d(rng.random((m, 3)) + 0.5))


def test_noalloc_direct_matches_allocating_direct_on_consecutive_calls():
    import torch
    import fmmlib3d_b200 as F
    lib = F.lib()
    for fn_name in ("fmm3d_l3dpartdirect_noalloc", "fmm3d_l3dpartdirect_device"):
        getattr(lib, fn_name).restype = ctypes.c_int
    lib.fmm3d_noalloc_last_error.restype = ctypes.c_char_p
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    # two calls in a row with different sizes and inputs: the second must not
    # see anything the first left in the shared scratch array
    for (n, m, seed) in ((40000, 20000, 1), (9000, 3000, 2)):
        args = _inputs(torch, n, m, seed)
        got = _call(lib.fmm3d_l3dpartdirect_noalloc, torch, *args)
        want = _call(lib.fmm3d_l3dpartdirect_device, torch, *args)
        assert got[0] == 0, lib.fmm3d_noalloc_last_error()
        assert want[0] == 0
        for a, b in zip(got[1:], want[1:]):
            assert np.all(np.isfinite(a))
            assert rel(a, b) < TOL


def test_noalloc_direct_rejects_sizes_above_its_limit():
    import torch
    import fmmlib3d_b200 as F
    lib = F.lib()
    lib.fmm3d_l3dpartdirect_noalloc.restype = ctypes.c_int
    lib.fmm3d_noalloc_last_error.restype = ctypes.c_char_p
    args = _inputs(torch, 65537, 10, 3)
    ier = _call(lib.fmm3d_l3dpartdirect_noalloc, torch, *args)[0]
    assert ier == 8
    assert b"65536" in lib.fmm3d_noalloc_last_error()
