"""The allocation-free direct sum (fmm3d_l3dpartdirect_noalloc).

Some callers cannot let this library allocate device memory: an application
whose framework allocator already owns the GPU's memory, or a service loop
that forbids cudaMalloc/cudaFree (which synchronise the device) once it is
running.  They call fmm3d_l3dpartdirect_noalloc, whose scratch is one fixed
array in the library's device image.  These tests check, through the C ABI:

* its values against the oracle's l3dpartdirect (the restatement of the
  reference's O(N^2) sum) and against fmm3d_l3dpartdirect_device, within the
  direct-sum tolerance of these tests (1e-13 relative), on two calls in a row
  with different sizes (every call shares the scratch array, so the second
  must not see what the first left there);
* every flag combination: charge only, dipole only, both; outputs whose flag
  is not 1 keep the caller's contents; a call with no sources gives zero
  target outputs, as the reference;
* that after the first call on the device (the set-up, which may load the
  array and kernels) calls allocate nothing: the device's free memory and the
  default memory pool's high-water mark are unchanged across calls;
* the size limit (ier 8 with a message, GPU untouched).

This file is collected last so that a run stopping at its first failure has
already run every other test; it passes alone in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _lib():
    import fmmlib3d_b200 as F
    lib = F.lib()
    for name in ("fmm3d_l3dpartdirect_noalloc", "fmm3d_l3dpartdirect_device"):
        getattr(lib, name).restype = ctypes.c_int
    lib.fmm3d_noalloc_last_error.restype = ctypes.c_char_p
    return lib


def _inputs(n, m, seed):
    rng = np.random.default_rng(seed)
    dv = rng.normal(size=(n, 3))
    return (rng.random((n, 3)), rng.uniform(-1, 1, (n, 2)), rng.uniform(-1, 1, (n, 2)), dv,
            rng.random((m, 3)) + 0.5)


def _call(fn, torch, arrs, ifc=1, ifd=1, flags=(1, 1, 1, 1)):
    """One call on device copies of arrs; outputs start as NaN so that untouched ones are visible."""
    src, q, ds, dv, trg = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]
    n, m = src.shape[0], trg.shape[0]
    outs = [torch.full(s, np.nan, dtype=torch.float64, device="cuda")
            for s in ((max(n, 1), 2), (max(n, 1), 6), (max(m, 1), 2), (max(m, 1), 6))]
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ier = fn(n, P(src), ifc, P(q), ifd, P(ds), P(dv), flags[0], P(outs[0]), flags[1], P(outs[1]), m, P(trg),
             flags[2], P(outs[2]), flags[3], P(outs[3]), s)
    torch.cuda.synchronize()
    c = lambda t, k: t.cpu().numpy()[:k]
    return ier, (c(outs[0], n), c(outs[1], n), c(outs[2], m), c(outs[3], m))


def _oracle(arrs, ifc, ifd, flags):
    import oracle as O
    src, q, ds, dv, trg = arrs
    z = lambda a: a[:, 0] + 1j * a[:, 1]
    pot, fld, pt, ft = O.l3dpartdirect(src, z(q) if ifc else None, z(ds) if ifd else None, dv if ifd else None, trg,
                                       *flags)
    r = lambda a, w: np.stack([a.real, a.imag], -1).reshape(len(a), w)
    return r(pot, 2), r(fld, 6), r(pt, 2), r(ft, 6)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _pool_high(dev=0):
    """High-water mark of used memory in the device's default memory pool (the pool this library's
    stream-ordered allocations come from), reset to the current use after reading."""
    from cuda.bindings import driver as drv
    (err,) = drv.cuInit(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    err, pool = drv.cuDeviceGetDefaultMemPool(dev)
    assert err == drv.CUresult.CUDA_SUCCESS
    A = drv.CUmemPool_attribute
    err, high = drv.cuMemPoolGetAttribute(pool, A.CU_MEMPOOL_ATTR_USED_MEM_HIGH)
    assert err == drv.CUresult.CUDA_SUCCESS
    (err,) = drv.cuMemPoolSetAttribute(pool, A.CU_MEMPOOL_ATTR_USED_MEM_HIGH, drv.cuuint64_t(0))
    assert err == drv.CUresult.CUDA_SUCCESS
    return int(high)


def test_noalloc_direct_matches_oracle_and_device_sum_on_consecutive_calls():
    import torch
    lib = _lib()
    _call(lib.fmm3d_l3dpartdirect_noalloc, torch, _inputs(100, 50, 9))   # set-up call on this device
    for (n, m, seed) in ((20000, 8000, 1), (7000, 3000, 2)):
        arrs = _inputs(n, m, seed)
        ier, got = _call(lib.fmm3d_l3dpartdirect_noalloc, torch, arrs)
        assert ier == 0, lib.fmm3d_noalloc_last_error()
        ier2, dev = _call(lib.fmm3d_l3dpartdirect_device, torch, arrs)
        assert ier2 == 0
        want = _oracle(arrs, 1, 1, (1, 1, 1, 1))
        for a, b, w in zip(got, dev, want):
            assert np.all(np.isfinite(a))
            assert _rel(a, w) < TOL
            assert _rel(a, b) < TOL


@pytest.mark.parametrize("ifc,ifd", [(1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("flags", [(1, 0, 0, 1), (0, 1, 1, 0), (0, 0, 1, 1), (1, 1, 0, 0)])
def test_noalloc_direct_flag_combinations(ifc, ifd, flags):
    import torch
    lib = _lib()
    arrs = _inputs(3000, 1500, 11 + ifc + 2 * ifd)
    ier, got = _call(lib.fmm3d_l3dpartdirect_noalloc, torch, arrs, ifc, ifd, flags)
    assert ier == 0, lib.fmm3d_noalloc_last_error()
    want = _oracle(arrs, ifc, ifd, flags)
    for a, w, f in zip(got, want, flags):
        if f == 1:
            assert _rel(a, w) < TOL
        else:
            assert np.all(np.isnan(a)), "an output whose flag is not 1 was written"


def test_noalloc_direct_without_sources_gives_zero_targets():
    import torch
    lib = _lib()
    arrs = _inputs(0, 700, 21)
    ier, got = _call(lib.fmm3d_l3dpartdirect_noalloc, torch, arrs)
    assert ier == 0, lib.fmm3d_noalloc_last_error()
    assert np.all(got[2] == 0) and np.all(got[3] == 0)


def test_noalloc_direct_allocates_nothing_after_setup():
    import torch
    lib = _lib()
    fn = lib.fmm3d_l3dpartdirect_noalloc
    arrs = [_inputs(30000, 12000, 31), _inputs(5000, 65536, 32)]
    d = [[torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in x] for x in arrs]
    outs = [[torch.empty(s, dtype=torch.float64, device="cuda")
             for s in ((x[0].shape[0], 2), (x[0].shape[0], 6), (x[4].shape[0], 2), (x[4].shape[0], 6))] for x in d]
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call(k):
        src, q, ds, dv, trg = d[k]
        o = outs[k]
        return fn(src.shape[0], P(src), 1, P(q), 1, P(ds), P(dv), 1, P(o[0]), 1, P(o[1]), trg.shape[0], P(trg), 1,
                  P(o[2]), 1, P(o[3]), s)

    assert call(0) == 0, lib.fmm3d_noalloc_last_error()   # set-up (module loading) on this device
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _pool_high()
    base = _pool_high()
    for k in (1, 0, 1):
        assert call(k) == 0, lib.fmm3d_noalloc_last_error()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, "device free memory changed across a call"
        assert _pool_high() <= base, "the default memory pool was drawn on during a call"


def test_noalloc_direct_rejects_sizes_above_its_limit():
    import torch
    lib = _lib()
    for n, m in ((65537, 10), (10, 65537), (-1, 10)):
        arrs = _inputs(max(n, 0), max(m, 0), 3)
        src, q, ds, dv, trg = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]
        out = torch.zeros((max(n, m, 1), 6), dtype=torch.float64, device="cuda")
        P = lambda t: ctypes.c_void_p(t.data_ptr())
        ier = lib.fmm3d_l3dpartdirect_noalloc(n, P(src), 1, P(q), 1, P(ds), P(dv), 1, P(out), 1, P(out), m, P(trg),
                                              1, P(out), 1, P(out), None)
        assert ier == 8
        assert b"65536" in lib.fmm3d_noalloc_last_error()
        assert float(out.abs().sum()) == 0.0
