"""Error paths of the drop-in entry points, made on the host (no GPU fault).

The reference reports workspace failures as ier 4 (tree), 8 (per-point
workspace) and 16 (expansion workspace) and returns without writing the
outputs (src/lfmm3dpart.f:309-330, 424-466; src/hfmm3dpart.f likewise).
Here an allocation failure is injected on the host (fmm3d_inject_alloc_failure
fails the first device allocation of one phase of the next call, as if the
device were out of memory) in each phase in turn: the call must return that
phase's code, leave the caller's outputs untouched, and the next call must
succeed with the same results as before.  The tensor-core
M2L's bounded waits are exercised by fmm3d_inject_tc_wait_expiry: its kernel
then takes its error path (drains the MMAs it issued, frees TMEM, flags the
error) and the call returns 16, after which the context is still usable.
Per-thread switch overrides are checked not to leak into other threads.
"""
import ctypes
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import fmmlib3d_b200
    lib = fmmlib3d_b200.lib()
    for name in ("fmm3d_inject_alloc_failure", "fmm3d_inject_tc_wait_expiry", "fmm3d_set_switch_thread"):
        getattr(lib, name).restype = ctypes.c_int
        getattr(lib, name).argtypes = [ctypes.c_int] * (2 if name == "fmm3d_set_switch_thread" else 1)
    return fmmlib3d_b200


def _inputs(n, m, seed):
    rng = np.random.default_rng(seed)
    src, trg = rng.random((n, 3)), rng.random((m, 3))
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    dv = rng.normal(size=(n, 3))
    return src, q, ds, dv, trg


def _call(F, kernel, iprec, src, q, ds, dv, trg, fill=np.nan):
    """One host-array call through the C ABI with NaN-filled outputs; returns (ier, outputs)."""
    lib = F.lib()
    n, m = len(src), len(trg)
    outs = [np.full(n, fill, np.complex128), np.full((n, 3), fill, np.complex128),
            np.full(m, fill, np.complex128), np.full((m, 3), fill, np.complex128)]
    P = lambda a: ctypes.c_void_p(a.ctypes.data)
    I = lambda v: ctypes.byref(ctypes.c_int(v))
    ier = ctypes.c_int(-1)
    zk = np.array([3.0, 0.2])
    head = [ctypes.byref(ier), I(iprec)] + ([P(zk)] if kernel == "helmholtz" else [])
    fn = lib.lfmm3dparttarg_ if kernel == "laplace" else lib.hfmm3dparttarg_
    src, trg, q, ds, dv = [np.ascontiguousarray(a) for a in (src, trg, q, ds, dv)]
    fn(*head, I(n), P(src), I(1), P(q), I(1), P(ds), P(dv), I(1), P(outs[0]), I(1), P(outs[1]), I(m), P(trg), I(1),
       P(outs[2]), I(1), P(outs[3]))
    return ier.value, outs


@pytest.mark.parametrize("kernel,precision", [("laplace", 0), ("laplace", 1), ("helmholtz", 0)])
def test_injected_allocation_failures_return_reference_codes(F, kernel, precision):
    args = _inputs(30000, 8000, 3)
    F.set_precision(precision)
    lib = F.lib()
    try:
        ier, good = _call(F, kernel, 1, *args)   # warm: per-device caches built
        assert ier == 0, F.last_error()
        # phase -> the reference's code: host copies 8, tree 4, per-point workspace 8, expansions 16
        for phase, code in ((1, 8), (2, 4), (3, 8), (4, 16)):
            assert lib.fmm3d_inject_alloc_failure(phase) == 0
            ier, outs = _call(F, kernel, 1, *args)
            assert ier == code, (phase, ier, F.last_error())
            for o in outs:
                assert np.all(np.isnan(o)), "outputs written by a failed call (phase %d)" % phase
            ier, again = _call(F, kernel, 1, *args)   # one call only; the next one succeeds, same bits
            assert ier == 0, F.last_error()
            for a, b in zip(again, good):
                assert np.array_equal(a, b)
        assert lib.fmm3d_inject_alloc_failure(5) == 1
    finally:
        lib.fmm3d_inject_alloc_failure(0)
        F.set_precision(0)


def test_tensor_core_m2l_wait_expiry_returns_16_and_context_stays_usable(F):
    import torch
    args = _inputs(60000, 20000, 4)
    F.set_precision(1)
    F.set_tensor_m2l(1)
    try:
        ier, good = _call(F, "laplace", 1, *args)
        assert ier == 0, F.last_error()
        F.lib().fmm3d_inject_tc_wait_expiry(1)
        try:
            ier, outs = _call(F, "laplace", 1, *args)
        finally:
            F.lib().fmm3d_inject_tc_wait_expiry(0)
        assert ier == 16
        assert "wait expired" in F.last_error()
        for o in outs:
            assert np.all(np.isnan(o))
        torch.cuda.synchronize()   # no sticky CUDA error
        ier, again = _call(F, "laplace", 1, *args)
        assert ier == 0, F.last_error()
        for a, b in zip(again, good):
            assert np.array_equal(a, b)
    finally:
        F.set_precision(0)


def test_switch_override_is_per_thread(F):
    """A thread's override (here: the mixed form) changes its own calls only; a thread without an
    override keeps the process-wide form (FP64), bitwise."""
    args = _inputs(20000, 5000, 5)
    lib = F.lib()
    ier, fp64 = _call(F, "laplace", 1, *args)
    assert ier == 0
    F.set_precision(1)
    ier, mixed = _call(F, "laplace", 1, *args)
    F.set_precision(0)
    assert ier == 0
    assert not np.array_equal(mixed[0], fp64[0])
    res = {}

    def worker(name, override):
        if override is not None:
            assert lib.fmm3d_set_switch_thread(1, override) == 0
        res[name] = _call(F, "laplace", 1, *args)

    ts = [threading.Thread(target=worker, args=("mixed", 1)), threading.Thread(target=worker, args=("plain", None))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert res["mixed"][0] == 0 and res["plain"][0] == 0
    for a, b in zip(res["mixed"][1], mixed):
        assert np.array_equal(a, b)
    for a, b in zip(res["plain"][1], fp64):
        assert np.array_equal(a, b)
    assert lib.fmm3d_set_switch_thread(1, 2) == 1 and lib.fmm3d_set_switch_thread(7, 0) == 1
