"""The serving loop (fmmlib3d_b200.serving): requests in a mix equal requests alone.

Requests of both kernels, several sizes, iprec values and geometries are
submitted together to a server with four slots (their kernels overlap on the
GPU), then one at a time; every result must be bitwise identical, and equal
to the plain C-ABI call.  A budget smaller than any request forces one
request at a time.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(count, seed):
    from fmmlib3d_b200.serving import Request
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(10 ** rng.uniform(3, 4.5))
        src = rng.random((n, 3)) if i % 2 else rng.normal(size=(n, 3)) * 0.2
        q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        helm = i % 3 == 0
        out.append(Request("helmholtz" if helm else "laplace", src, q, iprec=int(rng.integers(0, 3)),
                           zk=float(rng.uniform(1, 20)) if helm else 0.0, tag=i))
    return out


def test_results_equal_alone_and_in_the_mix():
    from fmmlib3d_b200.serving import FMMServer, run_stream
    import fmmlib3d_b200 as F
    reqs = _requests(12, 3)
    srv = FMMServer(slots=4)
    try:
        stats, mixed = run_stream(srv, reqs, float("inf"))
    finally:
        srv.close()
    assert stats["max_ier"] == 0 and srv.max_running > 1
    srv1 = FMMServer(slots=1)
    try:
        alone = [srv1.submit(r).result() for r in reqs]
    finally:
        srv1.close()
    for r, a, b in zip(reqs, mixed, alone):
        assert a.tag == b.tag == r.tag
        assert np.array_equal(a.pot, b.pot) and np.array_equal(a.fld, b.fld)
        if r.kernel == "laplace":
            ier, pot, fld, _, _ = F.lfmm3dparttarg(r.iprec, r.source, 1, r.charge, 0, None, None, 1, 1)
        else:
            ier, pot, fld, _, _ = F.hfmm3dparttarg(r.iprec, r.zk, r.source, 1, r.charge, 0, None, None, 1, 1)
        assert ier == 0 and np.array_equal(a.pot, pot) and np.array_equal(a.fld, fld)


def test_budget_limits_concurrency():
    from fmmlib3d_b200.serving import FMMServer, run_stream
    reqs = _requests(6, 4)
    srv = FMMServer(slots=4, hbm_budget_bytes=1)
    try:
        stats, _ = run_stream(srv, reqs, float("inf"))
    finally:
        srv.close()
    assert stats["max_ier"] == 0 and srv.max_running == 1


def test_precision_per_request():
    """A server in the mixed form (and requests that override it) gives every request the bits of a
    single call in that request's form; the process-wide setting is left as it was."""
    from fmmlib3d_b200.serving import FMMServer, run_stream
    import fmmlib3d_b200 as F
    reqs = _requests(10, 5)
    for i, r in enumerate(reqs):
        if r.kernel == "laplace" and i % 4 == 1:
            r.precision = 0
    srv = FMMServer(slots=4, precision=1)
    try:
        stats, res = run_stream(srv, reqs, float("inf"))
    finally:
        srv.close()
    assert stats["max_ier"] == 0
    for r, a in zip(reqs, res):
        form = 1 if r.precision is None else r.precision
        if r.kernel == "laplace":
            F.set_precision(form)
            try:
                ier, pot, fld, _, _ = F.lfmm3dparttarg(r.iprec, r.source, 1, r.charge, 0, None, None, 1, 1)
            finally:
                F.set_precision(0)
        else:
            ier, pot, fld, _, _ = F.hfmm3dparttarg(r.iprec, r.zk, r.source, 1, r.charge, 0, None, None, 1, 1)
        assert ier == 0 and np.array_equal(a.pot, pot) and np.array_equal(a.fld, fld), (r.tag, r.kernel, r.iprec)
    with pytest.raises(ValueError):
        F.set_precision_thread(2)


def test_repeated_geometries_run_on_resident_plans():
    """Laplace requests naming a repeated geometry run on a plan kept on the device: after the
    first request of each geometry no tree is rebuilt (plan hits), every result carries the bits of
    a plain call, and a plan budget smaller than two plans evicts the least recently used one and
    still gives the same bits."""
    from fmmlib3d_b200.serving import FMMServer, Request, run_stream
    import fmmlib3d_b200 as F
    rng = np.random.default_rng(9)
    geoms = [(rng.random((20000, 3)), 1), (rng.normal(size=(8000, 3)) * 0.3, 0), (rng.random((3000, 3)), 2)]
    reqs = []
    for i in range(18):
        g = i % 3
        src, iprec = geoms[g]
        q = rng.uniform(-1, 1, len(src)) + 1j * rng.uniform(-1, 1, len(src))
        reqs.append(Request("laplace", src, q, iprec=iprec, tag=i, geometry=g))
    want = []
    for r in reqs:
        ier, pot, fld, _, _ = F.lfmm3dparttarg(r.iprec, r.source, 1, r.charge, 0, None, None, 1, 1)
        assert ier == 0
        want.append((pot, fld))
    for plan_bytes in (None, 1):
        srv = FMMServer(slots=4, plan_bytes=plan_bytes)
        try:
            stats, res = run_stream(srv, reqs, float("inf"))
            st = srv.stats()
        finally:
            srv.close()
        assert stats["max_ier"] == 0
        for r, a, (pot, fld) in zip(reqs, res, want):
            assert a.tag == r.tag
            assert np.array_equal(a.pot, pot) and np.array_equal(a.fld, fld)
        if plan_bytes is None:
            assert st["plans_built"] == 3 and st["plan_hits"] == 15 and st["plans_evicted"] == 0
        else:
            assert st["plans_evicted"] >= 1
