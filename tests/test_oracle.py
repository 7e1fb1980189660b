"""CPU tests of the oracle (the C restatement of the reference) and of host logic.

The oracle is pinned against the FP64 direct sum (which it also restates) and
against the accuracy contract of each iprec (src/lfmm3dpart.f:156-165); the
committed fixture under tests/golden/ pins it against regressions.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle as O  # noqa: E402
from driver_inputs import driver_inputs  # noqa: E402

EPS = {-2: .5, -1: .5e-1, 0: .5e-2, 1: .5e-3, 2: .5e-6, 3: .5e-9}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_hkrand_first_value_is_dlaran_of_seed_0001():
    # dlaran (examples/dlaran.f:48-84) on seed (0,0,0,1): 494/4096 + ...
    v = O.hkrand_stream(3)
    assert abs(v[0] - (494 + (322 + (2508 + 2549 / 4096) / 4096) / 4096) / 4096) < 1e-15
    assert np.all((v > 0) & (v < 1))


def test_golden_fixture_reproduces():
    d = np.load(os.path.join(HERE, "golden", "driver_lap_n2000.npz"))
    assert np.array_equal(d["hkrand20"], O.hkrand_stream(20))
    src, trg, q, ds, dv = driver_inputs(2000)
    ier, pot, fld, pt, ft = O.lfmm3dparttarg(1, src, q, ds, dv, trg)
    assert ier == 0
    for a, b in ((pot, "pot"), (fld, "fld"), (pt, "pottarg"), (ft, "fldtarg")):
        assert rel(a[:100], d[b]) < 1e-12
    dp, df = O.direct_at(src, src[:100], np.arange(100), q, ds, dv)
    assert rel(dp, d["dpot"]) < 1e-14 and rel(df, d["dfld"]) < 1e-14


@pytest.mark.parametrize("eps,p", [(.5e-2, 9), (.5e-3, 14), (.5e-6, 26), (.5e-9, 39)])
def test_l3dterms_orders(eps, p):
    assert O.l3dterms(eps) == p


def test_list2_table_symmetry_and_range():
    t = O.l3dterms_list2(.5e-3)
    assert t[3 + 2, 3, 3] == 14          # offset (2,0,0): the worst case
    assert t.min() == 0 and t.max() == 14
    assert np.array_equal(t, t[::-1, :, :]) and np.array_equal(t, t[:, ::-1, :])
    assert t[3, 3, 3] == 0 and t[4, 4, 4] == 0   # near offsets are not in list 2


def test_iprec_tables():
    assert [O.lap_nbox(i, 10, 10) for i in range(-2, 6)] == [40, 50, 80, 160, 400, 800, 1200, 1400]
    assert O.lap_nbox(6, 10, 7) == 17
    assert O.lap_eps(1) == .5e-3


def test_direct_matches_numpy():
    rng = np.random.default_rng(0)
    n = 300
    src = rng.random((n, 3))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    ds = rng.normal(size=n) + 1j * rng.normal(size=n)
    dv = rng.normal(size=(n, 3))
    pot, fld, _, _ = O.l3dpartdirect(src, q, ds, dv)
    d = src[:, None, :] - src[None, :, :]
    r = np.linalg.norm(d, axis=2)
    np.fill_diagonal(r, np.inf)
    dot = np.einsum("ijk,jk->ij", d, dv)
    p = (q[None, :] / r).sum(1) + (ds[None, :] * dot / r ** 3).sum(1)
    f = (q[None, :, None] * d / r[..., None] ** 3).sum(1) + (
        ds[None, :, None] * (3 * dot[..., None] * d / r[..., None] ** 5 - dv[None, :, :] / r[..., None] ** 3)).sum(1)
    assert rel(pot, p) < 1e-13 and rel(fld, f) < 1e-13


@pytest.mark.parametrize("iprec", [-1, 0, 1, 2])
def test_oracle_fmm_within_bound(iprec):
    rng = np.random.default_rng(10 + iprec)
    n, m = 6000, 3000
    src = rng.random((n, 3))
    trg = rng.random((m, 3))
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ier, pot, fld, pt, ft = O.lfmm3dparttarg(iprec, src, q, None, None, trg)
    assert ier == 0
    k = 200
    si = rng.choice(n, k, replace=False)
    dp, df = O.direct_at(src, src[si], si, q)
    dpt, dft = O.direct_at(src, trg[:k], None, q)
    for a, b in ((pot[si], dp), (fld[si], df), (pt[:k], dpt), (ft[:k], dft)):
        assert rel(a, b) < EPS[iprec]


def test_oracle_operators_compose():
    # M2M then M2L then L2L then L2P equals the direct potential (far field)
    rng = np.random.default_rng(3)
    p = 20
    src = rng.random((30, 3)) * 0.5
    q = rng.normal(size=30) + 1j * rng.normal(size=30)
    c1 = np.array([.25, .25, .25])
    mp = O.formmp(src, c1, p, charge=q)
    c2 = np.array([.5, .5, .5])
    mp2 = O.translate(0, c1, c2, mp, p)
    c3 = c2 + np.array([3.0, 1.0, -1.0])
    lo = O.translate(1, c2, c3, mp2, p)
    c4 = c3 + np.array([.25, -.25, .25])
    lo2 = O.translate(2, c3, c4, lo, p)
    t = c4 + np.array([[.1, .05, -.1]])
    pv, fv = O.taeval(c4, lo2, p, t)
    dp, df = O.direct_at(src, t, None, q)
    assert rel(pv, dp) < 1e-7 and rel(fv, df) < 1e-6
