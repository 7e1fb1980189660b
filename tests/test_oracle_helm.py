"""CPU tests of the Helmholtz half of the oracle (hfmm3d_oracle.c).

The special functions are checked against scipy's independent
implementations; the expansion orders against the values the reference's
formulas give for a sphere of radius 1 at zk = 8 pi (67, 42, 31, 26, 24, 23, 23
for levels 0..6); the FMM against the FP64 direct sum it also restates, within
the accuracy contract of each iprec (src/hfmm3dpart.f:156-166); and the
committed fixture of the reference driver's inputs against regressions.
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


@pytest.mark.parametrize("z", [1e-3, 0.3, 2.5 + 0.1j, 12.0, 30 + 1j])
def test_bessel_hankel_match_scipy(z):
    sp = pytest.importorskip("scipy.special")
    n = 20
    nn = np.arange(n + 1)
    h, _ = O.h3dall(n, z, 1.0)
    ier, f, fd = O.jfuns3d(n, z, 1.0)
    assert ier == 0
    jr, yr = sp.spherical_jn(nn, z), sp.spherical_yn(nn, z)
    assert np.max(np.abs(f - jr) / np.abs(jr)) < 1e-12
    assert np.max(np.abs(h - (jr + 1j * yr)) / np.abs(jr + 1j * yr)) < 1e-12
    jd = sp.spherical_jn(nn, z, derivative=True)
    assert np.max(np.abs(fd - jd) / np.abs(jd)) < 1e-12


def test_scaled_functions_carry_scale_powers():
    z, s, n = 0.2 + 0.05j, 0.25, 12
    h1, _ = O.h3dall(n, z, 1.0)
    hs, _ = O.h3dall(n, z, s)
    _, j1, _ = O.jfuns3d(n, z, 1.0)
    _, js, _ = O.jfuns3d(n, z, s)
    k = np.arange(n + 1)
    assert np.allclose(hs, h1 * s ** k, rtol=1e-12, atol=0)
    assert np.allclose(js, j1 / s ** k, rtol=1e-12, atol=0)


def test_h3dterms_orders_at_the_sphere_workload():
    # sphere of radius 1 -> bounding cube of side 2; zk = 8 pi, iprec = 2
    got = [O.h3dterms(2.0 / 2 ** lev, 8 * np.pi, .5e-6)[0] for lev in range(7)]
    assert got == [67, 42, 31, 26, 24, 23, 23]


def test_h3dterms_list2_table():
    t = O.h3dterms_list2(0.25, 8 * np.pi, .5e-6)
    p = O.h3dterms(0.25, 8 * np.pi, .5e-6)[0]
    assert t[3, 3, 3] == 0 and t[4, 4, 4] == 0
    assert 0 < t[5, 3, 3] <= p + 1 and t.max() == t[5, 3, 3]
    assert np.array_equal(t, t[::-1, :, :]) and np.array_equal(t, t[:, :, ::-1])


def test_gauss_legendre_exactness():
    for n in (6, 17, 40):
        x, w = O.legewhts(n)
        assert np.all(np.diff(x) > 0)
        for k in (0, 2, 2 * n - 2):
            assert abs(np.sum(w * x ** k) - 2.0 / (k + 1)) < 1e-13


def test_helmholtz_direct_matches_numpy():
    rng = np.random.default_rng(5)
    n, m, zk = 60, 25, 3 + 0.2j
    src, trg = rng.random((n, 3)), rng.random((m, 3)) + 1
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    ds = rng.normal(size=n) + 1j * rng.normal(size=n)
    dv = rng.normal(size=(n, 3))
    pot, fld, pt, ft = O.h3dpartdirect(zk, src, q, ds, dv, trg)

    def field(x):
        r = x[None, :] - src
        d = np.linalg.norm(r, axis=1)
        ok = d > 0
        r, d, qq, dd, vv = r[ok], d[ok], q[ok], ds[ok], dv[ok]
        g = np.exp(1j * zk * d) / d
        gp = g * (1j * zk - 1 / d)               # dG/dd
        gpp = g * ((1j * zk - 1 / d) ** 2 + 1 / d ** 2)
        u = r / d[:, None]
        vu = np.sum(vv * u, axis=1)
        # a dipole is dipvec . grad_source G = -G'(d) (u . dipvec)
        p = np.sum(qq * g) - np.sum(dd * gp * vu)
        grad_q = (qq * gp)[:, None] * u
        grad_d = dd[:, None] * (gpp * vu)[:, None] * u + (dd * gp / d)[:, None] * (vv - vu[:, None] * u)
        return p, grad_d.sum(0) - grad_q.sum(0)

    for k in range(n):
        p, f = field(src[k])
        assert abs(pot[k] - p) <= 1e-12 * abs(p) and np.linalg.norm(fld[k] - f) <= 1e-12 * np.linalg.norm(f)
    for k in range(m):
        p, f = field(trg[k])
        assert abs(pt[k] - p) <= 1e-12 * abs(p) and np.linalg.norm(ft[k] - f) <= 1e-12 * np.linalg.norm(f)


def test_helmholtz_operators_compose():
    # P2M -> M2M -> M2L -> L2L -> L2P against the direct sum, at zk = 4
    rng = np.random.default_rng(7)
    zk, p, s = 4.0 + 0.0j, 20, 0.125
    c0 = np.array([0.0625, 0.0625, 0.0625])           # child of a level-3 box
    src = c0 + (rng.random((40, 3)) - 0.5) * s
    q = rng.normal(size=40) + 1j * rng.normal(size=40)
    sc = min(1.0, abs(zk) * s)
    mp = O.hformmp(zk, sc, src, c0, p, charge=q)
    cp = np.array([0.125, 0.125, 0.125])               # parent, side 2 s
    sc2 = min(1.0, abs(zk) * 2 * s)
    mpp = O.htranslate(0, zk, c0, cp, mp, p, sc, p, sc2, np.sqrt(3) * s, max(6, int(2.5 * p)))
    t_c = cp + np.array([0.75, 0.0, 0.0])              # separated by 3 boxes of side 2 s
    lo = O.htranslate(1, zk, cp, t_c, mpp, p, sc2, p, sc2, np.sqrt(3) * s, max(6, int(1.2 * p)))
    t_k = t_c + np.array([s / 2, -s / 2, s / 2])        # child of the target box
    lok = O.htranslate(2, zk, t_c, t_k, lo, p, sc2, p, sc, np.sqrt(3) / 2 * s, 2 * p)
    pts = t_k + (rng.random((30, 3)) - 0.5) * s
    pot, fld = O.htaeval(zk, sc, t_k, lok, p, pts)
    dp, df = O.hdirect_at(zk, src, pts, None, q)
    assert rel(pot, dp) < 1e-7 and rel(fld, df) < 1e-6
    # the multipole and the local expansion also evaluate directly
    mpot, mfld = O.hmpeval(zk, sc2, cp, mpp, p, pts)
    assert rel(mpot, dp) < 1e-8 and rel(mfld, df) < 1e-7
    lo4 = O.hformta(zk, sc, src, t_k, p, charge=q)
    lpot, lfld = O.htaeval(zk, sc, t_k, lo4, p, pts)
    assert rel(lpot, dp) < 1e-8 and rel(lfld, df) < 1e-7


@pytest.mark.parametrize("iprec,zk,geom", [(0, 3.0, "cube"), (1, 1 + 0.1j, "cube"), (2, 10.0, "cube"),
                                           (2, 8 * np.pi, "sphere"), (1, 30.0, "cube"),
                                           (1, 1 + 10j, "cube"), (2, 0.5 + 6j, "sphere")])
def test_helmholtz_fmm_within_bound(iprec, zk, geom):
    rng = np.random.default_rng(11 + iprec)
    n, m = 12000, 3000
    if geom == "sphere":
        v = rng.normal(size=(n, 3))
        src = v / np.linalg.norm(v, axis=1)[:, None]
    else:
        src = rng.random((n, 3))
    trg = rng.random((m, 3)) * 0.9
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    dv = rng.normal(size=(n, 3))
    ier, pot, fld, pt, ft = O.hfmm3dparttarg(iprec, zk, src, q, ds, dv, trg)
    assert ier == 0
    idx = np.arange(0, n, n // 150)
    jdx = np.arange(0, m, m // 100)
    dp, df = O.hdirect_at(zk, src, src[idx], idx, q, ds, dv)
    tp, tf = O.hdirect_at(zk, src, trg[jdx], None, q, ds, dv)
    for a, b in ((pot[idx], dp), (fld[idx], df), (pt[jdx], tp), (ft[jdx], tf)):
        assert rel(a, b) < EPS[iprec]


def test_helmholtz_golden_fixture_reproduces():
    d = np.load(os.path.join(HERE, "golden", "driver_helm_n2000.npz"))
    src, trg, q, ds, dv = driver_inputs(2000, shift=1.0)
    zk = complex(d["zk"])
    ier, pot, fld, pt, ft = O.hfmm3dparttarg(1, zk, src, q, ds, dv, trg)
    assert ier == 0
    for a, b in ((pot, "pot"), (fld, "fld"), (pt, "pottarg"), (ft, "fldtarg")):
        assert rel(a[:100], d[b]) < 1e-12
        assert rel(a[:100], d["d" + b]) < EPS[1]


@pytest.mark.parametrize("p", [12, 30, 31, 40, 67])
def test_rotation_by_projection_matches_recursion_and_is_unitary(p):
    """rotviaprojf90 (the reference's rotation for orders >= 30, src/rotproj.f:883) and the
    recursion of rotviarecur3 give the same rotation where the recursion is stable; the
    projection preserves the norm (the rotation is unitary) and -beta undoes +beta at every
    order, including those where the recursion drifts."""
    rng = np.random.default_rng(p)
    a = rng.normal(size=(p + 1) ** 2) + 1j * rng.normal(size=(p + 1) ** 2)
    for beta in (0.3, -1.1, 2.5):
        x = O.rotviaproj(beta, p, a)
        assert abs(np.linalg.norm(x) - np.linalg.norm(a)) < 1e-13 * np.linalg.norm(a)
        assert rel(O.rotviaproj(-beta, p, x), a) < 1e-13
        if p <= 40:
            assert rel(x, O.rotviarecur(beta, p, a)) < 1e-12
