"""The oracle's triangle-FMM restatement (CPU only).

Pins the closed forms of the exact integrals that the reference's near field
evaluates (direct3dtritarglaps2 / lapd2 and the self terms,
src/triquadflatlib.f:147-818, via triahquad, src/triahquad.f:63):
  - S, grad S, D, grad D against brute-force quadrature on 4^k subtriangles,
    above, below, beside and close to the triangle;
  - the in-plane (self) values against the average of the limits from the two
    sides, which is what the reference's iquad = 0 branch takes;
  - the collapsed Gauss-Legendre rules integrate every monomial up to the
    reference's degree (nqtri) exactly;
  - the oracle FMM (lfmm3dtriatarg) reaches its own direct sum
    (l3dtriadirect) within the iprec bound, with charges, dipoles, targets.
"""
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402
sys.path.insert(0, os.path.join(HERE, "..", "fmmlib3d_b200"))
from meshes import icosphere, normals_centroids, two_spheres  # noqa: E402  (numpy only; no library load)

EPS = {-1: .5e-1, 0: .5e-2, 1: .5e-3, 2: .5e-6, 3: .5e-9}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _rule(n):
    x, w = np.polynomial.legendre.leggauss(n)
    u, wu = (x + 1) / 2, w / 2
    U, V = np.meshgrid(u, u, indexing="ij")
    WU, WV = np.meshgrid(wu, wu, indexing="ij")
    return U.ravel(), ((1 - U) * V).ravel(), (2 * WU * WV * (1 - U)).ravel()


def _subdivide(tri, k):
    out = [tri]
    for _ in range(k):
        new = []
        for a, b, c in out:
            ab, bc, ca = (a + b) / 2, (b + c) / 2, (c + a) / 2
            new += [np.array([a, ab, ca]), np.array([ab, b, bc]), np.array([ca, bc, c]), np.array([ab, bc, ca])]
        out = new
    return out


def brute(tri, x, k, n=20):
    xi, eta, ww = _rule(n)
    nrm = np.cross(tri[1] - tri[0], tri[2] - tri[0])
    nrm /= np.linalg.norm(nrm)
    S, gS, D, gD = 0.0, np.zeros(3), 0.0, np.zeros(3)
    for t in _subdivide(tri, k):
        e1, e2 = t[1] - t[0], t[2] - t[0]
        w = ww * 0.5 * np.linalg.norm(np.cross(e1, e2))
        d = x - (t[0] + xi[:, None] * e1 + eta[:, None] * e2)
        r = np.linalg.norm(d, axis=1)
        nd = d @ nrm
        S += np.sum(w / r)
        gS -= np.sum(w[:, None] * d / r[:, None] ** 3, axis=0)
        D += np.sum(w * nd / r ** 3)
        gD += np.sum(w[:, None] * (nrm / r[:, None] ** 3 - 3 * nd[:, None] * d / r[:, None] ** 5), axis=0)
    return S, gS, D, gD


TRI = np.array([[0.1, 0.2, 0.0], [1.0, 0.1, 0.2], [0.3, 0.9, -0.1]])


@pytest.mark.parametrize("x,k,tol", [((0.4, 0.4, 0.8), 2, 1e-13), ((2.0, 1.0, 0.5), 1, 1e-13),
                                     ((0.45, 0.4, -0.05), 5, 1e-12), ((-0.3, 0.1, 0.05), 5, 1e-12),
                                     ((0.6, -0.4, 0.0), 4, 1e-12)])
def test_closed_forms_match_quadrature(x, k, tol):
    x = np.array(x)
    S, gS, D, gD = O.tri_near(TRI, x[None])
    bS, bgS, bD, bgD = brute(TRI, x, k)
    assert abs(S[0] - bS) <= tol * abs(bS)
    assert np.abs(gS[0] - bgS).max() <= tol * np.abs(bgS).max()
    assert abs(D[0] - bD) <= tol * max(abs(bD), 1e-3)
    assert np.abs(gD[0] - bgD).max() <= tol * np.abs(bgD).max()


def test_self_values_are_the_average_of_the_two_sides():
    c = TRI.mean(axis=0)
    n = np.cross(TRI[1] - TRI[0], TRI[2] - TRI[0])
    n /= np.linalg.norm(n)
    S0, gS0, D0, gD0 = O.tri_near(TRI, c[None], self=True)
    e = 1e-8
    Sa, gSa, Da, gDa = O.tri_near(TRI, (c + e * n)[None])
    Sb, gSb, Db, gDb = O.tri_near(TRI, (c - e * n)[None])
    assert abs(S0[0] - (Sa[0] + Sb[0]) / 2) < 1e-7
    assert np.abs(gS0[0] - (gSa[0] + gSb[0]) / 2).max() < 1e-6
    assert D0[0] == 0 and abs((Da[0] + Db[0]) / 2) < 1e-12
    assert abs(Da[0] - 2 * np.pi) < 1e-6 and abs(Db[0] + 2 * np.pi) < 1e-6   # the jump of the double layer
    assert np.abs(gD0[0] - gDa[0]).max() < 1e-5 * np.abs(gD0[0]).max()     # continuous across the triangle
    assert abs(np.dot(gSa[0] - gSb[0], n) + 4 * np.pi) < 1e-6                # the jump of grad S across the layer


@pytest.mark.parametrize("norder", [1, 2, 4, 6])
def test_rules_are_exact_to_the_reference_degree(norder):
    xi, eta, w = O.tri_rule(norder)
    for a in range(norder + 1):
        for b in range(norder + 1 - a):
            exact = math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2) * 2
            assert abs(np.sum(w * xi ** a * eta ** b) - exact) < 1e-14, (a, b)


def test_nbox_table():
    assert [O.tri_nbox(i, 10, 0) for i in range(-2, 6)] == [2, 5, 10, 20, 40, 80, 160, 233]


@pytest.mark.parametrize("iprec", [-1, 0, 1, 2, 3])
def test_oracle_fmm_reaches_direct_sum(iprec):
    T = icosphere(4)
    nrm, cen = normals_centroids(T)
    n = len(T)
    rng = np.random.default_rng(iprec + 10)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    trg = rng.normal(size=(300, 3))
    trg *= ((1.05 + 0.3 * rng.random(300)) / np.linalg.norm(trg, axis=1))[:, None]
    d = O.l3dtriadirect(T, cen, q, ds, trg)
    ier, *r = O.lfmm3dtriatarg(iprec, T, nrm, cen, q, ds, trg)
    assert ier == 0
    for a, b in zip(r, d):
        # above iprec 2 the degree-6 quadrature of the far field limits the accuracy
        assert rel(a, b) < (EPS[iprec] if iprec <= 2 else 1e-8)


def test_oracle_fmm_adaptive_mesh_charges_only_and_dipoles_only():
    T = two_spheres(3, 4)
    nrm, cen = normals_centroids(T)
    n = len(T)
    rng = np.random.default_rng(7)
    q = rng.uniform(-1, 1, n) + 0j
    for kw in (dict(charge=q), dict(dipstr=q)):
        d = O.l3dtriadirect(T, cen, target=None, **kw)
        ier, pot, fld, _, _ = O.lfmm3dtriatarg(1, T, nrm, cen, **kw)
        assert ier == 0
        assert rel(pot, d[0]) < EPS[1] and rel(fld, d[1]) < EPS[1]
