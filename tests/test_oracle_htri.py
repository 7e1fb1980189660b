"""The oracle's Helmholtz triangle-FMM restatement (CPU only).

Pins the near-field integrals that the reference's hfmm3dtria near field
evaluates (direct3dtritarghelms3 / helmd3 and the self terms with
triquadhelm2 / triquadselfhelm, src/triquadflatlib.f:819-2356): the Laplace
part exact, the difference kernel e^{ikr}/r - 1/r by the quadrature rule of
degree nqtri.
  - S, grad S, D, grad D against brute-force quadrature of e^{ikr}/r on 4^k
    subtriangles at points a triangle size away (the rule is accurate there);
  - at a triangle's own centroid, the difference terms against the average
    of brute-force limits from the two sides (the subtracted singular parts
    are what makes the rule usable there; the brute force limits the check
    to ~1e-3);
  - k -> 0 turns the Helmholtz integrals into the Laplace ones plus ik * area;
  - the oracle FMM (hfmm3dtriatarg) reaches its own direct sum within the
    iprec bound (iprec 2: the far field's degree-4 quadrature, norder for
    every iprec >= 0, limits it to a few 1e-6).
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402
from test_oracle_tri import _rule, _subdivide  # noqa: E402
sys.path.insert(0, os.path.join(HERE, "..", "fmmlib3d_b200"))
from meshes import icosphere, normals_centroids, two_spheres  # noqa: E402  (numpy only; no library load)

TRI = np.array([[0.1, 0.2, 0.0], [0.4, 0.15, 0.05], [0.2, 0.45, -0.02]])
ZK = 3.0 + 0.5j


def _kernels(zk, tri, x, k, n=16, diff=False, self=False):
    """Brute-force S, grad S, D, grad D of e^{ikr}/r (or of e^{ikr}/r - 1/r when diff)."""
    xi, eta, ww = _rule(n)
    nrm = np.cross(tri[1] - tri[0], tri[2] - tri[0])
    nrm /= np.linalg.norm(nrm)
    h = 0.0 if self else float(nrm @ (x - tri[0]))
    ik = 1j * zk
    S, gS, D, gD = 0j, np.zeros(3, complex), 0j, np.zeros(3, complex)
    for t in _subdivide(tri, k):
        e1, e2 = t[1] - t[0], t[2] - t[0]
        w = ww * 0.5 * np.linalg.norm(np.cross(e1, e2))
        d = x - (t[0] + xi[:, None] * e1 + eta[:, None] * e2)
        r = np.linalg.norm(d, axis=1)
        z = ik * r
        E = np.exp(z)
        F = E * (z - 1) + (1 if diff else 0)
        g = (E - (1 if diff else 0)) / r
        f2 = -F / r ** 3                           # n.grad_y of the kernel = h f2
        f2p = -(ik ** 2) * E / r ** 2 + 3 * F / r ** 4
        S += np.sum(w * g)
        gS += np.sum(w[:, None] * d * (F / r ** 3)[:, None], axis=0)
        D += np.sum(w * h * f2)
        gD += np.sum(w[:, None] * (nrm[None, :] * f2[:, None] + (h * f2p)[:, None] * d / r[:, None]), axis=0)
    return S, gS, D, gD


@pytest.mark.parametrize("x,k,tol", [((0.3, 0.3, 0.5), 2, 5e-6), ((1.5, 1.0, 0.5), 1, 1e-8),
                                     ((0.25, -0.3, -0.35), 2, 5e-6)])
def test_near_integrals_match_quadrature(x, k, tol):
    x = np.array(x)
    S, gS, D, gD = O.htri_near(ZK, TRI, x[None])
    bS, bgS, bD, bgD = _kernels(ZK, TRI, x, k)
    assert abs(S[0] - bS) <= tol * abs(bS)
    assert np.abs(gS[0] - bgS).max() <= tol * np.abs(bgS).max()
    assert abs(D[0] - bD) <= tol * abs(bD)
    assert np.abs(gD[0] - bgD).max() <= tol * np.abs(bgD).max()


def test_self_difference_terms_are_the_average_of_the_two_sides():
    c = TRI.mean(0)
    S, gS, D, gD = O.htri_near(ZK, TRI, c[None], self=True)
    lS, lgS, lD, lgD = O.tri_near(TRI, c[None], self=True)
    bS, bgS, bD, bgD = _kernels(ZK, TRI, c, 7, diff=True, self=True)
    assert D[0] == 0
    assert abs(S[0] - lS[0] - bS) <= 3e-3 * abs(bS)
    assert np.abs(gS[0] - lgS[0] - bgS).max() <= 5e-3 * np.abs(bgS).max()
    assert np.abs(gD[0] - lgD[0] - bgD).max() <= 3e-3 * np.abs(bgD).max()


@pytest.mark.parametrize("self", [False, True])
def test_small_wavenumber_reduces_to_laplace(self):
    zk = 1e-7
    x = TRI.mean(0) if self else np.array([0.3, 0.25, 0.2])
    S, gS, D, gD = O.htri_near(zk, TRI, x[None], self=self)
    lS, lgS, lD, lgD = O.tri_near(TRI, x[None], self=self)
    area = 0.5 * np.linalg.norm(np.cross(TRI[1] - TRI[0], TRI[2] - TRI[0]))
    assert abs(S[0] - (lS[0] + 1j * zk * area)) <= 1e-13 * abs(lS[0])
    assert np.abs(gS[0] - lgS[0]).max() <= 1e-12 * np.abs(lgS[0]).max()
    assert abs(D[0] - lD[0]) <= 1e-13 * max(abs(lD[0]), 1.0)
    assert np.abs(gD[0] - lgD[0]).max() <= 1e-12 * np.abs(lgD[0]).max()


def test_quadrature_degrees_follow_the_reference_table():
    assert [O.htri_nqtri(i) for i in (-3, -2, -1, 0, 1, 2, 3)] == [1, 2, 2, 4, 6, 6, 6]


EPS = {-1: .5e-1, 0: .5e-2, 1: .5e-3, 2: 5e-6}


@pytest.mark.parametrize("iprec", [-1, 0, 1, 2])
def test_oracle_fmm_reaches_direct_sum(iprec):
    T = icosphere(4)
    nrm, cen = normals_centroids(T)
    n = len(T)
    rng = np.random.default_rng(iprec + 40)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    trg = rng.normal(size=(300, 3))
    trg *= ((1.05 + 0.3 * rng.random(300)) / np.linalg.norm(trg, axis=1))[:, None]
    zk = 4.0 + 0.3j
    ier, pot, fld, pt, ft = O.hfmm3dtriatarg(iprec, zk, T, nrm, cen, q, ds, trg)
    assert ier == 0
    si = np.arange(0, n, 7)
    nq = O.htri_nqtri(iprec)
    dp, df = O.htri_direct_at(zk, T, cen[si], si, q, ds, nqtri=nq)
    tp, tf = O.htri_direct_at(zk, T, trg, None, q, ds, nqtri=nq)
    for a, b in ((pot[si], dp), (fld[si], df), (pt, tp), (ft, tf)):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < EPS[iprec]


def test_oracle_fmm_charges_only_dipoles_only_two_bodies():
    T = two_spheres(3, 4)
    nrm, cen = normals_centroids(T)
    n = len(T)
    rng = np.random.default_rng(7)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    zk = 2.0 + 0.0j
    si = np.arange(0, n, 5)
    for c, d in ((q, None), (None, ds)):
        ier, pot, fld, _, _ = O.hfmm3dtriatarg(1, zk, T, nrm, cen, c, d, None)
        assert ier == 0
        dp, df = O.htri_direct_at(zk, T, cen[si], si, c, d, nqtri=6)
        assert np.linalg.norm(pot[si] - dp) / np.linalg.norm(dp) < .5e-3
        assert np.linalg.norm(fld[si] - df) / np.linalg.norm(df) < .5e-3


def test_one_node_rule_at_own_centroid():
    """nqtri = 1 puts the rule's node on the triangle's own centroid: the bounded difference
    kernel contributes its limit there (value ik * area, no gradient)."""
    c = TRI.mean(0)
    S, gS, D, gD = O.htri_near(ZK, TRI, c[None], self=True, nqtri=1)
    lS, lgS, lD, lgD = O.tri_near(TRI, c[None], self=True)
    assert np.all(np.isfinite(S)) and np.all(np.isfinite(gS)) and np.all(np.isfinite(gD))
    area = 0.5 * np.linalg.norm(np.cross(TRI[1] - TRI[0], TRI[2] - TRI[0]))
    assert abs(S[0] - (lS[0] + 1j * ZK * area)) <= 1e-14 * abs(lS[0])
