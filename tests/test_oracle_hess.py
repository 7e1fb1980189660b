"""The oracle's Hessian restatement (CPU only).

Pins l3dtaevalhessd_trunc / l3dmpevalhessd_trunc (src/laprouts3d.f:7682,
7194) and the pair Hessians (lpotfld3dhess, lpotfld3dhess_dp, :5442, :5619)
against one another and against the oracle's first-derivative evaluators:
  - the potential and field they return equal taeval / mpeval's (the
    reference's own l3dtaeval / l3dmpeval) to rounding, for any rscale;
  - the Hessian of an expansion formed from charges and dipoles equals the
    direct pair Hessians of those sources to rounding;
  - the pair Hessian equals a centred finite difference of the pair field;
  - the FMM with Hessians leaves potentials and fields bitwise unchanged and
    its Hessians reach the direct sum within the iprec accuracy.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle as O  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _sources(rng, n=30):
    src = rng.random((n, 3)) * 0.5 + np.array([3.0, 0.2, -0.4])
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    return src, q, ds, rng.normal(size=(n, 3))


@pytest.mark.parametrize("p,rscale", [(4, 1.0), (12, 0.37), (20, 2.5)])
def test_evaluators_agree_with_first_derivative_evaluators_and_pairs(p, rscale):
    rng = np.random.default_rng(p)
    src, q, ds, dv = _sources(rng)
    n = np.array([int(np.floor(np.sqrt(i))) for i in range((p + 1) ** 2)])
    c = np.array([0.1, 0.2, 0.3])
    pts = c + (rng.random((9, 3)) - 0.5) * 0.4
    lo = O.formta(src, c, p, charge=q, dipstr=ds, dipvec=dv)
    pot, fld = O.taeval(c, lo, p, pts)
    pot2, fld2, h2 = O.taevalhess(c, lo / rscale ** n, p, pts, rscale=rscale)
    assert rel(pot2, pot) < 1e-13 and rel(fld2, fld) < 1e-13
    H = O.direct_hess_at(src, pts, charge=q, dipstr=ds, dipvec=dv)
    assert rel(h2, H) < 10.0 ** (-min(p, 14) * 0.45)   # truncation of the local expansion
    c2 = np.array([3.2, 0.45, -0.15])
    mp = O.formmp(src, c2, p, charge=q, dipstr=ds, dipvec=dv)
    far = c2 + np.array([-3.0, 0.1, 0.2]) + (rng.random((9, 3)) - 0.5)
    pot, fld = O.mpeval(c2, mp, p, far)
    pot2, fld2, h2 = O.mpevalhess(c2, mp * rscale ** n, p, far, rscale=rscale)
    assert rel(pot2, pot) < 1e-13 and rel(fld2, fld) < 1e-13
    H = O.direct_hess_at(src, far, charge=q, dipstr=ds, dipvec=dv)
    assert rel(h2, H) < 10.0 ** (-min(p, 14) * 0.45)


def test_pair_hessian_is_the_derivative_of_the_pair_field():
    rng = np.random.default_rng(3)
    src, q, ds, dv = _sources(rng, 5)
    t = np.array([[0.3, -0.2, 0.1]])
    H = O.direct_hess_at(src, t, charge=q, dipstr=ds, dipvec=dv)[0]
    h = 1e-4
    full = np.zeros((3, 3), complex)
    for a in range(3):
        e = np.zeros(3)
        e[a] = h
        _, fp = O.direct_at(src, t + e, charge=q, dipstr=ds, dipvec=dv)
        _, fm = O.direct_at(src, t - e, charge=q, dipstr=ds, dipvec=dv)
        full[a] = -(fp[0] - fm[0]) / (2 * h)       # fld = -grad
    want = np.array([full[0, 0], full[1, 1], full[2, 2], full[0, 1], full[0, 2], full[1, 2]])
    assert np.abs(H - want).max() < 1e-6 * np.abs(want).max()
    assert abs(H[0] + H[1] + H[2]) < 1e-12 * np.abs(H).max()   # harmonic


@pytest.mark.parametrize("iprec", [0, 1, 2])
def test_oracle_fmm_hessians(iprec):
    rng = np.random.default_rng(20 + iprec)
    n, m = 12000, 6000
    src, trg = rng.random((n, 3)), rng.random((m, 3))
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    dv = rng.normal(size=(n, 3))
    ier, pot, fld, hs, pt, ft, ht = O.lfmm3dparttarg_hess(iprec, src, q, ds, dv, trg)
    ier2, pot2, fld2, pt2, ft2 = O.lfmm3dparttarg(iprec, src, q, ds, dv, trg)
    assert ier == ier2 == 0
    for a, b in ((pot, pot2), (fld, fld2), (pt, pt2), (ft, ft2)):
        assert np.array_equal(a, b)
    i = rng.choice(n, 100, replace=False)
    j = rng.choice(m, 100, replace=False)
    H = O.direct_hess_at(src, src[i], skip=i, charge=q, dipstr=ds, dipvec=dv)
    Ht = O.direct_hess_at(src, trg[j], charge=q, dipstr=ds, dipvec=dv)
    eps = {0: .5e-2, 1: .5e-3, 2: .5e-6}[iprec]
    assert rel(hs[i], H) < eps and rel(ht[j], Ht) < eps
