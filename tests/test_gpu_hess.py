"""GPU parity tests of the Laplace Hessians through the C ABI against the oracle.

The oracle restates the reference's Hessian evaluators (l3dtaevalhessd_trunc,
l3dmpevalhessd_trunc, lpotfld3dhess, lpotfld3dhess_dp; src/laprouts3d.f) and
adds them to its FMM.  Tolerances: the GPU and the oracle use the same tree,
lists and orders, so in the FP64 form their Hessians agree to rounding
(relative L2 difference <= 1e-10); against the FP64 direct sum, every form's
Hessian error is at most 2x the oracle's own error (+1e-13).  The potentials
and fields of a call with Hessians are bitwise those of the call without.
The single-expansion evaluators agree with the oracle's to 1e-12 (relative to
the largest value).
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import fmmlib3d_b200
    return fmmlib3d_b200


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def points(kind, n, rng):
    if kind == "cube":
        return rng.random((n, 3))
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    if kind == "sphere":
        return v
    r = 0.1 / np.sqrt(rng.random(n) ** (-2 / 3) - 1)   # plummer, clipped
    return v * np.minimum(r, 1.0)[:, None]


def inputs(kind, n, m, seed, charges=True, dipoles=True):
    rng = np.random.default_rng(seed)
    src, trg = points(kind, n, rng), points(kind, m, rng) * 0.9 + 0.05
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n) if charges else None
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n) if dipoles else None
    dv = rng.normal(size=(n, 3)) if dipoles else None
    return src, q, ds, dv, trg


@pytest.mark.parametrize("kind,iprec,charges,dipoles", [
    ("cube", 1, True, True), ("cube", 2, True, False), ("sphere", 1, False, True), ("plummer", 0, True, True)])
def test_fmm_hessians_match_oracle_fp64(F, kind, iprec, charges, dipoles):
    src, q, ds, dv, trg = inputs(kind, 40000, 25000, 11, charges, dipoles)
    ic, idp = int(charges), int(dipoles)
    ier, pot, fld, hs, pt, ft, ht = F.lfmm3dparttarghess(iprec, src, ic, q, idp, ds, dv, 1, 1, 1, trg, 1, 1, 1)
    assert ier == 0, F.last_error()
    oier, opot, ofld, ohs, opt, oft, oht = O.lfmm3dparttarg_hess(iprec, src, q, ds, dv, trg)
    assert oier == 0
    assert rel(hs, ohs) < 1e-10 and rel(ht, oht) < 1e-10, (rel(hs, ohs), rel(ht, oht))
    # the potentials and fields are those of the call without Hessians, bit for bit
    ier2, pot2, fld2, pt2, ft2 = F.lfmm3dparttarg(iprec, src, ic, q, idp, ds, dv, 1, 1, trg, 1, 1)
    assert ier2 == 0
    for a, b in ((pot, pot2), (fld, fld2), (pt, pt2), (ft, ft2)):
        assert np.array_equal(a, b)
    # against the direct sum at sampled points
    rng = np.random.default_rng(5)
    i = rng.choice(len(src), 300, replace=False)
    j = rng.choice(len(trg), 300, replace=False)
    H = O.direct_hess_at(src, src[i], skip=i, charge=q, dipstr=ds, dipvec=dv)
    Ht = O.direct_hess_at(src, trg[j], charge=q, dipstr=ds, dipvec=dv)
    assert rel(hs[i], H) <= 2 * rel(ohs[i], H) + 1e-13
    assert rel(ht[j], Ht) <= 2 * rel(oht[j], Ht) + 1e-13


@pytest.mark.parametrize("kind", ["cube", "plummer"])
def test_fmm_hessians_mixed_form_within_twice_the_oracle_error(F, kind):
    src, q, ds, dv, trg = inputs(kind, 60000, 30000, 12)
    F.set_precision(1)
    try:
        ier, pot, fld, hs, pt, ft, ht = F.lfmm3dparttarghess(1, src, 1, q, 1, ds, dv, 1, 1, 1, trg, 1, 1, 1)
        assert ier == 0, F.last_error()
        ier2, pot2, fld2, pt2, ft2 = F.lfmm3dparttarg(1, src, 1, q, 1, ds, dv, 1, 1, trg, 1, 1)
    finally:
        F.set_precision(0)
    for a, b in ((pot, pot2), (fld, fld2), (pt, pt2), (ft, ft2)):
        assert np.array_equal(a, b)
    oier, _, _, ohs, _, _, oht = O.lfmm3dparttarg_hess(1, src, q, ds, dv, trg)
    rng = np.random.default_rng(6)
    i = rng.choice(len(src), 300, replace=False)
    j = rng.choice(len(trg), 300, replace=False)
    H = O.direct_hess_at(src, src[i], skip=i, charge=q, dipstr=ds, dipvec=dv)
    Ht = O.direct_hess_at(src, trg[j], charge=q, dipstr=ds, dipvec=dv)
    assert rel(hs[i], H) <= 2 * rel(ohs[i], H) + 1e-13
    assert rel(ht[j], Ht) <= 2 * rel(oht[j], Ht) + 1e-13


def test_hessian_flags_and_small_cases(F):
    """Hessians alone (no pot / fld), targets only, and a one-box tree (near field only)."""
    src, q, ds, dv, trg = inputs("cube", 30000, 9000, 13)
    ier, pot, fld, hs, pt, ft, ht = F.lfmm3dparttarghess(1, src, 1, q, 1, ds, dv, 0, 0, 1, trg, 0, 0, 0)
    assert ier == 0
    _, _, _, ohs, _, _, _ = O.lfmm3dparttarg_hess(1, src, q, ds, dv, trg)
    assert rel(hs, ohs) < 1e-10
    assert not pot.any() and not fld.any() and not pt.any() and not ht.any()
    ier, pot, fld, hs, pt, ft, ht = F.lfmm3dparttarghess(1, src, 1, q, 1, ds, dv, 0, 0, 0, trg, 0, 0, 1)
    assert ier == 0
    _, _, _, _, _, _, oht = O.lfmm3dparttarg_hess(1, src, q, ds, dv, trg)
    assert rel(ht, oht) < 1e-10 and not hs.any()
    # 50 sources, 20 targets: one leaf, every pair direct
    s, q, ds, dv, t = inputs("cube", 50, 20, 14)
    ier, pot, fld, hs, pt, ft, ht = F.lfmm3dparttarghess(1, s, 1, q, 1, ds, dv, 1, 1, 1, t, 1, 1, 1)
    assert ier == 0
    H = O.direct_hess_at(s, s, skip=np.arange(50), charge=q, dipstr=ds, dipvec=dv)
    Ht = O.direct_hess_at(s, t, charge=q, dipstr=ds, dipvec=dv)
    assert rel(hs, H) < 1e-13 and rel(ht, Ht) < 1e-13


def _expansions(p, rng):
    src = rng.random((40, 3)) * 0.4 + np.array([2.5, 0.3, -0.2])
    q = rng.uniform(-1, 1, 40) + 1j * rng.uniform(-1, 1, 40)
    ds = rng.uniform(-1, 1, 40) + 0j
    dv = rng.normal(size=(40, 3))
    c_loc = np.array([0.1, 0.2, 0.3])
    c_mp = np.array([2.7, 0.5, 0.0])
    lo = O.formta(src, c_loc, p, charge=q, dipstr=ds, dipvec=dv)
    mp = O.formmp(src, c_mp, p, charge=q, dipstr=ds, dipvec=dv)
    return c_loc, lo, c_mp, mp


@pytest.mark.parametrize("p,rscale", [(0, 1.0), (1, 0.5), (2, 1.0), (9, 0.37), (26, 2.0), (60, 0.8), (74, 1.0)])
def test_expansion_evaluators_match_oracle(F, p, rscale):
    import torch
    rng = np.random.default_rng(p + 100)
    c_loc, lo, c_mp, mp = _expansions(p, rng)
    n = np.array([int(np.floor(np.sqrt(i))) for i in range((p + 1) ** 2)])
    # the reference's scaled coefficients: local L / rscale^n, multipole M * rscale^n
    slo, smp = lo / rscale ** n, mp * rscale ** n
    tl = c_loc + (rng.random((500, 3)) - 0.5) * 0.3
    tm = c_mp + np.array([-2.5, 0.1, 0.2]) + (rng.random((500, 3)) - 0.5) * 0.4
    for kind, coef, ctr, pts, ofn in (("local", slo, c_loc, tl, O.taevalhess), ("mpole", smp, c_mp, tm, O.mpevalhess)):
        opot, ofld, ohess = ofn(ctr, coef, p, pts, rscale=rscale)
        ref = F._expansion_layout(coef, p)
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64).reshape(-1)).cuda()
        dc, dt = d(ref), torch.from_numpy(pts.copy()).cuda()
        pot = torch.zeros(len(pts), 2, dtype=torch.float64, device="cuda")
        fld = torch.zeros(len(pts), 6, dtype=torch.float64, device="cuda")
        hess = torch.zeros(len(pts), 12, dtype=torch.float64, device="cuda")
        assert F.evalhess_device(kind, rscale, ctr, dc, p, dt, pot, fld, hess) == 0, F.last_error()
        c = lambda t, k: t.cpu().numpy().view(np.complex128).reshape(-1, k)
        gp, gf, gh = c(pot, 1)[:, 0], c(fld, 3), c(hess, 6)
        scale = lambda a: max(np.abs(a).max(), 1e-300)
        assert np.abs(gp - opot).max() <= 1e-12 * scale(opot), kind
        assert np.abs(gf - ofld).max() <= 1e-12 * scale(ofld), kind
        assert np.abs(gh - ohess).max() <= 1e-12 * scale(ohess) + 1e-300, kind
        # pot only, and pot + Hessian (other kinds of staged arrays)
        pot2 = torch.zeros_like(pot)
        hess2 = torch.zeros_like(hess)
        assert F.evalhess_device(kind, rscale, ctr, dc, p, dt, pot2, None, hess2) == 0
        assert torch.equal(pot2, pot) and torch.allclose(hess2, hess, rtol=0, atol=1e-13 * scale(ohess))
        # the reference's one-point calling sequence
        ier, p1, f1, h1 = (F.l3dtaevalhess if kind == "local" else F.l3dmpevalhess)(rscale, ctr, coef, p, pts[7])
        assert ier == 0
        assert abs(p1 - gp[7]) <= 1e-14 * scale(opot) and np.abs(h1 - gh[7]).max() <= 1e-14 * scale(ohess)


def test_expansion_evaluator_refuses_order_above_the_table(F):
    import torch
    p = 75
    coef = torch.zeros((2 * p + 1) * (p + 1) * 2, dtype=torch.float64, device="cuda")
    t = torch.zeros(4, 3, dtype=torch.float64, device="cuda")
    pot = torch.full((4, 2), 7.0, dtype=torch.float64, device="cuda")
    assert F.evalhess_device("local", 1.0, np.zeros(3), coef, p, t, pot) == 16
    assert "nterms" in F.last_error()
    assert bool((pot == 7.0).all())
