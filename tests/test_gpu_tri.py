"""GPU parity tests of the triangle FMM (lfmm3dtriatarg_, l3dtriadirect_) through the C ABI.

The oracle restates lfmm3dtriatarg with the same tree (centroids and targets,
the triangle FMM's nbox), the same quadrature rule and the same exact
near-field integrals, so the GPU and the oracle agree to rounding: relative
L2 difference <= 1e-10 for the FMM and <= 1e-12 for the direct sums.  Against
the direct sum, the GPU FMM's error is at most 2x the oracle's (+1e-14) and
within the iprec bound.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402
from fmmlib3d_b200.meshes import icosphere, normals_centroids, two_spheres  # noqa: E402

pytestmark = pytest.mark.gpu
EPS = {-2: .5, -1: .5e-1, 0: .5e-2, 1: .5e-3, 2: .5e-6, 3: .5e-9}


@pytest.fixture(scope="module")
def F():
    import fmmlib3d_b200
    return fmmlib3d_b200


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _inputs(T, seed, m=2000):
    nrm, cen = normals_centroids(T)
    n = len(T)
    rng = np.random.default_rng(seed)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    c = cen.mean(axis=0)
    trg = rng.normal(size=(m, 3))
    trg = c + trg * ((0.5 + 1.2 * rng.random(m)) / np.linalg.norm(trg, axis=1))[:, None]
    return nrm, cen, q, ds, trg


def test_direct_sum_matches_oracle(F):
    T = icosphere(3)
    nrm, cen, q, ds, trg = _inputs(T, 1, 500)
    g = F.l3dtriadirect(T, nrm, cen, 1, q, 1, ds, 1, 1, trg, 1, 1)
    o = O.l3dtriadirect(T, cen, q, ds, trg)
    for a, b in zip(g, o):
        assert rel(a, b) < 1e-12


@pytest.mark.parametrize("mesh,iprec", [("sphere5", 1), ("sphere5", 2), ("sphere4", 0), ("sphere4", 3),
                                        ("two", 1), ("two", -1), ("ellipsoid", 2)])
def test_fmm_matches_oracle_and_direct(F, mesh, iprec):
    T = {"sphere5": lambda: icosphere(5), "sphere4": lambda: icosphere(4), "two": lambda: two_spheres(4, 5),
         "ellipsoid": lambda: icosphere(5, 1.0, (0.1, 0.0, 0.2), (1.0, 0.5, 0.25))}[mesh]()
    nrm, cen, q, ds, trg = _inputs(T, iprec + 20)
    ier, pot, fld, pt, ft = F.lfmm3dtriatarg(iprec, T, nrm, cen, 1, q, 1, ds, 1, 1, trg, 1, 1)
    assert ier == 0, F.last_error()
    oier, opot, ofld, opt, oft = O.lfmm3dtriatarg(iprec, T, nrm, cen, q, ds, trg)
    assert oier == 0
    for a, b in ((pot, opot), (fld, ofld), (pt, opt), (ft, oft)):
        assert rel(a, b) < 1e-10
    rng = np.random.default_rng(3)
    si = rng.choice(len(T), 400, replace=False)
    # direct sum at sampled centroids and targets (self by index)
    d = O.l3dtriadirect(T, cen, q, ds, trg)
    for a, o, ref in ((pot[si], opot[si], d[0][si]), (fld[si], ofld[si], d[1][si]), (pt, opt, d[2]), (ft, oft, d[3])):
        assert rel(a, ref) <= 2 * rel(o, ref) + 1e-14
        # above iprec 2 the far field's degree-6 quadrature (the reference's nqtri for every
        # iprec >= 1) limits the accuracy, not the expansion order
        assert rel(a, ref) < (EPS[iprec] if iprec <= 2 else 1e-8)


def test_flags_charges_dipoles_targets(F):
    T = two_spheres(3, 4)
    nrm, cen, q, ds, trg = _inputs(T, 5, 700)
    for kw in (dict(ifc=1, ifd=0), dict(ifc=0, ifd=1)):
        ier, pot, fld, pt, ft = F.lfmm3dtriatarg(1, T, nrm, cen, kw["ifc"], q, kw["ifd"], ds, 1, 1, trg, 1, 1)
        assert ier == 0
        o = O.lfmm3dtriatarg(1, T, nrm, cen, q if kw["ifc"] else None, ds if kw["ifd"] else None, trg)
        for a, b in zip((pot, fld, pt, ft), o[1:]):
            assert rel(a, b) < 1e-10
    # targets only (list-2 pruning), and no targets
    ier, pot, fld, pt, ft = F.lfmm3dtriatarg(1, T, nrm, cen, 1, q, 0, None, 0, 0, trg, 1, 1)
    o = O.lfmm3dtriatarg(1, T, nrm, cen, q, None, trg, ifpot=0, iffld=0)
    assert ier == 0 and not pot.any() and rel(pt, o[3]) < 1e-10 and rel(ft, o[4]) < 1e-10
    ier, pot, fld = F.lfmm3dtriaself(1, T, nrm, cen, 1, q, 1, ds, 1, 1)
    o = O.lfmm3dtriatarg(1, T, nrm, cen, q, ds, None)
    assert ier == 0 and rel(pot, o[1]) < 1e-10 and rel(fld, o[2]) < 1e-10


def test_device_entry_point_matches_host_entry_point(F):
    import torch
    T = icosphere(4)
    nrm, cen, q, ds, trg = _inputs(T, 8, 300)
    ier, pot, fld, pt, ft = F.lfmm3dtriatarg(1, T, nrm, cen, 1, q, 1, ds, 1, 1, trg, 1, 1)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64).reshape(len(a), -1)).cuda()
    n, m = len(T), len(trg)
    out = [torch.zeros(n, 2, dtype=torch.float64, device="cuda"), torch.zeros(n, 6, dtype=torch.float64, device="cuda"),
           torch.zeros(m, 2, dtype=torch.float64, device="cuda"), torch.zeros(m, 6, dtype=torch.float64, device="cuda")]
    ier2 = F.lfmm3dtriatarg_device(1, d(T.reshape(n, 9)), d(nrm), d(cen), d(q), d(ds), out[0], out[1], d(trg),
                                   out[2], out[3])
    torch.cuda.synchronize()
    assert ier == 0 and ier2 == 0
    c = lambda t, k: t.cpu().numpy().view(np.complex128).reshape(-1, k)
    for a, b, k in zip(out, (pot, fld, pt, ft), (1, 3, 1, 3)):
        assert np.array_equal(c(a, k).reshape(b.shape), b)


def test_sampled_direct_sum_matches_oracle(F):
    import torch
    T = two_spheres(3, 4)
    nrm, cen, q, ds, trg = _inputs(T, 9, 50)
    n = len(T)
    rng = np.random.default_rng(4)
    si = np.sort(rng.choice(n, 300, replace=False)).astype(np.int32)
    pts = np.concatenate([cen[si], trg])
    self_idx = np.concatenate([si, -np.ones(len(trg), np.int32)]).astype(np.int32)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64).reshape(len(a), -1)).cuda()
    pot = torch.zeros(len(pts), 2, dtype=torch.float64, device="cuda")
    fld = torch.zeros(len(pts), 6, dtype=torch.float64, device="cuda")
    ier = F.tri_direct_points_device(d(T.reshape(n, 9)), d(q), d(ds), d(pts), torch.from_numpy(self_idx).cuda(),
                                     pot, fld)
    assert ier == 0
    op, of = O.tri_direct_at(T, pts, self_idx, q, ds)
    c = lambda t, k: t.cpu().numpy().view(np.complex128).reshape(-1, k)
    assert rel(c(pot, 1)[:, 0], op) < 1e-12 and rel(c(fld, 3), of) < 1e-12
    # the full direct sum at the same centroids
    g = F.l3dtriadirect(T, nrm, cen, 1, q, 1, ds, 1, 1)
    assert rel(g[0][si], op[:300]) < 1e-12 and rel(g[1][si], of[:300]) < 1e-12


@pytest.mark.parametrize("iprec", [0, 1])
def test_mixed_form_within_twice_the_oracle_error(F, iprec):
    """set_precision(1): the triangle FMM's M2L on the tensor cores (split TF32); the exact near
    field stays FP64.  Errors against the direct sum within 2x the oracle's."""
    T = two_spheres(4, 5)
    nrm, cen, q, ds, trg = _inputs(T, 30 + iprec)
    F.set_precision(1)
    try:
        ier, pot, fld, pt, ft = F.lfmm3dtriatarg(iprec, T, nrm, cen, 1, q, 1, ds, 1, 1, trg, 1, 1)
        tuning, _ = F.last_tuning()
    finally:
        F.set_precision(0)
    assert ier == 0, F.last_error()
    assert tuning["form"] == "mixed-tc"
    oier, opot, ofld, opt, oft = O.lfmm3dtriatarg(iprec, T, nrm, cen, q, ds, trg)
    d = O.l3dtriadirect(T, cen, q, ds, trg)
    for a, o, ref in ((pot, opot, d[0]), (fld, ofld, d[1]), (pt, opt, d[2]), (ft, oft, d[3])):
        assert rel(a, ref) <= 2 * rel(o, ref)
