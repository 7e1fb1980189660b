"""GPU parity tests of the Helmholtz triangle FMM (hfmm3dtriatarg_, h3dtriadirect_) through the C ABI.

The oracle restates hfmm3dtriatarg with the same tree (centroids and targets,
the triangle FMM's nbox, the box scale from |zk|), the same far-field
quadrature nodes, the same near-field rule (nqtri) and the same exact Laplace
part, so the GPU and the oracle agree to rounding: relative L2 difference
<= 1e-10 for the FMM and <= 1e-12 for the direct sums.  Against the direct
sum of the same near-field rule, the GPU FMM's error is at most 2x the
oracle's (+1e-14).
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


@pytest.fixture(scope="module")
def F():
    import fmmlib3d_b200
    return fmmlib3d_b200


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _inputs(T, seed, m=1500):
    nrm, cen = normals_centroids(T)
    n = len(T)
    rng = np.random.default_rng(seed)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    c = cen.mean(axis=0)
    trg = rng.normal(size=(m, 3))
    trg = c + trg * ((0.5 + 1.2 * rng.random(m)) / np.linalg.norm(trg, axis=1))[:, None]
    return nrm, cen, q, ds, trg


@pytest.mark.parametrize("nqtri", [1, 2, 4, 6])
def test_direct_sum_matches_oracle(F, nqtri):
    T = icosphere(3)
    nrm, cen, q, ds, trg = _inputs(T, 1, 400)
    zk = 4.0 + 0.3j
    pot, fld, pt, ft = F.h3dtriadirect(nqtri, zk, T, nrm, cen, 1, q, 1, ds, 1, 1, trg, 1, 1)
    n = len(T)
    op, of = O.htri_direct_at(zk, T, cen, np.arange(n), q, ds, nqtri=nqtri)
    tp, tf = O.htri_direct_at(zk, T, trg, None, q, ds, nqtri=nqtri)
    for a, b in ((pot, op), (fld, of), (pt, tp), (ft, tf)):
        assert rel(a, b) < 1e-12


@pytest.mark.parametrize("mesh,iprec,zk", [("sphere5", 1, 4.0 + 0.3j), ("sphere4", 2, 4.0 + 0.3j),
                                           ("sphere4", 0, 10.0 + 0.0j), ("two", 1, 2.0 + 0.5j),
                                           ("two", -1, 6.0 + 0.0j),
                                           ("ellipsoid", 1, 8.0 + 1.0j)])
def test_fmm_matches_oracle_and_direct(F, mesh, iprec, zk):
    T = {"sphere5": lambda: icosphere(5), "sphere4": lambda: icosphere(4), "two": lambda: two_spheres(4, 5),
         "ellipsoid": lambda: icosphere(5, 1.0, (0.1, 0.0, 0.2), (1.0, 0.5, 0.25))}[mesh]()
    nrm, cen, q, ds, trg = _inputs(T, iprec + 50)
    ier, pot, fld, pt, ft = F.hfmm3dtriatarg(iprec, zk, T, nrm, cen, 1, q, 1, ds, 1, 1, trg, 1, 1)
    assert ier == 0, F.last_error()
    oier, opot, ofld, opt, oft = O.hfmm3dtriatarg(iprec, zk, T, nrm, cen, q, ds, trg)
    assert oier == 0
    for a, b in ((pot, opot), (fld, ofld), (pt, opt), (ft, oft)):
        assert rel(a, b) < 1e-10
    rng = np.random.default_rng(3)
    si = np.sort(rng.choice(len(T), 300, replace=False))
    nq = O.htri_nqtri(iprec)
    dp, df = O.htri_direct_at(zk, T, cen[si], si, q, ds, nqtri=nq)
    tp, tf = O.htri_direct_at(zk, T, trg, None, q, ds, nqtri=nq)
    for a, o, ref in ((pot[si], opot[si], dp), (fld[si], ofld[si], df), (pt, opt, tp), (ft, oft, tf)):
        assert rel(a, ref) <= 2 * rel(o, ref) + 1e-14


def test_flags_charges_dipoles_targets(F):
    T = two_spheres(3, 4)
    nrm, cen, q, ds, trg = _inputs(T, 5, 700)
    zk = 3.0 + 0.2j
    for ifc, ifd in ((1, 0), (0, 1)):
        ier, pot, fld, pt, ft = F.hfmm3dtriatarg(1, zk, T, nrm, cen, ifc, q, ifd, ds, 1, 1, trg, 1, 1)
        assert ier == 0
        o = O.hfmm3dtriatarg(1, zk, T, nrm, cen, q if ifc else None, ds if ifd else None, trg)
        for a, b in zip((pot, fld, pt, ft), o[1:]):
            assert rel(a, b) < 1e-10
    # targets only (list-2 pruning), and no targets
    ier, pot, fld, pt, ft = F.hfmm3dtriatarg(1, zk, T, nrm, cen, 1, q, 0, None, 0, 0, trg, 1, 1)
    o = O.hfmm3dtriatarg(1, zk, T, nrm, cen, q, None, trg, ifpot=0, iffld=0)
    assert ier == 0 and not pot.any() and rel(pt, o[3]) < 1e-10 and rel(ft, o[4]) < 1e-10
    ier, pot, fld = F.hfmm3dtriaself(1, zk, T, nrm, cen, 1, q, 1, ds, 1, 1)
    o = O.hfmm3dtriatarg(1, zk, T, nrm, cen, q, ds, None)
    assert ier == 0 and rel(pot, o[1]) < 1e-10 and rel(fld, o[2]) < 1e-10


def test_device_entry_point_matches_host_entry_point(F):
    import torch
    T = icosphere(4)
    nrm, cen, q, ds, trg = _inputs(T, 8, 300)
    zk = 5.0 + 0.1j
    ier, pot, fld, pt, ft = F.hfmm3dtriatarg(1, zk, T, nrm, cen, 1, q, 1, ds, 1, 1, trg, 1, 1)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64).reshape(len(a), -1)).cuda()
    n, m = len(T), len(trg)
    out = [torch.zeros(n, 2, dtype=torch.float64, device="cuda"), torch.zeros(n, 6, dtype=torch.float64, device="cuda"),
           torch.zeros(m, 2, dtype=torch.float64, device="cuda"), torch.zeros(m, 6, dtype=torch.float64, device="cuda")]
    ier2 = F.hfmm3dtriatarg_device(1, zk, d(T.reshape(n, 9)), d(nrm), d(cen), d(q), d(ds), out[0], out[1], d(trg),
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
    zk = 4.0 + 0.3j
    rng = np.random.default_rng(4)
    si = np.sort(rng.choice(n, 300, replace=False)).astype(np.int32)
    pts = np.concatenate([cen[si], trg])
    self_idx = np.concatenate([si, -np.ones(len(trg), np.int32)]).astype(np.int32)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64).reshape(len(a), -1)).cuda()
    pot = torch.zeros(len(pts), 2, dtype=torch.float64, device="cuda")
    fld = torch.zeros(len(pts), 6, dtype=torch.float64, device="cuda")
    ier = F.htri_direct_points_device(6, zk, d(T.reshape(n, 9)), d(q), d(ds), d(pts),
                                      torch.from_numpy(self_idx).cuda(), pot, fld)
    assert ier == 0, F.last_error()
    op, of = O.htri_direct_at(zk, T, pts, self_idx, q, ds, nqtri=6)
    c = lambda t, k: t.cpu().numpy().view(np.complex128).reshape(-1, k)
    assert rel(c(pot, 1)[:, 0], op) < 1e-12 and rel(c(fld, 3), of) < 1e-12
    # the full direct sum at the same centroids
    g = F.h3dtriadirect(6, zk, T, nrm, cen, 1, q, 1, ds, 1, 1)
    assert rel(g[0][si], op[:300]) < 1e-12 and rel(g[1][si], of[:300]) < 1e-12
