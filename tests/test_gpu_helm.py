"""GPU parity tests of the Helmholtz FMM through the C ABI against the oracle.

Tolerances: the GPU and the oracle compute the same tree, lists, per-level
expansion orders, scales, truncations and quadratures; the GPU applies the
reference's sphere-projection z-shifts as precomputed linear operators (the
same sums in another order), so the two agree to rounding amplified by the
translations: relative L2 difference <= 1e-9 here.  Against the FP64 direct
sum the GPU error must be no worse than 2x the oracle's own error (+1e-14)
and within the iprec bound.
"""
import ctypes
import os
import sys
import zlib

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402
from test_gpu_lap import geometry, rel  # noqa: E402

pytestmark = pytest.mark.gpu

# Accuracy bound per iprec (src/hfmm3dpart.f:159-168).  From iprec 4 on the
# bound is 1e-12: the oracle's own field error reaches 5.96e-13 at iprec 4 on
# the clustered case below (nominal .5e-12), and 5 and 6 (direct) ask for
# more than the rounding floor of the FP64 sums compared.  The gate that
# matters, no worse than twice the oracle's error, holds at every iprec.
EPS = {-2: .5, -1: .5e-1, 0: .5e-2, 1: .5e-3, 2: .5e-6, 3: .5e-9, 4: 1e-12, 5: 1e-12, 6: 1e-12}
TOL_ORACLE = 1e-9


@pytest.fixture(scope="module")
def F():
    import fmmlib3d_b200
    return fmmlib3d_b200


def check_against_oracle(F, iprec, zk, src, trg, q, ds, dv, rng, nsamp=200):
    n = src.shape[0]
    ifc, ifd = int(q is not None), int(ds is not None)
    ier, pot, fld, pt, ft = F.hfmm3dparttarg(iprec, zk, src, ifc, q, ifd, ds, dv, 1, 1, trg, 1, 1)
    assert ier == 0, F.last_error()
    oier, opot, ofld, opt, oft = O.hfmm3dparttarg(iprec, zk, src, q, ds, dv, trg)
    assert oier == 0
    for a, b in ((pot, opot), (fld, ofld), (pt, opt), (ft, oft)):
        if b.size:
            assert rel(a, b) < TOL_ORACLE
    k = min(nsamp, n)
    si = rng.choice(n, k, replace=False)
    dp, df = O.hdirect_at(zk, src, src[si], si, q, ds, dv)
    for a, o, d in ((pot[si], opot[si], dp), (fld[si], ofld[si], df)):
        eg, eo = rel(a, d), rel(o, d)
        assert eg <= 2 * eo + 1e-14
        assert eg < EPS[iprec]
    if trg is not None and len(trg):
        ti = rng.choice(len(trg), min(nsamp, len(trg)), replace=False)
        dpt, dft = O.hdirect_at(zk, src, trg[ti], None, q, ds, dv)
        for a, o, d in ((pt[ti], opt[ti], dpt), (ft[ti], oft[ti], dft)):
            assert rel(a, d) <= 2 * rel(o, d) + 1e-14
    return pot, fld, pt, ft


def strengths(rng, n):
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    dv = rng.normal(size=(n, 3))
    dv /= np.linalg.norm(dv, axis=1)[:, None]
    return q, ds, dv


def test_helmholtz_direct_sum_matches_oracle(F):
    rng = np.random.default_rng(1)
    n, m, zk = 2500, 700, 3 + 0.25j
    src, trg = rng.random((n, 3)), rng.random((m, 3))
    q, ds, dv = strengths(rng, n)
    g = F.h3dpartdirect(zk, src, 1, q, 1, ds, dv, 1, 1, trg, 1, 1)
    o = O.h3dpartdirect(zk, src, q, ds, dv, trg)
    for a, b in zip(g, o):
        assert rel(a, b) < 1e-13


@pytest.mark.parametrize("geom,iprec,zk", [("cube", 1, 1 + 0.1j), ("cube", 2, 10.0), ("sphere", 2, 8 * np.pi),
                                           ("cube", 0, 3.0), ("plummer", 1, 5.0), ("cube", 3, 20.0),
                                           ("sphere", -1, 2.0), ("ellipsoid", 2, 4 + 0.5j), ("cube", 1, 40.0),
                                           ("cube", 2, 0.01), ("cube", 3, 60.0),
                                           # Im(zk) far above Re(zk): the per-level scales follow the
                                           # reference's Re(zk)-only rule (src/hfmm3dpart.f:337-341)
                                           ("cube", 1, 1 + 10j), ("sphere", 2, 0.5 + 6j)])
def test_hfmm_parity_charges_dipoles_targets(F, geom, iprec, zk):
    rng = np.random.default_rng(zlib.crc32(('%s%d%s' % (geom, iprec, zk)).encode()))
    n, m = 12000, 4000
    src = geometry(geom, n, rng)
    trg = geometry(geom, m, rng) * 1.1
    q, ds, dv = strengths(rng, n)
    check_against_oracle(F, iprec, zk, src, trg, q, ds, dv, rng)


@pytest.mark.parametrize("geom,iprec,zk,n,m", [("plummer", 4, 1 + 0.1j, 15000, 3000),
                                               ("plummer", 5, 2.0, 15000, 3000),
                                               ("cube", 6, 3.0, 3000, 1000), ("cube", -2, 1.0, 15000, 5000)])
def test_hfmm_parity_remaining_iprec(F, geom, iprec, zk, n, m):
    """iprec 4 / 5: expansion orders 46 / 59 on a five-level clustered tree;
    6: every point in the root box; -2: the coarsest tables."""
    rng = np.random.default_rng(zlib.crc32(('hi%s%d' % (geom, iprec)).encode()))
    src = geometry(geom, n, rng)
    trg = geometry(geom, m, rng) * 1.1
    q, ds, dv = strengths(rng, n)
    check_against_oracle(F, iprec, zk, src, trg, q, ds, dv, rng)


@pytest.mark.parametrize("zk,iprec,order", [(40 * np.pi, 2, 80), (48 * np.pi, 2, 92), (55 * np.pi, 1, 93)])
def test_hfmm_high_orders(F, zk, iprec, order):
    """Expansion orders above 60 (20 to 27 wavelengths across the sphere): the translation
    buffers move to global scratch, the evaluation kernel runs 32 points per CTA and the
    P2M/P2L staging takes smaller chunks; results still match the oracle and the direct sum."""
    rng = np.random.default_rng(zlib.crc32(('high%d%d' % (iprec, order)).encode()))
    n = 8000
    src = geometry("sphere", n, rng)
    q, ds, dv = strengths(rng, n)
    oier, _, _, _, _, nts = O.hfmm3dparttarg(iprec, zk, src, q, nterms=True)
    assert max(nts[2:]) == order
    check_against_oracle(F, iprec, zk, src, None, q, None, None, rng)


def test_hfmm_order_above_the_limit_is_refused(F):
    """Orders above 104 return ier 16 with a message, outputs untouched (the reference runs to 1000)."""
    rng = np.random.default_rng(77)
    n = 6000
    src = geometry("sphere", n, rng)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ier, pot, fld, _, _ = F.hfmm3dparttarg(1, 70 * np.pi, src, 1, q, 0, None, None, 1, 1)
    assert ier == 16
    assert "expansion order" in F.last_error()


def test_hfmm_flags_and_coincident_points(F):
    """As for Laplace: flags other than 1 are off (src/hfmm3dpart.f:601-617), and a
    target on top of a source gets a non-finite value (no guard), nothing else."""
    rng = np.random.default_rng(18)
    n, m, zk = 3000, 800, 2.0 + 0.1j
    src, trg = rng.random((n, 3)), rng.random((m, 3))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    sentinel = 7.25 + 3.5j
    pot, pt = np.full(n, sentinel), np.full(m, sentinel)
    fld, ft = np.zeros((n, 3), complex), np.zeros((m, 3), complex)
    lib = F.lib()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    I = lambda v: ctypes.byref(ctypes.c_int(v))
    ier = ctypes.c_int(-1)
    zkc = np.array([zk], complex)
    dummy = np.zeros(2, complex)
    lib.hfmm3dparttarg_(ctypes.byref(ier), I(1), P(zkc), I(n), P(src), I(1), P(q), I(3), P(dummy), P(src), I(0),
                        P(pot), I(1), P(fld), I(m), P(trg), I(-4), P(pt), I(1), P(ft))
    assert ier.value == 0
    assert np.all(pot == sentinel) and np.all(pt == sentinel)
    _, _, ofld, _, oft = O.hfmm3dparttarg(1, zk, src, q, None, None, trg)
    assert rel(fld, ofld) < TOL_ORACLE and rel(ft, oft) < TOL_ORACLE
    trg[5] = src[123]
    ier, pot, fld, pt, ft = F.hfmm3dparttarg(1, zk, src, 1, q, 0, None, None, 1, 1, trg, 1, 1)
    _, opot, ofld, opt, oft = O.hfmm3dparttarg(1, zk, src, q, None, None, trg)
    assert ier == 0 and not np.isfinite(opt[5]) and not np.isfinite(pt[5]) and not np.all(np.isfinite(ft[5]))
    keep = np.arange(m) != 5
    assert np.all(np.isfinite(pot)) and np.all(np.isfinite(pt[keep])) and np.all(np.isfinite(ft[keep]))
    assert rel(pot, opot) < TOL_ORACLE and rel(fld, ofld) < TOL_ORACLE
    assert rel(pt[keep], opt[keep]) < TOL_ORACLE and rel(ft[keep], oft[keep]) < TOL_ORACLE


@pytest.mark.parametrize("mode", ["charge", "dipole"])
def test_hfmm_parity_source_kinds(F, mode):
    rng = np.random.default_rng(7)
    n = 20000
    src = geometry("sphere", n, rng)
    q, ds, dv = strengths(rng, n)
    if mode == "charge":
        ds = dv = None
    else:
        q = None
    check_against_oracle(F, 2, 6.0, src, None, q, ds, dv, rng)


def test_hfmm_reference_driver_inputs(F):
    # examples/hfmm3dpart_driver.f: 10,000 sources on a sphere of radius 0.5,
    # targets shifted by +1, zk = 1 + 0.1i, iprec = 1
    from driver_inputs import driver_inputs
    src, trg, q, ds, dv = driver_inputs(10000, shift=1.0)
    check_against_oracle(F, 1, 1 + 0.1j, src, trg, q, ds, dv, np.random.default_rng(0))


def test_hfmm_golden_fixture(F):
    from driver_inputs import driver_inputs
    d = np.load(os.path.join(HERE, "golden", "driver_helm_n2000.npz"))
    src, trg, q, ds, dv = driver_inputs(2000, shift=1.0)
    zk = complex(d["zk"])
    ier, pot, fld, pt, ft = F.hfmm3dparttarg(1, zk, src, 1, q, 1, ds, dv, 1, 1, trg, 1, 1)
    assert ier == 0
    for a, b in ((pot, "pot"), (fld, "fld"), (pt, "pottarg"), (ft, "fldtarg")):
        assert rel(a[:100], d[b]) < TOL_ORACLE
        assert rel(a[:100], d["d" + b]) <= 2 * rel(d[b], d["d" + b]) + 1e-14


@pytest.mark.parametrize("geom", ["plane", "two_clusters"])
def test_hfmm_degenerate_geometries(F, geom):
    rng = np.random.default_rng(11)
    n = 8000
    src = geometry(geom, n, rng)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    zk = 2.0 if geom == "plane" else 0.5
    check_against_oracle(F, 1, zk, src, None, q, None, None, rng)


def test_hfmm_expansion_orders_match_oracle(F):
    rng = np.random.default_rng(3)
    n = 60000
    src = geometry("sphere", n, rng)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    F.set_stats(True)
    try:
        ier, pot, fld = F.hfmm3dpartself(2, 8 * np.pi, src, 1, q, 0, None, None, 1, 1)
        st = F.last_stats()
    finally:
        F.set_stats(False)
    assert ier == 0
    oier, opot, ofld, _, _, nt = O.hfmm3dparttarg(2, 8 * np.pi, src, q, nterms=True)
    nlev = st["nlev"]
    # the GPU records the orders of the levels that carry expansions (>= 2)
    assert st["nterms_level"][2:nlev + 1] == [int(v) for v in nt[2:nlev + 1]]
    assert st["nterms"] == max(int(v) for v in nt[2:nlev + 1])
    assert rel(pot, opot) < TOL_ORACLE and rel(fld, ofld) < TOL_ORACLE


def test_hfmm_small_and_empty_cases(F):
    rng = np.random.default_rng(5)
    for n in (1, 2, 7, 500):
        src = rng.random((n, 3))
        q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        ier, pot, fld, pt, ft = F.hfmm3dparttarg(1, 2.0, src, 1, q, 0, None, None, 1, 1, rng.random((3, 3)), 1, 1)
        assert ier == 0
        dp, df, _, _ = O.h3dpartdirect(2.0, src, q, None, None, None)
        if n > 1:
            assert rel(pot, dp) < 1e-12 and rel(fld, df) < 1e-12
        else:
            assert np.all(pot == 0) and np.all(fld == 0)
    # iprec outside -2..6 is rejected
    assert F.hfmm3dpartself(9, 1.0, rng.random((10, 3)), 1, np.ones(10, complex), 0, None, None, 1, 1)[0] != 0


def test_hfmm_unrequested_outputs_untouched(F):
    rng = np.random.default_rng(9)
    n, m = 3000, 800
    src, trg = rng.random((n, 3)), rng.random((m, 3))
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    lib = F.lib()
    sentinel = 12345.0 + 6789.0j
    pot = np.full(n, sentinel)
    fld = np.full((n, 3), sentinel)
    pt = np.zeros(m, complex)
    ft = np.full((m, 3), sentinel)
    ier = ctypes.c_int(-1)
    zk = np.array([3.0, 0.0])
    I = lambda v: ctypes.byref(ctypes.c_int(v))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lib.hfmm3dparttarg_(ctypes.byref(ier), I(1), P(zk), I(n), P(src), I(1), P(q), I(0), P(q), P(src), I(0), P(pot),
                        I(0), P(fld), I(m), P(trg), I(1), P(pt), I(0), P(ft))
    assert ier.value == 0
    assert np.all(pot == sentinel) and np.all(fld == sentinel) and np.all(ft == sentinel)
    _, _, opt, _ = O.h3dpartdirect(3.0, src, q, None, None, trg, ifpot=0, iffld=0)
    assert rel(pt, opt) < EPS[1]


def test_hfmm_device_entry_point_matches_host_entry_point(F):
    import torch
    rng = np.random.default_rng(13)
    n, m, zk = 20000, 5000, 7 + 0.2j
    src, trg = geometry("cube", n, rng), geometry("cube", m, rng)
    q, ds, dv = strengths(rng, n)
    ier, pot, fld, pt, ft = F.hfmm3dparttarg(2, zk, src, 1, q, 1, ds, dv, 1, 1, trg, 1, 1)
    assert ier == 0
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    c2 = lambda a: d(np.stack([a.real, a.imag], -1))
    z = lambda k: torch.zeros((k, 2), dtype=torch.float64, device="cuda")
    out = [z(n), torch.zeros((n, 6), dtype=torch.float64, device="cuda"), z(m),
           torch.zeros((m, 6), dtype=torch.float64, device="cuda")]
    ier2 = F.hfmm3dparttarg_device(2, zk, d(src), c2(q), c2(ds), d(dv), out[0], out[1], d(trg), out[2], out[3],
                                   stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert ier2 == 0
    cv = lambda t: t.cpu().numpy().view(np.complex128)
    assert np.array_equal(cv(out[0]).reshape(-1), pot)
    assert np.array_equal(cv(out[1]).reshape(n, 3), fld)
    assert np.array_equal(cv(out[2]).reshape(-1), pt)
    assert np.array_equal(cv(out[3]).reshape(m, 3), ft)


def test_hfmm_repeat_calls_bitwise_identical(F):
    rng = np.random.default_rng(17)
    n = 30000
    src = geometry("sphere", n, rng)
    q, ds, dv = strengths(rng, n)
    a = F.hfmm3dpartself(2, 8 * np.pi, src, 1, q, 1, ds, dv, 1, 1)
    b = F.hfmm3dpartself(2, 8 * np.pi, src, 1, q, 1, ds, dv, 1, 1)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


def test_hfmm_direct_points_entry(F):
    import torch
    rng = np.random.default_rng(19)
    n, k, zk = 5000, 300, 4.0 + 0.1j
    src = rng.random((n, 3))
    q, ds, dv = strengths(rng, n)
    idx = rng.choice(n, k, replace=False).astype(np.int32)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    c2 = lambda a: d(np.stack([a.real, a.imag], -1))
    pot = torch.zeros((k, 2), dtype=torch.float64, device="cuda")
    fld = torch.zeros((k, 6), dtype=torch.float64, device="cuda")
    ier = F.hdirect_points_device(zk, d(src), c2(q), c2(ds), d(dv), d(src[idx]), d(idx), pot, fld,
                                  stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert ier == 0
    op, of = O.hdirect_at(zk, src, src[idx], idx, q, ds, dv)
    assert rel(pot.cpu().numpy().view(np.complex128).reshape(-1), op) < 1e-13
    assert rel(fld.cpu().numpy().view(np.complex128).reshape(k, 3), of) < 1e-13
