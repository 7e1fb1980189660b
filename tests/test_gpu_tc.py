"""Tensor-core (tcgen05, split TF32) path: the GEMM self-test against numpy, and the
mixed form's M2L on the tensor cores against the FP64 direct sum and the oracle.

Tolerances: split TF32 products (hi*hi + hi*lo + lo*hi [+ lo*lo], FP32 accumulation)
carry a relative error of a few 2^-24 per product, so the self-test bound is 5e-6 of the sum
of |a||b| per entry (TF32 high parts alone: about 2^-11); the FMM with tensor-core
M2L must meet the mixed form's gate: error vs the FP64 direct sum within the iprec
bound and at most 2x the oracle's, or, where the oracle's own error is below the
mixed form's FP32 arithmetic floor (errors under 1e-8), no worse than the mixed form
with its M2L on the CUDA cores.
"""
import os
import sys
import zlib

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle as O  # noqa: E402
from test_gpu_lap import EPS, geometry, rel  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import fmmlib3d_b200 as F
    return F


@pytest.mark.parametrize("n,k", [(16, 32), (64, 96), (128, 256), (112, 64)])
def test_selftest_matches_numpy(F, n, k):
    rng = np.random.default_rng(1000 * n + k)
    A = rng.uniform(-1, 1, (128, k)).astype(np.float32)
    B = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64).T
    st, D = F.tc_selftest(A, B, 3)
    assert st == 0
    err3 = np.max(np.abs(D - ref) / scale)
    assert err3 < 5e-6, err3
    st, D4 = F.tc_selftest(A, B, 4)
    assert st == 0
    err4 = np.max(np.abs(D4 - ref) / scale)
    assert err4 < 5e-6 and err4 <= err3 * 1.01, (err4, err3)
    st, D1 = F.tc_selftest(A, B, 1)
    assert st == 0
    err1 = np.max(np.abs(D1 - ref) / scale)
    assert 1e-5 < err1 < 4e-3, err1     # the high parts alone: TF32 accuracy
    assert err3 < err1 / 50


def test_selftest_rejects_bad_shapes(F):
    A = np.zeros((128, 40), np.float32)
    B = np.zeros((16, 40), np.float32)
    assert F.tc_selftest(A, B)[0] == 1
    assert F.tc_selftest(np.zeros((128, 32), np.float32), np.zeros((20, 32), np.float32))[0] == 1


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("geom,iprec", [("cube", 1), ("cube", 0), ("sphere", 1), ("plummer", 1), ("cube", -1)])
def test_tensor_m2l_within_twice_reference_error(F, mode, geom, iprec):
    rng = np.random.default_rng(zlib.crc32(('tc%s%d' % (geom, iprec)).encode()))
    n, m = 40000, 20000
    src = geometry(geom, n, rng)
    trg = geometry(geom, m, rng) * 1.05
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    ds = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    dv = rng.normal(size=(n, 3))
    dv /= np.linalg.norm(dv, axis=1)[:, None]
    F.set_precision(1)
    try:
        F.set_tensor_m2l(0)
        ref = F.lfmm3dparttarg(iprec, src, 1, q, 1, ds, dv, 1, 1, trg, 1, 1)
        F.set_tensor_m2l(mode)
        ier, pot, fld, pt, ft = F.lfmm3dparttarg(iprec, src, 1, q, 1, ds, dv, 1, 1, trg, 1, 1)
    finally:
        F.set_tensor_m2l(1)
        F.set_precision(0)
    assert ier == 0 and ref[0] == 0
    # same far field as the FP32 CUDA-core M2L up to FP32-level differences
    for a, b in zip((pot, fld, pt, ft), ref[1:]):
        assert rel(a, b) < 1e-5
    oier, opot, ofld, opt, oft = O.lfmm3dparttarg(iprec, src, q, ds, dv, trg)
    k = 400
    si = rng.choice(n, k, replace=False)
    ti = rng.choice(m, k, replace=False)
    dp, df = O.direct_at(src, src[si], si, q, ds, dv)
    dpt, dft = O.direct_at(src, trg[ti], None, q, ds, dv)
    cases = ((pot, opot, ref[1], si, dp), (fld, ofld, ref[2], si, df), (pt, opt, ref[3], ti, dpt),
             (ft, oft, ref[4], ti, dft))
    for a, o, c, ix, d in cases:
        eg, eo, ec = rel(a[ix], d), rel(o[ix], d), rel(c[ix], d)
        assert eg < EPS[iprec]
        # the 2x gate; where the oracle's error is near the FP32 arithmetic floor
        # of the mixed form (~1e-9), no worse than the CUDA-core mixed form
        assert eg <= 2 * eo or (eg < 1e-8 and eg <= 1.02 * ec), (eg, eo, ec)


def test_tensor_m2l_repeatable_and_fp64_path_untouched(F):
    rng = np.random.default_rng(7)
    n = 30000
    src = geometry("sphere", n, rng)
    q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    F.set_tensor_m2l(1)
    try:
        a = F.lfmm3dpartself(1, src, 1, q, 0, None, None, 1, 1)
        F.set_precision(1)
        b = F.lfmm3dpartself(1, src, 1, q, 0, None, None, 1, 1)
        c = F.lfmm3dpartself(1, src, 1, q, 0, None, None, 1, 1)
    finally:
        F.set_precision(0)
    d = F.lfmm3dpartself(1, src, 1, q, 0, None, None, 1, 1)
    assert np.array_equal(b[1], c[1]) and np.array_equal(b[2], c[2])    # deterministic
    assert np.array_equal(a[1], d[1]) and np.array_equal(a[2], d[2])    # FP64 form ignores the switch
    with pytest.raises(ValueError):
        F.set_tensor_m2l(5)


def test_tensor_m2l_gate_on_adaptive_batch(F):
    """Mixed form with tensor-core M2L on a batch of adaptive instances (Plummer
    spheres and ellipsoid surfaces): error vs the FP64 direct sum at most 2x the FP64
    form's error on the same points (the FP64 form equals the oracle to rounding)."""
    import torch
    rng = np.random.default_rng(44)
    srcs = []
    for i in range(48):
        n = int(rng.integers(2000, 12000))
        srcs.append(geometry("plummer" if i % 2 else "ellipsoid", n, rng))
    off = np.concatenate([[0], np.cumsum([len(s) for s in srcs])]).astype(np.int32)
    src = np.concatenate(srcs)
    q = rng.uniform(-1, 1, (len(src), 2))
    dev = torch.device("cuda", 0)
    d_src, d_q = torch.from_numpy(src).to(dev), torch.from_numpy(q).to(dev)
    out = {}
    for form in (0, 1):
        pot = torch.empty((len(src), 2), dtype=torch.float64, device=dev)
        fld = torch.empty((len(src), 6), dtype=torch.float64, device=dev)
        F.set_precision(form)
        try:
            assert F.lfmm3dparttarg_batched_device(1, off, d_src, d_q, None, None, pot, fld) == 0
        finally:
            F.set_precision(0)
        torch.cuda.synchronize()
        out[form] = (pot.cpu().numpy(), fld.cpu().numpy())
    num = {0: [0.0, 0.0], 1: [0.0, 0.0]}
    den = [0.0, 0.0]
    for i in range(0, 48, 3):
        a, b = int(off[i]), int(off[i + 1])
        idx = rng.choice(b - a, 40, replace=False)
        qc = q[a:b, 0] + 1j * q[a:b, 1]
        dp, df = O.direct_at(src[a:b], src[a:b][idx], idx, qc)
        dp = np.stack([dp.real, dp.imag], -1)
        df = np.stack([df.real, df.imag], -1).reshape(len(idx), 6)
        den[0] += np.sum(dp ** 2)
        den[1] += np.sum(df ** 2)
        for form in (0, 1):
            num[form][0] += np.sum((out[form][0][a:b][idx] - dp) ** 2)
            num[form][1] += np.sum((out[form][1][a:b][idx] - df) ** 2)
    for c in range(2):
        e64, emx = (num[0][c] / den[c]) ** .5, (num[1][c] / den[c]) ** .5
        assert e64 < EPS[1] and emx <= 2 * e64, (c, emx, e64)
