"""Batched Laplace FMM (fmm3d_lfmm3dparttarg_batched_device): many uneven
instances in one call give, instance by instance, the results of single calls.

Every instance gets its own octree inside one forest, and every pass runs
once for the whole batch, so each instance's arithmetic is that of its single
call: results must be bitwise equal, in the FP64 and the mixed form, and the
batch must take about as many kernel launches as one single call.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _instances(rng, k):
    out = []
    for i in range(k):
        n = int(10 ** rng.uniform(0, 4.3)) if i % 5 else int(rng.integers(1, 8))
        g = i % 3
        if g == 0:
            src = rng.random((n, 3)) * rng.uniform(0.1, 10) + rng.uniform(-5, 5, 3)
        elif g == 1:
            u = rng.random(n)
            r = np.minimum(0.1 / np.sqrt(np.maximum(u ** (-2 / 3) - 1, 1e-12)), 1.0)
            v = rng.normal(size=(n, 3))
            src = v / np.linalg.norm(v, axis=1)[:, None] * r[:, None]
        else:
            v = rng.normal(size=(n, 3))
            src = v / np.linalg.norm(v, axis=1)[:, None] * rng.uniform(0.2, 1, 3)
        m = 0 if i % 4 == 1 else int(rng.integers(0, max(n // 2, 2)))
        trg = src[rng.integers(0, n, m)] + rng.normal(size=(m, 3)) * 0.01 if m else np.zeros((0, 3))
        q = rng.uniform(-1, 1, (n, 2))
        dq = rng.uniform(-1, 1, (n, 2))
        dv = rng.normal(size=(n, 3))
        out.append((src, trg, q, dq, dv))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_batched_equals_single_calls(precision):
    import torch
    import fmmlib3d_b200 as F
    rng = np.random.default_rng(42 + precision)
    inst = _instances(rng, 24)
    so = np.concatenate([[0], np.cumsum([len(x[0]) for x in inst])]).astype(np.int32)
    to = np.concatenate([[0], np.cumsum([len(x[1]) for x in inst])]).astype(np.int32)
    cat = lambda j: np.ascontiguousarray(np.concatenate([x[j] for x in inst]))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    src, trg, q, dq, dv = (d(cat(j)) for j in range(5))
    n, m = int(so[-1]), int(to[-1])
    z = lambda k, w: torch.zeros((max(k, 1), w), dtype=torch.float64, device="cuda")
    pot, fld, pt, ft = z(n, 2), z(n, 6), z(m, 2), z(m, 6)
    s = torch.cuda.current_stream().cuda_stream
    F.set_precision(precision)
    try:
        ier = F.lfmm3dparttarg_batched_device(1, so, src, q, dq, dv, pot, fld, to, trg, pt, ft, stream=s)
        torch.cuda.synchronize()
        assert ier == 0, F.last_error()
        batched_launches = F.last_launches()
        single_launches = []
        for i, (a, b, c, e, f) in enumerate(inst):
            ni, mi = len(a), len(b)
            p1, f1, p2, f2 = z(ni, 2), z(ni, 6), z(mi, 2), z(mi, 6)
            ier = F.lfmm3dparttarg_device(1, d(a), d(c), d(e), d(f), p1, f1, d(b) if mi else None,
                                          p2 if mi else None, f2 if mi else None, stream=s)
            torch.cuda.synchronize()
            assert ier == 0
            single_launches.append(F.last_launches())
            assert torch.equal(pot[so[i]:so[i + 1]], p1[:ni]) and torch.equal(fld[so[i]:so[i + 1]], f1[:ni]), i
            if mi:
                assert torch.equal(pt[to[i]:to[i + 1]], p2[:mi]) and torch.equal(ft[to[i]:to[i + 1]], f2[:mi]), i
    finally:
        F.set_precision(0)
    # one launch per pass for the whole batch, not one set per instance
    assert batched_launches < 2 * max(single_launches)


def test_batched_rejects_bad_offsets():
    import torch
    import fmmlib3d_b200 as F
    src = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    q = torch.zeros((4, 2), dtype=torch.float64, device="cuda")
    pot = torch.zeros((4, 2), dtype=torch.float64, device="cuda")
    assert F.lfmm3dparttarg_batched_device(1, [0, 3, 2], src, q, None, None, pot, None) == 4
    assert F.lfmm3dparttarg_batched_device(1, [1, 4], src, q, None, None, pot, None) == 4
