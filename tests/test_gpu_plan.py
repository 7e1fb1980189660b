"""Laplace plans (fixed geometry, many charge vectors; CUDA-graph replay of the passes)
and the d3tgetb / d3tgetl tree queries.

Tolerances: a plan runs the same tree, passes and kernels as a single call, so its
outputs must equal the single call's bitwise (graph replay or not); the tree queries
must reproduce the oracle's tree exactly (boxes, counts, types and lists 1-5 as sets).
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import oracle as O  # noqa: E402
from test_gpu_lap import geometry  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import fmmlib3d_b200 as F
    return F


def _inputs(n, m, seed, geom="plummer"):
    import torch
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", 0)
    src = geometry(geom, n, rng)
    trg = geometry(geom, m, rng) * 1.1
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    qs = [t(rng.uniform(-1, 1, (n, 2))) for _ in range(2)]
    ds = [t(rng.uniform(-1, 1, (n, 2))) for _ in range(2)]
    dv = rng.normal(size=(n, 3))
    dv /= np.linalg.norm(dv, axis=1)[:, None]
    return t(src), t(trg), qs, ds, t(dv)


def _outs(n, m):
    import torch
    f = lambda k, c: torch.full((k, c), np.nan, dtype=torch.float64, device="cuda")
    out = f(n, 2), f(n, 6), f(m, 2), f(m, 6)
    torch.cuda.synchronize()      # the library works on its own streams
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_plan_equals_single_calls(F, precision):
    import torch
    n, m = 30000, 12000
    src, trg, qs, ds, dv = _inputs(n, m, 5 + precision)
    F.set_precision(precision)
    try:
        plan = F.LaplacePlan(1, src, 1, 1, 1, 1, trg, 1, 1)
        for k in range(2):
            ref = _outs(n, m)
            assert F.lfmm3dparttarg_device(1, src, qs[k], ds[k], dv, ref[0], ref[1], trg, ref[2], ref[3]) == 0
            for use_graph in (True, False, True):
                out = _outs(n, m)
                assert plan.execute(qs[k], ds[k], dv, *out, use_graph=use_graph) == 0, F.last_error()
                torch.cuda.synchronize()
                for a, b in zip(out, ref):
                    assert torch.equal(a, b)
        plan.close()
    finally:
        F.set_precision(0)


def test_plan_graph_follows_new_pointers_and_charges(F):
    import torch
    n = 20000
    src, _, qs, _, _ = _inputs(n, 1, 9, "sphere")
    plan = F.LaplacePlan(1, src, 1, 0, 1, 1)
    pot_a, fld_a = torch.zeros((n, 2), dtype=torch.float64, device="cuda"), torch.zeros((n, 6), dtype=torch.float64, device="cuda")
    pot_b, fld_b = torch.zeros_like(pot_a), torch.zeros_like(fld_a)
    q = qs[0].clone()
    torch.cuda.synchronize()
    assert plan.execute(q, None, None, pot_a, fld_a) == 0
    q.copy_(qs[1])                 # same pointer, new values: the replayed graph reads them
    torch.cuda.synchronize()
    assert plan.execute(q, None, None, pot_b, fld_b) == 0
    ref = torch.zeros_like(pot_a), torch.zeros_like(fld_a)
    torch.cuda.synchronize()
    assert F.lfmm3dparttarg_device(1, src, qs[1], None, None, ref[0], ref[1]) == 0
    torch.cuda.synchronize()
    assert torch.equal(pot_b, ref[0]) and torch.equal(fld_b, ref[1])
    assert not torch.equal(pot_a, pot_b)
    launches = F.last_launches()
    assert launches > 20          # the graph holds the passes' kernels
    plan.close()


def compare_tree(plan, T):
    """The plan's tree (getb / getl) equals the oracle tree T: the same boxes by
    (level, i, j, k), counts, types, parents, children and lists 1-5 as sets."""
    info = plan.info()
    assert info["nboxes"] == T.nboxes and info["nlev"] == T.nlev
    key = lambda lev, i, j, k: (int(lev), int(i), int(j), int(k))
    okey = {key(*T.box[b, 0:4]): b for b in range(T.nboxes)}
    gkey, gbox = {}, {}
    for ib in range(1, info["nboxes"] + 1):
        ier, box, c, corners = plan.getb(ib)
        assert ier == 0
        gkey[ib] = key(*box[0:4])
        gbox[ib] = box.copy()
        side = info["size"] / 2 ** box[0]
        assert np.allclose(corners.mean(0), c) and np.isclose(corners[7, 0] - corners[0, 0], side)
    assert sorted(okey) == sorted(gkey.values())
    to_o = {ib: okey[k] for ib, k in gkey.items()}
    for ib, box in gbox.items():
        ob = T.box[to_o[ib]]
        assert box[14] == ob[14] and box[16] == ob[16]            # source and target counts
        assert box[17] == ob[17] and box[18] == ob[18]            # box types
        par = box[4]
        assert (ob[4] < 0) == (par == 0)
        if par:
            assert to_o[par] == ob[4]
        kids = {to_o[c] for c in box[5:13] if c}
        assert kids == {c for c in ob[5:13] if c >= 0}
        for ty in range(1, 6):
            ier, lst = plan.getl(ib, ty)
            assert ier == (0 if len(lst) else 4)
            assert {to_o[c] for c in lst} == set(T.list_of(ty, to_o[ib]).tolist()), (ib, ty)
    assert plan.getb(0)[0] == 2 and plan.getb(info["nboxes"] + 1)[0] == 2
    assert plan.getl(1, 6)[0] == 2


def test_plan_tree_queries_match_oracle(F):
    import torch
    n, m = 6000, 2000
    rng = np.random.default_rng(21)
    src = geometry("plummer", n, rng)
    trg = geometry("plummer", m, rng) * 0.9
    dev = torch.device("cuda", 0)
    plan = F.LaplacePlan(1, torch.from_numpy(src).to(dev), 1, 0, 1, 1, torch.from_numpy(trg).to(dev), 1, 1)
    compare_tree(plan, O.Tree(src, trg, O.lap_nbox(1, n, m)))
    plan.close()


def test_batched_plan_equals_batched_call(F):
    import torch
    rng = np.random.default_rng(31)
    srcs = [geometry(("cube", "plummer", "ellipsoid")[i % 3], int(rng.integers(500, 8000)), rng) for i in range(20)]
    off = np.concatenate([[0], np.cumsum([len(x) for x in srcs])]).astype(np.int32)
    src = torch.from_numpy(np.concatenate(srcs)).cuda()
    n = int(off[-1])
    q = torch.from_numpy(rng.uniform(-1, 1, (n, 2))).cuda()
    F.set_precision(1)
    try:
        pot, fld = torch.zeros((n, 2), dtype=torch.float64, device="cuda"), torch.zeros((n, 6), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert F.lfmm3dparttarg_batched_device(1, off, src, q, None, None, pot, fld) == 0
        plan = F.LaplacePlan(1, src, 1, 0, 1, 1, src_offsets=off)
        p2, f2 = torch.zeros_like(pot), torch.zeros_like(fld)
        torch.cuda.synchronize()
        assert plan.execute(q, None, None, p2, f2) == 0
        torch.cuda.synchronize()
        assert torch.equal(p2, pot) and torch.equal(f2, fld)
        assert plan.info()["nboxes"] >= 20
        plan.close()
    finally:
        F.set_precision(0)


@pytest.mark.parametrize("precision", [0, 1])
def test_overlapped_and_serial_passes_agree_bitwise(F, precision):
    """The near field concurrent with the far field (default) or all passes in order: same bits."""
    import torch
    n, m = 25000, 8000
    src, trg, qs, ds, dv = _inputs(n, m, 40 + precision, "cube")
    F.set_precision(precision)
    try:
        a, b = _outs(n, m), _outs(n, m)
        assert F.lfmm3dparttarg_device(1, src, qs[0], ds[0], dv, a[0], a[1], trg, a[2], a[3]) == 0
        F.set_overlap(False)
        assert F.lfmm3dparttarg_device(1, src, qs[0], ds[0], dv, b[0], b[1], trg, b[2], b[3]) == 0
        torch.cuda.synchronize()
    finally:
        F.set_overlap(True)
        F.set_precision(0)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


@pytest.mark.parametrize("ifempty,minlevel,maxlevel", [(0, 0, 100), (1, 0, 100), (0, 3, 100), (1, 2, 4),
                                                       (0, 0, 2)])
def test_d3tstrcrem_matches_oracle(F, ifempty, minlevel, maxlevel):
    """d3tstrcrem (src/d3tstrcr.f:264): empty boxes kept or dropped, a minimum
    and a maximum level, on clustered sources and targets."""
    import torch
    rng = np.random.default_rng(3)
    src = geometry("plummer", 3000, rng)
    trg = geometry("plummer", 1000, rng) * 0.9
    dev = torch.device("cuda", 0)
    tree = F.OctTree(torch.from_numpy(src).to(dev), 40, torch.from_numpy(trg).to(dev), ifempty, minlevel,
                     maxlevel)
    compare_tree(tree, O.Tree(src, trg, 40, ifempty, minlevel, maxlevel))
    assert tree.execute() == 4
    tree.close()
    with pytest.raises(RuntimeError):
        F.OctTree(torch.from_numpy(src).to(dev)[:0], 40)
