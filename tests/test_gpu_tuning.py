"""Launch-shape knobs and the autotuner on the GPU.

Tolerances: none — the knobs change tile sizes, staging, stream overlap and points per
lane, never the order of any sum, so every setting must reproduce the automatic
setting's outputs bitwise (plans with and without graph replay, and single calls that
take their knobs from the tuning cache).
"""
import numpy as np
import pytest

from test_gpu_lap import geometry

pytestmark = pytest.mark.gpu


@pytest.fixture()
def F():
    import fmmlib3d_b200 as F
    yield F
    F.set_precision(0)
    F.set_m2l_mode(0)
    F.set_tuning_cache(None)


def _problem(n, m, seed, geom="plummer"):
    import torch
    rng = np.random.default_rng(seed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    src = t(geometry(geom, n, rng))
    trg = t(geometry(geom, m, rng) * 1.1)
    q = t(rng.uniform(-1, 1, (n, 2)))
    d = t(rng.uniform(-1, 1, (n, 2)))
    v = rng.normal(size=(n, 3))
    v = t(v / np.linalg.norm(v, axis=1)[:, None])
    return src, trg, q, d, v


def _outs(n, m):
    import torch
    f = lambda k, c: torch.full((k, c), np.nan, dtype=torch.float64, device="cuda")
    out = f(n, 2), f(n, 6), f(m, 2), f(m, 6)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("precision,iprec,m2l_mode,form", [(1, 1, 0, "mixed-tc"), (0, 1, 0, "fp64-dense"),
                                                           (0, 1, 1, "fp64-rotation"), (0, 2, 0, "fp64-rotation")])
def test_every_setting_gives_the_same_bits(F, precision, iprec, m2l_mode, form):
    import torch
    from fmmlib3d_b200 import autotune as A
    n, m = 24000, 9000
    src, trg, q, d, v = _problem(n, m, 100 + 10 * precision + iprec + 3 * m2l_mode)
    F.set_precision(precision)
    F.set_m2l_mode(m2l_mode)
    F.set_tuning_cache("")
    plan = F.LaplacePlan(iprec, src, 1, 1, 1, 1, trg, 1, 1)
    t = plan.get_tuning()
    assert t["form"] == form and not t["from_cache"]
    ref = _outs(n, m)
    assert plan.execute(q, d, v, *ref, use_graph=False) == 0
    torch.cuda.synchronize()
    tried = 0
    for knob, values in A.candidates(form):
        for val in values:
            if plan.set_tuning({knob: val}) != 0:
                continue
            assert plan.get_tuning()[knob] == val
            for g in (False, True):
                out = _outs(n, m)
                assert plan.execute(q, d, v, *out, use_graph=g) == 0, F.last_error()
                torch.cuda.synchronize()
                for a, b in zip(out, ref):
                    assert torch.equal(a, b), (knob, val, g)
            tried += 1
    assert tried >= 6
    plan.close()


def test_bad_values_are_refused_and_the_plan_keeps_its_knobs(F):
    import torch
    n = 8000
    src, _, q, _, _ = _problem(n, 1, 7, "cube")
    F.set_precision(1)
    F.set_tuning_cache("")
    plan = F.LaplacePlan(1, src, 1, 0, 1, 1)
    assert plan.set_tuning({"m2l_kt": 32, "trans_kt": 4}) == 0
    before = plan.get_tuning()
    for bad in ({"m2l_kt": 24}, {"m2l_kt": 272}, {"trans_kt": 3}, {"trans_kt": 16}, {"overlap": 3},
                {"tc_variant": 5}, {"p2p_ept": 3}):
        assert plan.set_tuning(bad) == 2, bad
        assert plan.get_tuning() == before
    with pytest.raises(ValueError):
        plan.set_tuning({"tile": 4})
    pot, fld = torch.zeros((n, 2), dtype=torch.float64, device="cuda"), torch.zeros((n, 6), dtype=torch.float64,
                                                                                    device="cuda")
    torch.cuda.synchronize()
    assert plan.execute(q, None, None, pot, fld) == 0
    plan.close()


def test_tune_writes_the_cache_and_single_calls_use_it(F, tmp_path):
    import json
    import torch
    from fmmlib3d_b200 import autotune as A
    n, m = 30000, 12000
    src, trg, q, d, v = _problem(n, m, 55, "cube")
    F.set_precision(1)
    path = str(tmp_path / "tune.json")
    F.set_tuning_cache(path)
    ref = _outs(n, m)
    assert F.lfmm3dparttarg_device(1, src, q, d, v, ref[0], ref[1], trg, ref[2], ref[3]) == 0
    knobs0, sig0 = F.last_tuning()
    assert not knobs0["from_cache"] and sig0.startswith("laplace iprec=1 form=mixed-tc")
    plan = F.LaplacePlan(1, src, 1, 1, 1, 1, trg, 1, 1)
    assert plan.signature() == sig0
    out = _outs(n, m)
    res = A.tune(plan, q, d, v, *out, reps=1, min_gain=-1.0)   # keep every trial that runs: a non-default setting
    assert res["cache"] == path and res["signature"] == sig0 and len(res["trials"]) >= 8
    assert res["knobs"] != {k: knobs0[k] for k in res["knobs"]}
    ent = json.load(open(path))["entries"][sig0]
    assert ent["knobs"] == res["knobs"]
    # a single call on the same geometry takes the tuned knobs from the cache, same bits
    out2 = _outs(n, m)
    assert F.lfmm3dparttarg_device(1, src, q, d, v, out2[0], out2[1], trg, out2[2], out2[3]) == 0
    torch.cuda.synchronize()
    knobs1, sig1 = F.last_tuning()
    assert sig1 == sig0 and knobs1["from_cache"]
    assert {k: knobs1[k] for k in res["knobs"]} == res["knobs"]
    for a, b in zip(out2, ref):
        assert torch.equal(a, b)
    # and so does a new plan
    plan2 = F.LaplacePlan(1, src, 1, 1, 1, 1, trg, 1, 1)
    assert plan2.get_tuning()["from_cache"]
    plan.close()
    plan2.close()
