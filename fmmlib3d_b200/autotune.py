"""Autotuner of the Laplace passes' launch shapes, with a JSON cache.

Knobs (``TUNING_KNOBS``, 0 = automatic):
  m2l_kt      M2L targets per tile (tensor-core form 16..256; FP64 dense operators 16 or 64;
              rotations 1, 2, 4, 8)
  trans_kt    M2M / L2L targets per tile (1, 2, 4, 8)
  tc_variant  tensor-core M2L shared-memory staging (1: K chunks of 16, three stages;
              2: K chunks of 32, two stages)
  overlap     1: near field concurrent with the far field; 2: all passes in order
  p2p_ept     mixed-form P2P: at most 1, 2 or 4 evaluation points per lane

They change launch shapes only: every setting gives the same outputs bitwise.

``tune(plan, ...)`` times the plan's passes (CUDA-graph replays, CUDA events on the
stream the passes run on) by coordinate search: from the plan's current setting, each
knob in turn takes each of its values with the others fixed, and a value is kept when
it is at least ``min_gain`` faster.  The best setting stays in the plan and, unless
``cache`` is False, is written to the JSON cache under the plan's problem signature;
single calls and new plans with that signature then take it (the library reads the
cache when it builds a tree; tuning is never an argument of the reference's API).

Cache file (as the library resolves it): ``set_tuning_cache(path)``, else
``$FMM3D_TUNING_CACHE``, else ``tuning_cache.json`` beside libfmm3d_b200.so.
"""
import datetime
import json
import os

import numpy as np

from . import TUNING_KNOBS, set_tuning_cache, tuning_cache_path, tuning_reload  # noqa: F401

CACHE_FORMAT = "fmm3d_b200 tuning cache"


def candidates(form):
    """(knob, values) in search order for a form (as ``LaplacePlan.get_tuning()["form"]``)."""
    c = []
    if form == "mixed-tc":
        c.append(("m2l_kt", [16, 32, 64, 128, 256]))
    elif form == "fp64-dense":
        c.append(("m2l_kt", [16, 64]))
    elif form == "fp64-rotation":
        c.append(("m2l_kt", [1, 2, 4, 8]))
    c.append(("trans_kt", [1, 2, 4, 8]))
    if form == "mixed-tc":
        c.append(("tc_variant", [1, 2]))
    if form.startswith("mixed"):
        c.append(("p2p_ept", [1, 2, 4]))
    c.append(("overlap", [1, 2]))
    return c


def read_cache(path):
    """The cache's entries ({signature: entry}); {} for a missing or unreadable file."""
    try:
        with open(path) as fh:
            data = json.load(fh)
    except (OSError, ValueError):
        return {}
    if not isinstance(data, dict) or not isinstance(data.get("entries"), dict):
        return {}
    return data["entries"]


def write_cache(path, signature, entry):
    """Add or replace one entry (read, merge, write a temporary file, rename)."""
    entries = read_cache(path)
    entries[signature] = entry
    data = {"format": CACHE_FORMAT, "version": 1, "entries": entries}
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    tmp = "%s.tmp%d" % (path, os.getpid())
    with open(tmp, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
        fh.write("\n")
    os.replace(tmp, path)


def _knobs_only(t):
    return {k: int(t[k]) for k in TUNING_KNOBS}


def tune(plan, charge=None, dipstr=None, dipvec=None, pot=None, fld=None, pottarg=None, fldtarg=None,
         reps=3, min_gain=0.02, cache=True, cache_path=None, stream=None, log=None):
    """Tune ``plan`` (a ``LaplacePlan``) on the given device inputs and outputs (as
    ``LaplacePlan.execute``).  Returns a dict: signature, form, knobs, ms, auto_ms
    (the setting the plan had), trials [(knobs, ms)], cache path (or None)."""
    import torch
    if stream is None:
        # a stream of its own, so that the events and the passes share it
        torch.cuda.synchronize()
        stream = torch.cuda.Stream()
    args = (charge, dipstr, dipvec, pot, fld, pottarg, fldtarg)
    h = stream.cuda_stream

    def run():
        ier = plan.execute(*args, use_graph=True, stream=h)
        if ier != 0:
            from . import last_error
            raise RuntimeError("plan execute ier=%d: %s" % (ier, last_error()))

    def timed(nrep):
        run()                       # capture (a new setting drops the old graph) and warm up
        stream.synchronize()
        ts = []
        for _ in range(nrep):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    start = plan.get_tuning()
    form = start["form"]
    best = _knobs_only(start)
    plan.set_tuning(best)
    t0 = timed(1)
    nrep = reps if t0 < 1000.0 else 1       # passes over a second: one timed replay per setting
    auto_ms = best_ms = timed(nrep)
    trials = [(dict(best), best_ms)]
    if log:
        log("start %s: %.3f ms" % (best, best_ms))
    for knob, values in candidates(form):
        base = dict(best)
        for v in values:
            if v == base[knob]:
                continue
            trial = dict(base)
            trial[knob] = v
            if plan.set_tuning(trial) != 0:
                continue            # not available at this size (shared memory, tile range)
            ms = timed(nrep)
            trials.append((dict(trial), ms))
            if log:
                log("  %s=%d: %.3f ms" % (knob, v, ms))
            if ms < best_ms * (1.0 - min_gain):
                best, best_ms = trial, ms
    plan.set_tuning(best)
    sig = plan.signature()
    out = {"signature": sig, "form": form, "knobs": best, "ms": best_ms, "auto_ms": auto_ms,
           "trials": trials, "cache": None}
    if cache:
        path = cache_path or tuning_cache_path()
        if path and path != "none":
            write_cache(path, sig, {"knobs": best, "ms": round(best_ms, 4), "start_ms": round(auto_ms, 4),
                                    "form": form, "trials": len(trials),
                                    "tuned_at": datetime.datetime.now().isoformat(timespec="seconds")})
            if cache_path is None or os.path.abspath(cache_path) == os.path.abspath(tuning_cache_path()):
                tuning_reload()
            out["cache"] = path
    return out
