#!/usr/bin/env python3
"""Benchmark of the B200 particle FMM on the Laplace 2M-source / 2M-target workload.

Workload (one "step" = one lfmm3dparttarg call): N = 2,000,000 sources and
M = 2,000,000 separate targets, both uniform in the unit cube; complex charges
and dipole strengths with parts uniform in [-1, 1]; dipole directions uniform on
the unit sphere; iprec = 1; potential and field at sources and targets.
Inputs are seeded synthetic data (no dataset is involved).  The step runs in
two arithmetic forms: "mixed" (FP32 compensated P2P and M2L on the tensor
cores with operands split into TF32 pairs, FP64 elsewhere; the headline) and
"fp64" (the reference's arithmetic throughout), both reported.

  value     points/s = (N + M) * steps / device time of the mixed form, inputs
            resident in HBM (fmm3d_lfmm3dparttarg_device), max over ranks.
  e2e       the same metric through the Fortran C ABI (lfmm3dparttarg_) with
            host arrays: H2D of inputs and D2H of outputs inside the timed
            region; pageable numpy arrays (what a Fortran caller passes) as
            the value, pinned arrays beside it.
  roofline  the dominant pass of the step and (roofline.passes) P2P and M2L,
            from the library's per-pass CUDA events of one extra step with the
            passes serialised, against GEMM rates measured in the same run
            (cuBLAS 8192^3: FP32 CUDA cores for the mixed P2P, TF32 tensor cores
            for the mixed M2L, FP64 for the fp64 form) -- MEASURED_PEAKS.json
            holds only HBM and bf16 figures.
  errors    relative L2 error vs the FP64 direct sum at 1,000 seeded sources
            (self excluded) and 1,000 seeded targets, per output.
  cpu_baseline  the C restatement of the reference (oracle/, OpenMP, all host
            cores): one call on the whole workload, with the same inputs; the
            Fortran reference cannot be compiled (no Fortran compiler on
            either machine).
  parity    the oracle's FMM on each workload's own inputs (the headline
            cube, the 100k sphere, the Helmholtz sphere) at the same seeded
            evaluation points as the errors: per output the GPU's FP64 form
            against the oracle's FMM, the oracle's error against its own FP64
            direct sum, the GPU forms' errors, and their ratio to the
            oracle's (the acceptance gate: at most 2).
  laplace_sphere  the CPU-runnable Laplace workload measured in the same run:
            lfmm3dpartself on 100,000 sources on the unit sphere (seed 1),
            charges only, iprec = 1, FP64, with the CPU restatement timed on
            the same input.
  laplace_iprec2  the same N = M = 2M workload at iprec 2 (nterms 26), FP64.
  plans     repeated solves on a fixed geometry: single calls vs plan executes (tree built
            once) vs plan executes replaying a CUDA graph of the passes (sphere 100k and
            10k, FP64; the batched workload as a plan, mixed form).
  batched   4,096 independent Laplace instances in one batched call
            (fmm3d_lfmm3dparttarg_batched_device, one launch per pass): N per
            instance floor(10^U[3, log10 2e5]) (seed 4), geometry per instance
            uniformly a unit cube, a Plummer sphere (scale 0.1, r <= 1) or an
            ellipsoid surface with semi-axes U[0.2, 1]; charges in [-1, 1]^2;
            iprec = 1, mixed form; points/s over all instances and errors at
            sampled points of sampled instances.
  serving   the request loop of fmmlib3d_b200.serving (4 slots, admission by
            projected HBM footprint) on a seeded stream of requests (70%
            Laplace, 30% Helmholtz with zk uniform in [1, 20], N log-uniform in
            [1e3, 1e6], iprec in {0, 1, 2}, cube / Plummer / ellipsoid
            geometries), Poisson arrivals at swept rates: p50/p99 latency and
            points/s per rate (host arrays in and out, copies included);
            serving_mixed: the same stream with the Laplace requests of iprec <= 1
            in the mixed form; serving_repeated: the Laplace requests drawn from
            8 repeated source sets with fresh charges, served by resident plans
            (tree kept on the device, CUDA-graph replay).
  laplace_triangles  lfmm3dtriaself on an icosphere of 327,680 flat
            triangles (unit sphere), single and double layer, iprec 1, FP64;
            errors against the exact direct sum at sampled centroids.
  helmholtz the Helmholtz workload measured in the same run (not the
            headline): hfmm3dpartself on N = 1,000,000 sources uniform on the
            unit sphere, zk = 8 pi, charges uniform in the unit disk, iprec = 2,
            FP64, with its errors, per-pass times and the restatement's time
            on the same inputs.

Multi-GPU: an FMM call does not shard; `--gpus N` runs N independent replicas
(one per rank, scaling "weak"), timed as the max over ranks.
`--impl reference` times the CPU restatement on the host cores (rank 0 only), one call on the
whole headline workload per step.
`--autotune PATH` tunes the Laplace workloads' launch shapes (fmmlib3d_b200.autotune) into the
JSON cache PATH and exits; every measured workload reports the knobs it ran with ("tuning").
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "FMM pts/s at N=2M iprec=1 (FP64 GPU vs mixed), err vs FP64 direct; p50/p99 ms"
UNIT = "points/s"
# dipole + charge pair cost of lpotfld3dall_sdp_targ (src/laprouts3d.f:2394-2416),
# counting sqrt and divide as one flop each
P2P_FLOPS_PER_PAIR = 62
P2P_FLOPS_CHARGE = 31
# DRAM bytes per evaluation point of one mixed-form P2P launch (k_p2p32), from the
# committed ncu capture (profiles/); traffic scales with the points, not the pairs.
P2P_DRAM_BYTES_PER_POINT = 235.2   # 941.0 MB per launch at N = M = 2,000,000 (4M evaluation points)


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=2_000_000, help="sources (= targets)")
    ap.add_argument("--iprec", type=int, default=1)
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="sources (= targets) of the reference arm's steps (0: the workload's own --n)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--err-samples", type=int, default=1000)
    ap.add_argument("--m2l-mode", type=int, default=0, help="0 auto, 1 rotate-shift-rotate, 2 dense operators")
    ap.add_argument("--tensor-m2l", type=int, default=1,
                    help="mixed-form M2L: 0 FP32 CUDA cores, 1/2 tensor cores (tcgen05 split TF32)")
    ap.add_argument("--helm-n", type=int, default=1_000_000, help="sources of the Helmholtz workload (0: skip)")
    ap.add_argument("--helm-cpu-sample", type=int, default=1_000_000,
                    help="sources of the Helmholtz oracle call (parity and CPU baseline; capped at --helm-n)")
    ap.add_argument("--batch-instances", type=int, default=4096, help="instances of the batched workload (0: skip)")
    ap.add_argument("--serve-requests", type=int, default=400, help="requests per serving rate (0: skip)")
    ap.add_argument("--serve-rates", default="20,60,inf", help="Poisson arrival rates (requests/s)")
    ap.add_argument("--autotune", metavar="PATH", default=None,
                    help="tune the Laplace workloads' launch shapes into the JSON cache PATH and exit")
    ap.add_argument("--tri-level", type=int, default=7,
                    help="triangle workload: icosphere subdivision level (20 * 4^level triangles)")
    ap.add_argument("--htri-level", type=int, default=6,
                    help="Helmholtz triangle workload (zk = 4 pi): icosphere subdivision level (0: skip)")
    ap.add_argument("--workload", choices=["all", "laplace", "helmholtz", "batched", "triangles"], default="all",
                    help="all: the Laplace headline line with the other workloads' objects (default); "
                         "laplace / helmholtz / batched: one workload only (profiling runs)")
    return ap.parse_args(argv)


def make_inputs(n, m, seed):
    """Seeded inputs of the workload: Fortran layouts as float64 numpy arrays."""
    rng = np.random.default_rng(seed)
    src = rng.random((n, 3))
    trg = rng.random((m, 3))
    q = rng.uniform(-1, 1, (n, 2))
    dq = rng.uniform(-1, 1, (n, 2))
    dv = rng.normal(size=(n, 3))
    dv /= np.linalg.norm(dv, axis=1)[:, None]
    return src, q, dq, dv, trg


HELM_ZK = 8 * np.pi
HELM_IPREC = 2


def helm_inputs(n, seed=3):
    """Sphere of radius 1 (normalized Gaussian directions), charges uniform in the unit disk."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    src = v / np.linalg.norm(v, axis=1)[:, None]
    r, a = np.sqrt(rng.random(n)), rng.random(n) * 2 * np.pi
    q = np.stack([r * np.cos(a), r * np.sin(a)], -1)
    return src, q


def sphere_inputs(n, seed=1):
    """Unit-sphere surface (normalized Gaussian directions), charges with parts uniform in [-1, 1]."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    src = v / np.linalg.norm(v, axis=1)[:, None]
    return src, rng.uniform(-1, 1, (n, 2))


def run_laplace_sphere(args, R, n=100_000):
    """lfmm3dpartself on the sphere workload: device time (FP64 form), errors, CPU restatement time."""
    torch, F = R["torch"], R["F"]
    src, q = sphere_inputs(n)
    dev = torch.device("cuda", torch.cuda.current_device())
    d_src, d_q = torch.from_numpy(src).to(dev), torch.from_numpy(q).to(dev)
    d_pot = torch.empty((n, 2), dtype=torch.float64, device=dev)
    d_fld = torch.empty((n, 6), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    F.set_precision(0)

    def step():
        ier = F.lfmm3dparttarg_device(1, d_src, d_q, None, None, d_pot, d_fld, stream=stream)
        if ier != 0:
            raise RuntimeError("sphere FMM ier=%d: %s" % (ier, F.last_error()))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(args.steps):
        step()
    ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / args.steps
    rng = np.random.default_rng(97)
    k = min(args.err_samples, n)
    si = np.sort(rng.choice(n, k, replace=False)).astype(np.int32)
    it = torch.from_numpy(si).to(dev)
    dp = torch.empty((k, 2), dtype=torch.float64, device=dev)
    df = torch.empty((k, 6), dtype=torch.float64, device=dev)
    F.direct_points_device(d_src, d_q, None, None, d_src[it.long()].contiguous(), it, dp, df, stream=stream)
    torch.cuda.synchronize()
    out = {"workload": "laplace_lfmm3dpartself_sphere_100k_iprec1", "n_sources": n, "iprec": 1, "dtype": "f64",
           "value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
           "errors": {"pot": float("%.3e" % float(torch.linalg.norm(d_pot[it.long()] - dp) / torch.linalg.norm(dp))),
                      "fld": float("%.3e" % float(torch.linalg.norm(d_fld[it.long()] - df) / torch.linalg.norm(df)))}}
    if R["rank"] == 0 and not args.no_cpu:
        gv = {"pot": d_pot[it.long()].cpu().numpy(), "fld": d_fld[it.long()].cpu().numpy()}
        gd = {"pot": dp.cpu().numpy(), "fld": df.cpu().numpy()}

        def cpu_job(line):
            dt, rep = oracle_laplace_parity(1, src, q, None, None, None, si, None, {"fp64": gv}, gd)
            rep.update(points="%d seeded sources (self excluded)" % k, inputs="the sphere workload's own inputs",
                       oracle_call_s=round(dt, 3))
            line.setdefault("parity", {})["laplace_sphere"] = rep
            out["cpu_baseline"] = {"value": n / dt, "unit": UNIT, "cores": int(os.environ.get("OMP_NUM_THREADS", "1")),
                                   "kind": "port", "sample": "the whole workload, one call (%.2f s)" % dt}

        R.setdefault("cpu_jobs", []).append(cpu_job)
    return out


def run_triangles(args, R, k=7, iprec=1, zk=None):
    """lfmm3dtriaself on a triangulated unit sphere (icosphere of 20 * 4^k flat triangles), single and
    double layer with densities in [-1, 1]^2, iprec 1, FP64: device time, errors against the exact
    direct sum at sampled centroids, and the oracle (parity, CPU baseline) on the same inputs.
    With zk: hfmm3dtriaself (Helmholtz, FP64 only), errors against the direct sum of the same
    near-field rule (h3dtriadirect)."""
    from fmmlib3d_b200.meshes import icosphere, normals_centroids
    torch, F = R["torch"], R["F"]
    T = icosphere(k)
    nrm, cen = normals_centroids(T)
    n = len(T)
    rng = np.random.default_rng(11)
    q = np.stack([rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)], 1)
    dq = np.stack([rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)], 1)
    dev = torch.device("cuda", torch.cuda.current_device())
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64).reshape(n, -1)).to(dev)
    d_tri, d_nrm, d_cen, d_q, d_dq = d(T.reshape(n, 9)), d(nrm), d(cen), d(q), d(dq)
    d_pot = torch.empty((n, 2), dtype=torch.float64, device=dev)
    d_fld = torch.empty((n, 6), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream

    def step(pot=d_pot, fld=d_fld):
        if zk is None:
            ier = F.lfmm3dtriatarg_device(iprec, d_tri, d_nrm, d_cen, d_q, d_dq, pot, fld, stream=stream)
        else:
            ier = F.hfmm3dtriatarg_device(iprec, zk, d_tri, d_nrm, d_cen, d_q, d_dq, pot, fld, stream=stream)
        if ier != 0:
            raise RuntimeError("triangle FMM ier=%d: %s" % (ier, F.last_error()))

    def timed(**kw):
        for _ in range(args.warmup):
            step(**kw)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(args.steps):
            step(**kw)
        ev[1].record()
        torch.cuda.synchronize()
        t = ev[0].elapsed_time(ev[1]) / args.steps
        F.set_timing(True)
        step(**kw)
        torch.cuda.synchronize()
        ps = F.last_timing()
        F.set_timing(False)
        return t, ps

    ms, passes = timed()
    m_pot = m_fld = None
    if zk is None:
        # the mixed form: M2L on the tensor cores, the exact near field FP64
        m_pot = torch.empty_like(d_pot)
        m_fld = torch.empty_like(d_fld)
        F.set_precision(1)
        try:
            ms_mixed, passes_mixed = timed(pot=m_pot, fld=m_fld)
        finally:
            F.set_precision(0)
    m = min(args.err_samples, n)
    si = np.sort(rng.choice(n, m, replace=False)).astype(np.int32)
    it = torch.from_numpy(si).to(dev)
    dp = torch.empty((m, 2), dtype=torch.float64, device=dev)
    df = torch.empty((m, 6), dtype=torch.float64, device=dev)
    # the near-field rule degree of hfmm3dtriatarg (src/hfmm3dtria.f:730-751)
    nqtri = 2 if iprec in (-2, -1) else 4 if iprec == 0 else 6 if iprec >= 1 else 1
    if zk is None:
        ier = F.tri_direct_points_device(d_tri, d_q, d_dq, d_cen[it.long()].contiguous(), it, dp, df, stream=stream)
    else:
        ier = F.htri_direct_points_device(nqtri, zk, d_tri, d_q, d_dq, d_cen[it.long()].contiguous(), it, dp, df,
                                          stream=stream)
    torch.cuda.synchronize()
    if ier != 0:
        raise RuntimeError("triangle direct ier=%d" % ier)
    gp, gf = d_pot[it.long()], d_fld[it.long()]
    kind = "laplace_lfmm3dtriaself" if zk is None else "helmholtz_hfmm3dtriaself_zk%g" % zk.real
    out = {"workload": "%s_icosphere_%d_triangles_iprec%d" % (kind, n, iprec), "n_triangles": n,
           "iprec": iprec, "dtype": "f64", "value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
           "pass_ms": {kk: round(v, 3) for kk, v in passes.items()},
           "errors": {"pot": float("%.3e" % float(torch.linalg.norm(gp - dp) / torch.linalg.norm(dp))),
                      "fld": float("%.3e" % float(torch.linalg.norm(gf - df) / torch.linalg.norm(df)))},
           "note": "errors against the direct sum (%s) at %d sampled centroids"
                   % ("l3dtriadirect" if zk is None else "h3dtriadirect, nqtri %d" % nqtri, m)}
    if zk is not None:
        out["zk"] = [zk.real, zk.imag]
    forms = {"fp64": None}
    if m_pot is not None:
        mp, mf = m_pot[it.long()], m_fld[it.long()]
        out["mixed"] = {"value": n / (ms_mixed * 1e-3), "ms_per_step": ms_mixed,
                        "pass_ms": {kk: round(v, 3) for kk, v in passes_mixed.items()},
                        "errors": {"pot": float("%.3e" % float(torch.linalg.norm(mp - dp) / torch.linalg.norm(dp))),
                                   "fld": float("%.3e" % float(torch.linalg.norm(mf - df) / torch.linalg.norm(df)))},
                        "form": "M2L on the tensor cores (split TF32); near field and other passes FP64"}
    if R["rank"] == 0 and not args.no_cpu:
        forms["fp64"] = {"pot": gp.cpu().numpy(), "fld": gf.cpu().numpy()}
        if m_pot is not None:
            forms["mixed"] = {"pot": mp.cpu().numpy(), "fld": mf.cpu().numpy()}
        gd = {"pot": dp.cpu().numpy(), "fld": df.cpu().numpy()}
        key = "laplace_triangles" if zk is None else "helmholtz_triangles"

        def cpu_job(line):
            import oracle
            c = lambda a: a[:, 0] + 1j * a[:, 1]
            t0 = time.perf_counter()
            if zk is None:
                oier, opot, ofld, _, _ = oracle.lfmm3dtriatarg(iprec, T, nrm, cen, c(q), c(dq))
            else:
                oier, opot, ofld, _, _ = oracle.hfmm3dtriatarg(iprec, zk, T, nrm, cen, c(q), c(dq))
            dt = time.perf_counter() - t0
            if oier != 0:
                raise RuntimeError("oracle ier=%d" % oier)
            if zk is None:
                tp, tf = oracle.tri_direct_at(T, cen[si], si, c(q), c(dq))
            else:
                tp, tf = oracle.htri_direct_at(zk, T, cen[si], si, c(q), c(dq), nqtri=nqtri)
            rep = parity_report({"pot": _as_pairs(opot[si], 2), "fld": _as_pairs(ofld[si], 6)},
                                {"pot": _as_pairs(tp, 2), "fld": _as_pairs(tf, 6)}, forms, gd)
            rep.update(points="%d seeded centroids (own triangle in-plane)" % m,
                       inputs="the triangle workload's own inputs", oracle_call_s=round(dt, 2))
            line.setdefault("parity", {})[key] = rep
            out["cpu_baseline"] = {"value": n / dt, "unit": UNIT, "cores": int(os.environ.get("OMP_NUM_THREADS", "1")),
                                   "kind": "port", "sample": "the whole workload, one call (%.1f s)" % dt}

        R.setdefault("cpu_jobs", []).append(cpu_job)
    return out


def run_plans(args, R, batch=None):
    """Repeated solves on a fixed geometry: single calls vs plan executes (tree built once) vs plan
    executes replaying a CUDA graph of the passes.  Sphere workloads (FP64) of 100k (cfg1) and 10k
    sources, and, when given, the batched workload (mixed form) as a plan."""
    torch, F = R["torch"], R["F"]
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream().cuda_stream
    out = {}

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    F.set_precision(0)
    for n in (100_000, 10_000):
        src, q = sphere_inputs(n)
        d_src, d_q = torch.from_numpy(src).to(dev), torch.from_numpy(q).to(dev)
        pot = torch.empty((n, 2), dtype=torch.float64, device=dev)
        fld = torch.empty((n, 6), dtype=torch.float64, device=dev)
        single = timed(lambda: F.lfmm3dparttarg_device(1, d_src, d_q, None, None, pot, fld, stream=stream), 20)
        t0 = time.perf_counter()
        plan = F.LaplacePlan(1, d_src, 1, 0, 1, 1, stream=stream)
        create = 1e3 * (time.perf_counter() - t0)
        plain = timed(lambda: plan.execute(d_q, None, None, pot, fld, use_graph=False, stream=stream), 20)
        graph = timed(lambda: plan.execute(d_q, None, None, pot, fld, use_graph=True, stream=stream), 20)
        out["sphere_%dk" % (n // 1000)] = {
            "n_sources": n, "dtype": "f64", "single_call_ms": round(single, 3), "plan_create_ms": round(create, 3),
            "plan_execute_ms": round(plain, 3), "plan_graph_execute_ms": round(graph, 3),
            "kernels_per_execute": F.last_launches(), "graph_points_per_s": n / (graph * 1e-3)}
        plan.close()
    if batch is not None:
        d_src, d_q, off, pot, fld = batch
        F.set_precision(1)
        F.set_tensor_m2l(args.tensor_m2l)
        t0 = time.perf_counter()
        plan = F.LaplacePlan(1, d_src, 1, 0, 1, 1, stream=stream, src_offsets=off)
        create = 1e3 * (time.perf_counter() - t0)
        graph = timed(lambda: plan.execute(d_q, None, None, pot, fld, use_graph=True, stream=stream), 2)
        n = int(off[-1])
        out["batched"] = {"instances": len(off) - 1, "n_total": n, "dtype": "mixed", "plan_create_ms": round(create, 1),
                          "plan_graph_execute_ms": round(graph, 1), "kernels_per_execute": F.last_launches(),
                          "graph_points_per_s": n / (graph * 1e-3)}
        plan.close()
        F.set_precision(0)
    return out


def batched_inputs(k, seed=4):
    """The batched workload's instances, concatenated: (sources, charges, offsets)."""
    rng = np.random.default_rng(seed)
    srcs, qs = [], []
    for _ in range(k):
        n = int(10 ** rng.uniform(3, np.log10(2e5)))
        g = int(rng.integers(3))
        if g == 0:
            src = rng.random((n, 3))
        elif g == 1:
            parts, have = [], 0
            while have < n:
                u = rng.random(n)
                r = 0.1 / np.sqrt(np.maximum(u ** (-2 / 3) - 1, 1e-300))
                v = rng.normal(size=(n, 3))
                keep = r <= 1
                p = v[keep] / np.linalg.norm(v[keep], axis=1)[:, None] * r[keep][:, None]
                parts.append(p)
                have += len(p)
            src = np.concatenate(parts)[:n]
        else:
            v = rng.normal(size=(n, 3))
            src = v / np.linalg.norm(v, axis=1)[:, None] * rng.uniform(0.2, 1, 3)
        srcs.append(src)
        qs.append(rng.uniform(-1, 1, (n, 2)))
    off = np.concatenate([[0], np.cumsum([len(x) for x in srcs])]).astype(np.int32)
    return np.concatenate(srcs), np.concatenate(qs), off


def run_batched(args, R):
    torch, F = R["torch"], R["F"]
    src, q, off = batched_inputs(args.batch_instances)
    n = int(off[-1])
    dev = torch.device("cuda", torch.cuda.current_device())
    d_src, d_q = torch.from_numpy(src).to(dev), torch.from_numpy(q).to(dev)
    d_pot = torch.empty((n, 2), dtype=torch.float64, device=dev)
    d_fld = torch.empty((n, 6), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    F.set_precision(1)
    F.set_tensor_m2l(args.tensor_m2l)
    F.set_timing(True)

    def step():
        ier = F.lfmm3dparttarg_batched_device(1, off, d_src, d_q, None, None, d_pot, d_fld, stream=stream)
        if ier != 0:
            raise RuntimeError("batched FMM ier=%d: %s" % (ier, F.last_error()))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    steps = max(1, min(args.steps, 3))
    passes, launches = [], []
    ev[0].record()
    for _ in range(steps):
        step()
        passes.append(F.last_timing())
        launches.append(F.last_launches())
    ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / steps
    knobs, _ = F.last_tuning()
    # errors: 50 points of each of 20 seeded instances against the FP64 direct sum
    rng = np.random.default_rng(96)
    num = {"pot": 0.0, "fld": 0.0}
    den = {"pot": 0.0, "fld": 0.0}
    for i in rng.choice(args.batch_instances, min(20, args.batch_instances), replace=False):
        a, b = int(off[i]), int(off[i + 1])
        k = min(50, b - a)
        idx = np.sort(rng.choice(b - a, k, replace=False)).astype(np.int32)
        it = torch.from_numpy(idx).to(dev)
        dp = torch.empty((k, 2), dtype=torch.float64, device=dev)
        df = torch.empty((k, 6), dtype=torch.float64, device=dev)
        F.direct_points_device(d_src[a:b], d_q[a:b], None, None, d_src[a:b][it.long()].contiguous(), it, dp, df,
                               stream=stream)
        torch.cuda.synchronize()
        gp, gf = d_pot[a:b][it.long()], d_fld[a:b][it.long()]
        num["pot"] += float(torch.sum((gp - dp) ** 2)); den["pot"] += float(torch.sum(dp ** 2))
        num["fld"] += float(torch.sum((gf - df) ** 2)); den["fld"] += float(torch.sum(df ** 2))
    F.set_precision(0)
    R["batch_arrays"] = (d_src, d_q, off, d_pot, d_fld)
    mean = {kk: round(float(np.mean([p[kk] for p in passes])), 3) for kk in passes[0]}
    return {"workload": "laplace_batched_%d_instances_logN_1e3_2e5_iprec1_mixed" % args.batch_instances,
            "instances": args.batch_instances, "n_total": n, "value": n / (ms * 1e-3), "unit": UNIT,
            "ms_per_step": ms, "steps": steps, "gpu_launches_per_step": int(np.mean(launches)),
            "errors": {kk: float("%.3e" % np.sqrt(num[kk] / den[kk])) for kk in num}, "pass_ms_mean": mean,
            "tuning": knobs}


def run_serving(args, precision=None, geometries=0, rates=None):
    """Swept-rate serving measurement (one warm-up pass over the same requests first); precision 1
    serves the Laplace requests with iprec <= 1 in the mixed form; geometries > 0 draws the Laplace
    requests from that many repeated source sets, served by resident plans."""
    from fmmlib3d_b200.serving import FMMServer, make_request_stream, run_stream
    reqs = make_request_stream(args.serve_requests, seed=7, geometries=geometries)
    srv = FMMServer(slots=4, precision=precision)
    out = {"slots": 4, "requests_per_rate": len(reqs), "mean_n": float(np.mean([len(r.source) for r in reqs])),
           "laplace_fraction": float(np.mean([r.kernel == "laplace" for r in reqs])),
           "precision": "mixed for Laplace iprec <= 1" if precision == 1 else "fp64", "rates": []}
    if geometries:
        out["repeated_geometries"] = geometries
    try:
        run_stream(srv, reqs, float("inf"))  # warm-up: memory pools, operator plans, resident geometry plans
        for rate in [float(x) for x in (rates or args.serve_rates).split(",")]:
            st, _ = run_stream(srv, reqs, rate, seed=int(rate) if rate != float("inf") else 0)
            st["rate_hz"] = None if rate == float("inf") else rate
            out["rates"].append({k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()})
        out["max_on_gpu"] = srv.max_running
        if geometries:
            out.update({k: v for k, v in srv.stats().items() if k.startswith("plan") or k.startswith("resident")})
    finally:
        srv.close()
    if geometries:
        # the same stream with plans switched off: every request rebuilds its tree
        srv = FMMServer(slots=4, precision=precision, plan_bytes=0)
        try:
            run_stream(srv, reqs, float("inf"))
            st, _ = run_stream(srv, reqs, float("inf"), seed=0)
            out["saturated_without_plans"] = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()
                                              if k in ("points_per_s", "p50_ms", "p99_ms", "max_ier")}
        finally:
            srv.close()
    return out


def cpu_helm_sample(n):
    """One hfmm3dpartself restatement call on the sphere workload with n sources; returns seconds."""
    import oracle
    src, q = helm_inputs(n, seed=3)
    t0 = time.perf_counter()
    ier = oracle.hfmm3dparttarg(HELM_IPREC, HELM_ZK, src, q[:, 0] + 1j * q[:, 1])[0]
    t1 = time.perf_counter()
    if ier != 0:
        raise RuntimeError("oracle ier=%d" % ier)
    return t1 - t0


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reduce_max(dist, value, device):
    """Max of a per-rank float over all ranks (the replicas' device time); plain value on one rank."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons.  The sampler starts before the
    warm-up (nvidia-smi needs a few hundred ms to produce its first line), every sample
    carries nvidia-smi's timestamp, and only the samples inside the timed window
    (`begin()` .. `stop()`, host wall clock) are summarised."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, interval_ms=25):
        self.gpu = gpu_index
        self.proc = None
        self.interval_ms = interval_ms
        self.t0 = None
        self.path = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(prefix="fmm3d_clocks_gpu%d_" % self.gpu, suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def begin(self):
        """Start of the timed window."""
        import datetime
        self.t0 = datetime.datetime.now()

    def stop(self):
        if self.proc is None:
            return None
        import datetime
        t1 = datetime.datetime.now()
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
                rows.append((ts, float(f[2]), float(f[3]), f[6:10]))
            except ValueError:
                continue
        try:
            os.unlink(self.path)
        except OSError:
            pass
        if not rows:
            return None
        inside = [r for r in rows if self.t0 is None or self.t0 <= r[0] <= t1]
        window = bool(inside)
        use = inside or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = {nm for r in use for nm, v in zip(names, r[3]) if v.lower() == "active"}
        mx = use[-1][2]
        sm = [r[1] for r in use]
        loaded = [v for v in sm if mx and v > 0.5 * mx] or sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "in_timed_window": window, "interval_ms": self.interval_ms}


def measured_peak(torch, dev, dtype, tf32=False):
    """cuBLAS GEMM throughput (8192^3, best of 5) in TFLOP/s for dtype; FP32 inputs run on the
    CUDA cores (TF32 off) or, with tf32=True, on the tensor cores in TF32."""
    torch.backends.cuda.matmul.allow_tf32 = bool(tf32)
    a = torch.randn(8192, 8192, dtype=dtype, device=dev)
    b = torch.randn(8192, 8192, dtype=dtype, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    return 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12


def cpu_fmm_sample(n, iprec, seed=2):
    """One run of the CPU restatement (oracle/) on n sources + n targets; returns (seconds, points)."""
    import oracle
    src, q, dq, dv, trg = make_inputs(n, n, seed)
    t0 = time.perf_counter()
    ier = oracle.lfmm3dparttarg(iprec, src, q[:, 0] + 1j * q[:, 1], dq[:, 0] + 1j * dq[:, 1], dv, trg)[0]
    t1 = time.perf_counter()
    if ier != 0:
        raise RuntimeError("oracle ier=%d" % ier)
    return t1 - t0, 2 * n


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def sample_indices(n, m, k, seed=99):
    """The seeded evaluation points of the error and parity checks: k sources and k targets."""
    rng = np.random.default_rng(seed)
    si = np.sort(rng.choice(n, min(k, n), replace=False)).astype(np.int32)
    ti = np.sort(rng.choice(m, min(k, m), replace=False)).astype(np.int32) if m else np.zeros(0, np.int32)
    return si, ti


def _as_pairs(z, width):
    """complex (k,) or (k,3) -> float64 (k, width) in the library's interleaved layout."""
    return np.ascontiguousarray(z).view(np.float64).reshape(len(z), width)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(float(np.linalg.norm(b)), 1e-300))


def parity_report(oracle_vals, direct_vals, gpu_forms, gpu_direct=None, gate=2.0):
    """Per output: the GPU's FP64 form against the oracle's FMM on the same points, each error
    against the oracle's FP64 direct sum, and the GPU errors divided by the oracle's (the
    acceptance criterion: at most `gate`).  gpu_forms maps a form name to its sampled outputs."""
    out = {}
    ok = True
    for key in oracle_vals:
        o, d = oracle_vals[key], direct_vals[key]
        e_or = _rel(o, d)
        row = {"oracle_err": float("%.3e" % e_or)}
        for form, vals in gpu_forms.items():
            e = _rel(vals[key], d)
            row["gpu_%s_err" % form] = float("%.3e" % e)
            row["%s_over_oracle" % form] = round(e / max(e_or, 1e-300), 3)
            ok = ok and e <= gate * e_or
            if form == "fp64":
                row["gpu_fp64_vs_oracle"] = float("%.3e" % _rel(vals[key], o))
        if gpu_direct is not None:
            row["gpu_direct_vs_oracle_direct"] = float("%.3e" % _rel(gpu_direct[key], d))
        out[key] = row
    out["gate"] = "GPU error <= %g x the oracle's, per output" % gate
    out["pass"] = bool(ok)
    return out


def oracle_laplace_parity(iprec, src, q, dq, dv, trg, si, ti, gpu_forms, gpu_direct=None):
    """The oracle's FMM (the C restatement of lfmm3dparttarg, OpenMP over all host cores) on the
    whole workload, timed, and its FP64 direct sum at the sampled points; returns (seconds, report)."""
    import oracle
    c = lambda a: None if a is None else a[:, 0] + 1j * a[:, 1]
    t0 = time.perf_counter()
    ier, pot, fld, pt, ft = oracle.lfmm3dparttarg(iprec, src, c(q), c(dq), dv, trg)
    dt = time.perf_counter() - t0
    if ier != 0:
        raise RuntimeError("oracle ier=%d" % ier)
    ov = {"pot": _as_pairs(pot[si], 2), "fld": _as_pairs(fld[si], 6)}
    dp, df = oracle.direct_at(src, src[si], si, c(q), c(dq), dv)
    dv_ = {"pot": _as_pairs(dp, 2), "fld": _as_pairs(df, 6)}
    if trg is not None and len(ti):
        ov.update(pottarg=_as_pairs(pt[ti], 2), fldtarg=_as_pairs(ft[ti], 6))
        tp, tf = oracle.direct_at(src, trg[ti], None, c(q), c(dq), dv)
        dv_.update(pottarg=_as_pairs(tp, 2), fldtarg=_as_pairs(tf, 6))
    return dt, parity_report(ov, dv_, gpu_forms, gpu_direct)


def oracle_helm_parity(S):
    """The oracle's hfmm3dpartself (C restatement, OpenMP) on the Helmholtz workload's own inputs,
    timed, against the GPU's FP64 outputs at the sampled sources; returns (seconds, report)."""
    import oracle
    src, q, si = S["src"], S["q"][:, 0] + 1j * S["q"][:, 1], S["si"]
    t0 = time.perf_counter()
    ier, pot, fld, _, _ = oracle.hfmm3dparttarg(HELM_IPREC, HELM_ZK, src, q)
    dt = time.perf_counter() - t0
    if ier != 0:
        raise RuntimeError("oracle ier=%d" % ier)
    dp, df = oracle.hdirect_at(HELM_ZK, src, src[si], si, q)
    rep = parity_report({"pot": _as_pairs(pot[si], 2), "fld": _as_pairs(fld[si], 6)},
                        {"pot": _as_pairs(dp, 2), "fld": _as_pairs(df, 6)},
                        {"fp64": {"pot": S["pot"], "fld": S["fld"]}},
                        {"pot": S["direct_pot"], "fld": S["direct_fld"]})
    rep.update(points="%d seeded sources (self excluded)" % len(si), inputs="the Helmholtz workload's own inputs",
               oracle_call_s=round(dt, 2))
    return dt, rep


def run_b200(args):
    import torch
    import torch.distributed as dist
    import fmmlib3d_b200 as F

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    n = m = args.n
    src, q, dq, dv, trg = make_inputs(n, m, 2 + rank)
    g = lambda a: torch.from_numpy(a).to(dev)
    d_src, d_q, d_dq, d_dv, d_trg = g(src), g(q), g(dq), g(dv), g(trg)
    d_pot = torch.empty((n, 2), dtype=torch.float64, device=dev)
    d_fld = torch.empty((n, 6), dtype=torch.float64, device=dev)
    d_pt = torch.empty((m, 2), dtype=torch.float64, device=dev)
    d_ft = torch.empty((m, 6), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    F.set_m2l_mode(args.m2l_mode)
    F.set_tensor_m2l(args.tensor_m2l)

    def step():
        ier = F.lfmm3dparttarg_device(args.iprec, d_src, d_q, d_dq, d_dv, d_pot, d_fld, d_trg, d_pt, d_ft,
                                      stream=stream)
        if ier != 0:
            raise RuntimeError("FMM ier=%d: %s" % (ier, F.last_error()))

    def errors():
        """Relative L2 errors vs the GPU's FP64 direct sum at the sampled points, and the sampled
        values themselves (FMM outputs and direct sums, for the parity check against the oracle)."""
        si, ti = sample_indices(n, m, args.err_samples)
        k = len(si)
        out, vals = {}, {"si": si, "ti": ti}
        dp = torch.empty((k, 2), dtype=torch.float64, device=dev)
        df = torch.empty((k, 6), dtype=torch.float64, device=dev)
        for name, idx, pts, skip, P, Fd in (("src", si, d_src[si], torch.from_numpy(si).to(dev), d_pot, d_fld),
                                            ("targ", ti, d_trg[ti], None, d_pt, d_ft)):
            ier = F.direct_points_device(d_src, d_q, d_dq, d_dv, pts.contiguous(), skip, dp, df, stream=stream)
            torch.cuda.synchronize()
            if ier != 0:
                raise RuntimeError("direct ier=%d" % ier)
            it = torch.from_numpy(idx).to(dev).long()
            kp, kf = ("pot", "fld") if name == "src" else ("pottarg", "fldtarg")
            out[kp] = float(torch.linalg.norm(P[it] - dp) / torch.linalg.norm(dp))
            out[kf] = float(torch.linalg.norm(Fd[it] - df) / torch.linalg.norm(df))
            vals[kp], vals[kf] = P[it].cpu().numpy(), Fd[it].cpu().numpy()
            vals["direct_" + kp], vals["direct_" + kf] = dp.cpu().numpy(), df.cpu().numpy()
        return out, vals

    def measure(form):
        F.set_precision(form)
        F.set_timing(True)
        clk = ClockSampler(local)
        clk.start()
        for w in range(args.warmup):
            F.set_stats(w == args.warmup - 1)   # tree statistics from the last warm-up call only
            step()
        F.set_stats(False)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clk.begin()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        passes, launches = [], []
        ev[0].record()
        for k in range(args.steps):
            step()
            ev[k + 1].record()
            passes.append(F.last_timing())
            launches.append(F.last_launches())
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        clocks = clk.stop()
        knobs, _ = F.last_tuning()
        # one more step with the passes serialised, after the timed region: per-kernel
        # times for the roofline (with the default overlap the near-field kernel shares the GPU)
        F.set_overlap(False)
        step()
        serial = F.last_timing()
        F.set_overlap(True)
        step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
        total_ms = ev[0].elapsed_time(ev[args.steps])
        total_ms = reduce_max(dist if ws > 1 else None, total_ms, dev)
        errs, vals = errors()
        return dict(total_ms=total_ms, step_ms=step_ms, passes=passes, launches=launches, stats=F.last_stats(),
                    clocks=clocks, errs=errs, samples=vals, points=n + m, serial=serial, tuning=knobs)

    forms = {"mixed": measure(1), "fp64": measure(0)}
    peaks = {"fp64": measured_peak(torch, dev, torch.float64), "fp32": measured_peak(torch, dev, torch.float32),
             "tf32": measured_peak(torch, dev, torch.float32, tf32=True)}
    return dict(n=n, m=m, ws=ws, rank=rank, forms=forms, peaks=peaks, torch=torch, F=F,
                dist=dist if ws > 1 else None, arrays=(src, q, dq, dv, trg))


def run_iprec2(args, R, steps=2):
    """The same N = M workload at iprec 2 (nterms 26), FP64 form (the mixed form covers iprec <= 1)."""
    torch, F = R["torch"], R["F"]
    src, q, dq, dv, trg = R["arrays"]
    n, m = R["n"], R["m"]
    dev = torch.device("cuda", torch.cuda.current_device())
    g = lambda a: torch.from_numpy(a).to(dev)
    d_src, d_q, d_dq, d_dv, d_trg = g(src), g(q), g(dq), g(dv), g(trg)
    pot, fld = torch.empty((n, 2), dtype=torch.float64, device=dev), torch.empty((n, 6), dtype=torch.float64, device=dev)
    pt, ft = torch.empty((m, 2), dtype=torch.float64, device=dev), torch.empty((m, 6), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    F.set_precision(0)
    F.set_timing(True)
    step = lambda: F.lfmm3dparttarg_device(2, d_src, d_q, d_dq, d_dv, pot, fld, d_trg, pt, ft, stream=stream)
    step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    passes = []
    for _ in range(steps):
        if step() != 0:
            raise RuntimeError("iprec 2 FMM failed: %s" % F.last_error())
        passes.append(F.last_timing())
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    rng = np.random.default_rng(98)
    k = 500
    si = np.sort(rng.choice(n, k, replace=False)).astype(np.int32)
    it = torch.from_numpy(si).to(dev)
    dp, df = torch.empty((k, 2), dtype=torch.float64, device=dev), torch.empty((k, 6), dtype=torch.float64, device=dev)
    F.direct_points_device(d_src, d_q, d_dq, d_dv, d_src[it.long()].contiguous(), it, dp, df, stream=stream)
    torch.cuda.synchronize()
    err = lambda a, b: float("%.3e" % float(torch.linalg.norm(a - b) / torch.linalg.norm(b)))
    return {"workload": "laplace_lfmm3dparttarg_cube_2M_src_2M_targ_iprec2", "dtype": "f64",
            "value": (n + m) / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "steps": steps,
            "errors": {"pot": err(pot[it.long()], dp), "fld": err(fld[it.long()], df)},
            "pass_ms_mean": {kk: round(float(np.mean([p[kk] for p in passes])), 3) for kk in passes[0]}}


def run_e2e(args, R):
    """Same workload through the Fortran C ABI (lfmm3dparttarg_) with host arrays, H2D of the inputs
    and D2H of the outputs inside the timed region: pageable arrays (what a Fortran or numpy caller
    passes; the headline) and pinned arrays."""
    torch, F = R["torch"], R["F"]
    src, q, dq, dv, trg = R["arrays"]
    n, m = R["n"], R["m"]
    import ctypes
    lib = F.lib()
    I = lambda v: ctypes.byref(ctypes.c_int(v))
    ier = ctypes.c_int(0)

    def measure(ins, outs, ptr):
        P = lambda a: ctypes.c_void_p(ptr(a))

        def call():
            lib.lfmm3dparttarg_(ctypes.byref(ier), I(args.iprec), I(n), P(ins[0]), I(1), P(ins[1]), I(1), P(ins[2]),
                                P(ins[3]), I(1), P(outs[0]), I(1), P(outs[1]), I(m), P(ins[4]), I(1), P(outs[2]), I(1),
                                P(outs[3]))
            if ier.value != 0:
                raise RuntimeError("e2e ier=%d" % ier.value)

        for _ in range(args.warmup):
            call()
        torch.cuda.synchronize()
        if R["dist"] is not None:
            R["dist"].barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            call()  # synchronous: returns after the outputs are in host memory
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        return reduce_max(R["dist"], dt, "cuda")

    shapes = ((n, 2), (n, 6), (m, 2), (m, 6))
    # pageable: plain numpy arrays (outputs freshly allocated, as a caller's own arrays)
    ins = [np.ascontiguousarray(a) for a in (src, q, dq, dv, trg)]
    outs = [np.empty(sh) for sh in shapes]
    dt_page = measure(ins, outs, lambda a: a.ctypes.data)

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        return t

    h = [pinned(a) for a in ins]
    houts = [torch.empty(sh, dtype=torch.float64, pin_memory=True) for sh in shapes]
    dt_pin = measure(h, houts, lambda t: t.data_ptr())
    h2d = n * (24 + 16 + 16 + 24) + m * 24
    d2h = n * (16 + 48) + m * (16 + 48)
    rate = lambda dt: R["ws"] * (n + m) * args.steps / dt
    return {"value": rate(dt_page), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": 1e3 * dt_page / args.steps, "host_memory": "pageable (numpy arrays)",
            "pinned": {"value": rate(dt_pin), "ms_per_step": 1e3 * dt_pin / args.steps}}


def run_helm(args, R):
    """The Helmholtz sphere workload on the device (hfmm3dpartself, FP64)."""
    torch, F = R["torch"], R["F"]
    n = args.helm_n
    src, q = helm_inputs(n, seed=3 + R["rank"])
    dev = torch.device("cuda", torch.cuda.current_device())
    d_src, d_q = torch.from_numpy(src).to(dev), torch.from_numpy(q).to(dev)
    d_pot = torch.empty((n, 2), dtype=torch.float64, device=dev)
    d_fld = torch.empty((n, 6), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream

    def step():
        ier = F.hfmm3dparttarg_device(HELM_IPREC, HELM_ZK, d_src, d_q, None, None, d_pot, d_fld, stream=stream)
        if ier != 0:
            raise RuntimeError("Helmholtz FMM ier=%d: %s" % (ier, F.last_error()))

    F.set_timing(True)
    for w in range(args.warmup):
        F.set_stats(w == args.warmup - 1)
        step()
    F.set_stats(False)
    stats = F.last_stats()
    torch.cuda.synchronize()
    if R["dist"] is not None:
        R["dist"].barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    passes = []
    ev[0].record()
    for k in range(args.steps):
        step()
        ev[k + 1].record()
        passes.append(F.last_timing())
    torch.cuda.synchronize()
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[args.steps])
    total_ms = reduce_max(R["dist"], total_ms, dev)
    # errors at 1,000 seeded sources against the FP64 direct sum
    rng = np.random.default_rng(98)
    k = min(args.err_samples, n)
    si = np.sort(rng.choice(n, k, replace=False)).astype(np.int32)
    dp = torch.empty((k, 2), dtype=torch.float64, device=dev)
    df = torch.empty((k, 6), dtype=torch.float64, device=dev)
    it = torch.from_numpy(si).to(dev)
    ier = F.hdirect_points_device(HELM_ZK, d_src, d_q, None, None, d_src[it.long()].contiguous(), it, dp, df,
                                  stream=stream)
    torch.cuda.synchronize()
    if ier != 0:
        raise RuntimeError("Helmholtz direct ier=%d" % ier)
    errs = {"pot": float(torch.linalg.norm(d_pot[it.long()] - dp) / torch.linalg.norm(dp)),
            "fld": float(torch.linalg.norm(d_fld[it.long()] - df) / torch.linalg.norm(df))}
    R["helm_samples"] = dict(src=src, q=q, si=si, pot=d_pot[it.long()].cpu().numpy(),
                             fld=d_fld[it.long()].cpu().numpy(), direct_pot=dp.cpu().numpy(),
                             direct_fld=df.cpu().numpy())
    mean = {kk: round(float(np.mean([p[kk] for p in passes])), 3) for kk in passes[0]}
    out = {"workload": "helmholtz_hfmm3dpartself_sphere_%dk_zk_8pi_iprec2" % (n // 1000), "n_sources": n,
           "zk": "8*pi", "iprec": HELM_IPREC, "dtype": "f64",
           "value": R["ws"] * n * args.steps / (total_ms * 1e-3), "unit": UNIT,
           "ms_per_step": total_ms / args.steps, "p50_ms": float(np.percentile(step_ms, 50)),
           "p99_ms": float(np.percentile(step_ms, 99)), "errors": {kk: float("%.3e" % v) for kk, v in errs.items()},
           "pass_ms_mean": mean, "stats": {kk: v for kk, v in stats.items() if kk != "m2l_pt_hist"},
           "p2p_pairs_per_s": stats.get("p2p_pairs", 0) / (mean["p2p"] * 1e-3) if mean.get("p2p") else None}
    return out


PEAK_SOURCE = {"fp64": "cuBLAS DGEMM 8192^3", "fp32": "cuBLAS SGEMM 8192^3 (TF32 off, CUDA cores)",
               "tf32": "cuBLAS SGEMM 8192^3 with TF32 (tensor cores)"}


def roofline_of(M, peaks, form, tensor_m2l=False, iprec=1):
    """Roofline of the dominant pass (and of P2P and M2L separately) of one form, from the per-pass
    CUDA events of its timed steps.  P2P and M2L are compute passes: P2P on the CUDA cores (FP32 in
    the mixed form, FP64 otherwise), M2L on the tensor cores (TF32) when the mixed form runs it there.
    Peaks are cuBLAS GEMM rates measured in the same run (MEASURED_PEAKS.json holds HBM and bf16
    figures only)."""
    keys = [k for k in M["passes"][0] if k not in ("total",)]
    mean = {k: float(np.mean([p[k] for p in M["passes"]])) for k in keys}
    # kernel times from the serialised step (each pass with the GPU to itself)
    alone = {k: float(M["serial"][k]) for k in keys} if M.get("serial") else mean
    top = max(alone, key=alone.get)
    st = M["stats"]
    # the mixed form applies to iprec <= 1; above, both forms run FP64
    if iprec > 1:
        form, tensor_m2l = "fp64", False
    cuda = "fp32" if form == "mixed" else "fp64"
    # the FP64 rotate-shift-rotate M2L (orders <= 28) runs its products on the FP64 tensor cores (DMMA)
    dmma = cuda == "fp64" and M.get("tuning", {}).get("form") == "fp64-rotation" and st.get("nterms", 99) <= 28
    per = {}
    p2p_flops = st["p2p_pairs"] * P2P_FLOPS_PER_PAIR
    m2l_fl = sum(cnt * m2l_flops(pt) for pt, cnt in st["m2l_pt_hist"].items())
    for name, flops, bound in (("p2p", p2p_flops, cuda), ("m2l", m2l_fl, "tf32" if tensor_m2l else cuda)):
        ach = flops / (alone[name] * 1e-3) / 1e12
        label = ("tensor" if bound == "tf32" else
                 "fp64 tensor cores (DMMA)" if (name == "m2l" and dmma) else bound + " CUDA cores")
        per[name] = {"bound": label, "achieved": round(ach, 3),
                     "peak": round(peaks[bound], 2), "unit": "TFLOP/s", "frac": round(ach / peaks[bound], 4),
                     "peak_source": PEAK_SOURCE[bound] + ", measured in this run", "flops_per_launch": float(flops),
                     "ms": round(alone[name], 3)}
    per["p2p"]["traffic"] = None if P2P_DRAM_BYTES_PER_POINT is None else P2P_DRAM_BYTES_PER_POINT * M["points"]
    out = dict(per.get(top, {"bound": None, "achieved": None, "peak": None, "unit": None, "frac": None}))
    out.setdefault("traffic", None)
    out.update(kernel=top, pass_ms_mean={k: round(v, 3) for k, v in mean.items()},
               pass_ms_serial={k: round(v, 3) for k, v in alone.items()}, passes=per,
               note="pass_ms_mean: the timed steps, near field overlapped with the far field (pass times then "
                    "overlap); pass_ms_serial and the fractions: one extra step with the passes serialised")
    return out


def m2l_flops(pt):
    """Flops of one rotate-shift-rotate M2L at truncation pt, as the reference's scheme counts them:
    two rotations 2*[4*sum (2n+1)^2], the z-shift 4*sum_n sum_|m|<=n (pt-|m|+1), phases 12(pt+1)^2."""
    rot = 2 * 4 * sum((2 * n + 1) ** 2 for n in range(pt + 1))
    z = 4 * sum(pt - abs(mm) + 1 for n in range(pt + 1) for mm in range(-n, n + 1))
    return rot + z + 12 * (pt + 1) ** 2


def run_reference(args):
    """CPU restatement of the reference (oracle/, OpenMP over all host cores): every step is one
    lfmm3dparttarg call on the whole workload (the same N, M, distribution and seed as the GPU
    arm's), so both arms report the same config."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return None
    n = args.cpu_sample or args.n
    for _ in range(args.warmup):
        cpu_fmm_sample(n, args.iprec)
    times = []
    for _ in range(args.steps):
        dt, pts = cpu_fmm_sample(n, args.iprec)
        times.append(dt)
    v = 2 * n * len(times) / sum(times)
    cores = int(os.environ["OMP_NUM_THREADS"])
    helm = None
    if args.helm_n > 0 and args.helm_cpu_sample > 0:
        dt = cpu_helm_sample(args.helm_cpu_sample)
        helm = {"workload": "helmholtz_hfmm3dpartself_sphere_zk_8pi_iprec2", "value": args.helm_cpu_sample / dt,
                "unit": UNIT, "sample": "%d sources, one call (%.1f s)" % (args.helm_cpu_sample, dt)}
    sample = "N=M=%d uniform cube, charges+dipoles, iprec=%d, one lfmm3dparttarg restatement call per step" % (
        n, args.iprec)
    config = config_of(args, ws)
    if n != args.n:
        config["cpu_steps_n"] = n
    return {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "p50_ms": 1e3 * float(np.percentile(times, 50)), "p99_ms": 1e3 * float(np.percentile(times, 99)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config, "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores,
                                                             "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "helmholtz": helm}


def config_of(args, ws):
    return {"workload": "laplace_lfmm3dparttarg_cube_%dM_src_%dM_targ" % (args.n // 10 ** 6, args.n // 10 ** 6),
            "n_sources": args.n, "n_targets": args.n, "iprec": args.iprec, "charges": True, "dipoles": True,
            "outputs": "pot+fld at sources and targets", "forms": "mixed (headline) and fp64",
            "parallelism": "replicas x%d" % ws,
            "l2_policy": "inputs larger than L2 (%.0f MB per step of inputs vs 126 MB L2)" % (args.n * 104 / 1e6)}


def run_autotune(args):
    """Tune every Laplace workload of this bench (as plans on the same geometry and flags, so the
    signatures equal those of the measured calls) and write the knobs to the JSON cache."""
    import torch
    import fmmlib3d_b200 as F
    from fmmlib3d_b200 import autotune as A
    torch.cuda.set_device(dist_env()[2])
    dev = torch.device("cuda", torch.cuda.current_device())
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    e = lambda k, c: torch.empty((k, c), dtype=torch.float64, device=dev)
    path = os.path.abspath(args.autotune)
    F.set_tuning_cache(path)
    F.set_tensor_m2l(args.tensor_m2l)
    out = {}

    def one(name, precision, iprec, src, ins, outs, **kw):
        F.set_precision(precision)
        plan = F.LaplacePlan(iprec, src, **kw)
        r = A.tune(plan, *ins, *outs, cache_path=path, log=lambda s: print(name, s, file=sys.stderr, flush=True))
        out[name] = {"form": r["form"], "knobs": r["knobs"], "ms": round(r["ms"], 3),
                     "start_ms": round(r["auto_ms"], 3), "trials": len(r["trials"]), "signature": r["signature"]}
        plan.close()
        F.set_precision(0)

    n = m = args.n
    src, q, dq, dv, trg = make_inputs(n, m, 2)
    d = [g(a) for a in (src, q, dq, dv, trg)]
    outs = (e(n, 2), e(n, 6), e(m, 2), e(m, 6))
    flags = dict(ifcharge=1, ifdipole=1, ifpot=1, iffld=1, target=d[4], ifpottarg=1, iffldtarg=1)
    one("cube_mixed", 1, 1, d[0], d[1:4], outs, **flags)
    one("cube_fp64", 0, 1, d[0], d[1:4], outs, **flags)
    if args.n == 2_000_000:
        one("cube_iprec2_fp64", 0, 2, d[0], d[1:4], outs, **flags)
    del d, outs
    for ns in (100_000, 10_000):
        s_src, s_q = sphere_inputs(ns)
        one("sphere_%dk_fp64" % (ns // 1000), 0, 1, g(s_src), (g(s_q), None, None), (e(ns, 2), e(ns, 6)),
            ifcharge=1, ifdipole=0, ifpot=1, iffld=1)
    if args.batch_instances > 0:
        b_src, b_q, off = batched_inputs(args.batch_instances)
        nb = int(off[-1])
        one("batched_mixed", 1, 1, g(b_src), (g(b_q), None, None), (e(nb, 2), e(nb, 6)),
            ifcharge=1, ifdipole=0, ifpot=1, iffld=1, src_offsets=off)
    return {"autotune": path, "device": torch.cuda.get_device_name(), "workloads": out}


def main(argv=None):
    args = parse_args(argv)
    ws, rank, _ = dist_env()
    os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
    if args.autotune:
        if rank == 0:
            print(json.dumps(run_autotune(args)), flush=True)
        return 0
    if args.impl == "reference":
        line = run_reference(args)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    if args.workload == "helmholtz":
        import torch
        import fmmlib3d_b200 as F
        torch.cuda.set_device(dist_env()[2])
        R = dict(torch=torch, F=F, rank=rank, ws=1, dist=None)
        out = run_helm(args, R)
        line = {"metric": "Helmholtz FMM pts/s (sphere, zk=8pi, iprec=2)", "value": out["value"], "unit": UNIT,
                "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "helmholtz": out}
        if not args.no_cpu and args.helm_cpu_sample >= args.helm_n:
            dt, line["parity"] = oracle_helm_parity(R.pop("helm_samples"))
        print(json.dumps(line), flush=True)
        return 0
    if args.workload == "triangles":
        import torch
        import fmmlib3d_b200 as F
        torch.cuda.set_device(dist_env()[2])
        R = dict(torch=torch, F=F, rank=rank, ws=1, dist=None)
        out = run_triangles(args, R, k=args.tri_level)
        line = {"metric": "triangle FMM triangles/s (icosphere, iprec=1)", "value": out["value"], "unit": UNIT,
                "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "laplace_triangles": out}
        if args.htri_level > 0:
            line["helmholtz_triangles"] = run_triangles(args, R, k=args.htri_level, zk=complex(4 * math.pi))
        for job in R.get("cpu_jobs", []):
            job(line)
        print(json.dumps(line), flush=True)
        return 0
    if args.workload == "batched":
        import torch
        import fmmlib3d_b200 as F
        torch.cuda.set_device(dist_env()[2])
        R = dict(torch=torch, F=F, rank=rank, ws=1, dist=None)
        out = run_batched(args, R)
        plans = run_plans(args, R, R.pop("batch_arrays", None))
        print(json.dumps({"metric": "batched Laplace FMM pts/s", "value": out["value"], "unit": UNIT,
                          "n_gpus": 1, "steps": out["steps"], "warmup": args.warmup, "batched": out,
                          "plans": plans}), flush=True)
        return 0
    if args.workload == "laplace":
        args.helm_n = 0
        args.batch_instances = 0
        args.serve_requests = 0
    R = run_b200(args)
    R["F"].set_precision(1)
    e2e = None if args.no_e2e else run_e2e(args, R)
    n, m = R["n"], R["m"]

    def summary(M):
        return {"value": ws * (n + m) * args.steps / (M["total_ms"] * 1e-3), "ms_per_step": M["total_ms"] / args.steps,
                "p50_ms": float(np.percentile(M["step_ms"], 50)), "p99_ms": float(np.percentile(M["step_ms"], 99)),
                "errors": {k: float("%.3e" % v) for k, v in M["errs"].items()}, "tuning": M["tuning"]}

    H = R["forms"]["mixed"]
    head = summary(H)
    line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "p50_ms": head["p50_ms"],
            "p99_ms": head["p99_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64 mixed (P2P, M2L in f32; tree, recurrences, other passes f64)",
            "data": "synthetic (seeded uniform cube; charges, dipoles)", "config": config_of(args, ws),
            "errors": head["errors"], "gpu_launches": int(sum(H["launches"])), "clocks": H["clocks"], "e2e": e2e,
            "roofline": roofline_of(H, R["peaks"], "mixed", tensor_m2l=args.tensor_m2l > 0, iprec=args.iprec),
            "forms": {"mixed": head, "fp64": dict(summary(R["forms"]["fp64"]),
                                                  roofline=roofline_of(R["forms"]["fp64"], R["peaks"], "fp64",
                                                                       iprec=args.iprec),
                                                  gpu_launches=int(sum(R["forms"]["fp64"]["launches"])))},
            "stats": {k: v for k, v in H["stats"].items() if k != "m2l_pt_hist"}}
    line["forms"]["mixed_over_fp64"] = round(head["value"] / line["forms"]["fp64"]["value"], 3)
    # CPU work (the oracle on each workload's own inputs: parity at the sampled points, and its
    # time as the CPU baseline) runs after every GPU workload, so that it does not share the host
    # with them
    cpu_jobs = R.setdefault("cpu_jobs", [])
    if rank == 0 and ws == 1 and not args.no_cpu:
        def cube_job(line):
            src, q, dq, dv, trg = R["arrays"]
            Sm, Sf = R["forms"]["mixed"]["samples"], R["forms"]["fp64"]["samples"]
            keys = ("pot", "fld", "pottarg", "fldtarg")
            gpu_forms = {"fp64": {k: Sf[k] for k in keys}, "mixed": {k: Sm[k] for k in keys}}
            dt, rep = oracle_laplace_parity(args.iprec, src, q, dq, dv, trg, Sf["si"], Sf["ti"], gpu_forms,
                                            {k: Sf["direct_" + k] for k in keys})
            rep.update(points="%d seeded sources (self excluded) and %d seeded targets" % (len(Sf["si"]),
                                                                                           len(Sf["ti"])),
                       inputs="the headline workload's own inputs", oracle_call_s=round(dt, 2))
            line.setdefault("parity", {})["laplace_cube"] = rep
            line["cpu_baseline"] = {"value": (n + m) / dt, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
                                    "kind": "port",
                                    "sample": "the whole workload (N=M=%d uniform cube, charges+dipoles, iprec=%d), "
                                              "one lfmm3dparttarg restatement call (%.1f s)" % (n, args.iprec, dt)}

        cpu_jobs.append(cube_job)
    line["laplace_sphere"] = run_laplace_sphere(args, R)
    line["laplace_triangles"] = run_triangles(args, R, k=args.tri_level)
    if args.htri_level > 0:
        line["helmholtz_triangles"] = run_triangles(args, R, k=args.htri_level, zk=complex(4 * math.pi))
    if args.n == 2_000_000 and args.iprec == 1:
        line["laplace_iprec2"] = run_iprec2(args, R)
    if args.batch_instances > 0:
        line["batched"] = run_batched(args, R)
    line["plans"] = run_plans(args, R, R.pop("batch_arrays", None))
    if args.serve_requests > 0 and ws == 1:
        line["serving"] = run_serving(args)
        line["serving_mixed"] = run_serving(args, precision=1)
        line["serving_repeated"] = run_serving(args, geometries=8, rates="60,inf")
    if args.helm_n > 0:
        H2 = run_helm(args, R)
        if rank == 0 and ws == 1 and not args.no_cpu and args.helm_cpu_sample > 0:
            HS = R.pop("helm_samples")

            def helm_job(line):
                if args.helm_cpu_sample >= args.helm_n:
                    dt, rep = oracle_helm_parity(HS)
                    line.setdefault("parity", {})["helmholtz_sphere"] = rep
                    what = "the whole workload (the same inputs), one call (%.1f s)" % dt
                    nc = args.helm_n
                else:
                    dt = cpu_helm_sample(args.helm_cpu_sample)
                    what = "%d sources, same distribution, one call (%.1f s)" % (args.helm_cpu_sample, dt)
                    nc = args.helm_cpu_sample
                H2["cpu_baseline"] = {"value": nc / dt, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
                                      "kind": "port", "sample": what}

            cpu_jobs.append(helm_job)
        line["helmholtz"] = H2
    for job in cpu_jobs:
        job(line)
    if R["dist"] is not None:
        R["dist"].barrier()
        R["dist"].destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
