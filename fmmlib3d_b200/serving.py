"""A serving loop for FMM requests on one GPU (continuous batching).

Requests (Laplace or Helmholtz particle FMMs of any size and iprec) arrive at
any time.  A scheduler keeps up to `slots` requests on the GPU at once: a
waiting request is admitted as soon as a slot is free and its projected HBM
footprint fits in what the running requests leave of the budget, so requests
that arrive while others run start without waiting for them to finish.  Each
slot is a host thread with its own CUDA stream (the library gives every host
thread its own stream), so the admitted requests' kernels, copies and
workspace allocations overlap on the device.  Every call is independent and
deterministic, so a request's result is the same alone and in the mix.

    server = FMMServer(slots=4)       # precision=1: mixed form for Laplace requests with iprec <= 1
    fut = server.submit(Request("helmholtz", source, charge, iprec=1, zk=5.0))
    pot, fld = fut.result().pot, fut.result().fld
    server.close()

Repeated geometries: a Laplace request that names a `geometry` key (requests
with the same key must carry the same sources) runs on a plan kept on the
device (LaplacePlan: tree, lists, sorted coordinates and workspace built once),
replaying its CUDA graph with the request's charges, so only the charges
cross PCIe and no tree is rebuilt.  Resident plans are held within
`plan_bytes` (least recently used evicted first) and count against the HBM
budget; a request on a resident plan is admitted for its transient buffers
alone, sized from the plan's built tree.  Each slot keeps its CUDA stream and
its pinned host buffers for the life of the server.

Latency of a request = completion time - submission time; `stats()` gives
p50/p99 latency and the points/s of the completed requests.
"""
import collections
import math
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    kernel: str                     # "laplace" or "helmholtz"
    source: np.ndarray              # (N, 3) float64
    charge: np.ndarray              # (N,) complex128
    iprec: int = 1
    zk: complex = 0.0
    tag: object = None
    precision: int = None           # 0 FP64, 1 mixed (Laplace, iprec <= 1); None: the server's
    geometry: object = None         # hashable key of a repeated source set (Laplace): served by a resident plan
    submitted: float = field(default=0.0, repr=False)


@dataclass
class Result:
    pot: np.ndarray
    fld: np.ndarray
    ier: int
    latency_s: float
    queue_s: float
    n: int
    tag: object = None


_NBOX = {-2: 40, -1: 50, 0: 80, 1: 160, 2: 400, 3: 800, 4: 1200, 5: 1400}


def projected_bytes(req):
    """Projected peak HBM footprint of one request (inputs, tree-ordered copies,
    outputs, tree, expansions and translation scratch), used for admission."""
    n = len(req.source)
    per_point = 24 + 16 + 64 + 24 + 16 + 64 + 64     # caller arrays, sorted copies, outputs, keys/sort
    nbox = _NBOX.get(req.iprec, 160)
    boxes = 2.5 * max(n / nbox, 1) * 8 / 7 + 64
    if req.kernel == "helmholtz":
        p = 12 + 4 * abs(complex(req.zk)) + 4 * max(req.iprec, 0)   # generous order estimate
        p = min(p, 60)
    else:
        p = {-2: 4, -1: 6, 0: 9, 1: 14, 2: 26, 3: 39}.get(req.iprec, 39)
    exps = boxes * 2 * (p + 1) ** 2 * 16
    return int(n * per_point + exps + boxes * 600 + (64 << 20))


def plan_bytes(info):
    """HBM held by a resident plan, from its built tree (LaplacePlan.info()): expansions and
    box arrays per box, sorted coordinates, charges and output workspace per point, and the
    server's charge / output buffers for the plan."""
    p, nb, n = info["nterms"], info["nboxes"], info["nsource"] + info["ntarget"]
    return int(nb * (2 * (p + 1) ** 2 * 16 + 600) + n * (24 + 16 + 64) + info["nsource"] * (24 + 16 + 64))


def transient_bytes(n):
    """Per-request device buffers of a request on a resident plan (charges in, pot / fld out)."""
    return int(n * (16 + 16 + 48))


class _PlanEntry:
    def __init__(self):
        self.lock = threading.Lock()   # one request at a time on a plan (its buffers, its graph)
        self.ready = False
        self.failed = False
        self.plan = None
        self.bytes = 0
        self.users = 0
        self.stream = None
        self.q = self.pot = self.fld = None


class FMMServer:
    def __init__(self, slots=4, hbm_budget_bytes=None, device=0, precision=None, plan_bytes=None):
        """precision: arithmetic form of Laplace requests that do not name one (0 FP64, 1 mixed
        for iprec <= 1; None: the process-wide setting).  plan_bytes: HBM for resident plans of
        repeated geometries (default a quarter of the budget; 0 disables plans)."""
        import torch
        import fmmlib3d_b200 as F
        self._torch, self._F = torch, F
        self.device = device
        self.precision = precision
        if hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget_bytes = int(0.8 * free)
        self.budget = hbm_budget_bytes
        self.plan_budget = self.budget // 4 if plan_bytes is None else int(plan_bytes)
        self._plans = collections.OrderedDict()   # (geometry, iprec, form) -> _PlanEntry, LRU order
        self._resident = 0
        self.plan_hits = 0
        self.plans_built = 0
        self.plans_evicted = 0
        self._cv = threading.Condition()
        self._wait = collections.deque()
        self._in_use = 0
        self._running = 0
        self.max_running = 0       # most requests seen on the GPU at once
        self._closed = False
        self._done = []
        self._tls = threading.local()
        self._workers = [threading.Thread(target=self._worker, daemon=True) for _ in range(slots)]
        for w in self._workers:
            w.start()

    def submit(self, req):
        fut = Future()
        req.submitted = time.perf_counter()
        with self._cv:
            if self._closed:
                raise RuntimeError("server closed")
            self._wait.append((req, fut))
            self._cv.notify_all()
        return fut

    def _form(self, req):
        return req.precision if req.precision is not None else self.precision

    def _plan_key(self, req):
        if req.geometry is None or req.kernel != "laplace" or self.plan_budget <= 0:
            return None
        return (req.geometry, req.iprec, self._form(req))

    def _need(self, req):
        key = self._plan_key(req)
        e = self._plans.get(key) if key is not None else None
        if e is not None and e.ready:
            return transient_bytes(len(req.source))   # the tree is built and resident
        return projected_bytes(req)

    def _evict(self, room):
        # least recently used plans not in use, until `room` more bytes fit
        for key in list(self._plans):
            if self._resident + room <= self.plan_budget:
                break
            e = self._plans[key]
            if e.users == 0 and e.ready:
                del self._plans[key]
                self._resident -= e.bytes
                self.plans_evicted += 1
                e.plan.close()

    def _next(self):
        # first waiting request whose footprint fits beside the running requests and the
        # resident plans (a request larger than the whole budget runs alone).  A request whose
        # geometry's plan is in use waits in the queue, not in a slot: one request at a time
        # runs on a plan, and the slot goes to the next request that can run.
        for i, (req, fut) in enumerate(self._wait):
            key = self._plan_key(req)
            e = self._plans.get(key) if key is not None else None
            if e is not None and e.users > 0:
                continue
            need = self._need(req)
            if self._in_use + self._resident + need <= self.budget or self._running == 0:
                del self._wait[i]
                if key is not None:
                    if e is None:
                        e = self._plans[key] = _PlanEntry()
                    self._plans.move_to_end(key)
                    e.users += 1
                return req, fut, need, e
        return None

    def _worker(self):
        torch = self._torch
        torch.cuda.set_device(self.device)
        # the slot's stream and pinned host buffers, kept for the life of the server
        self._tls.stream = torch.cuda.Stream(device=torch.device("cuda", self.device))
        self._tls.pinned = {}
        while True:
            with self._cv:
                item = None
                while not (self._closed and not self._wait):
                    item = self._next()
                    if item is not None:
                        break
                    self._cv.wait()
                if item is None:
                    return
                req, fut, need, entry = item
                self._in_use += need
                self._running += 1
                self.max_running = max(self.max_running, self._running)
            start = time.perf_counter()
            try:
                res = self._run(req, entry)
                res.queue_s = start - req.submitted
                res.latency_s = time.perf_counter() - req.submitted
                fut.set_result(res)
                with self._cv:
                    self._done.append(res)
            except Exception as exc:  # noqa: BLE001 -- reported through the future
                fut.set_exception(exc)
            finally:
                with self._cv:
                    self._in_use -= need
                    self._running -= 1
                    self._cv.notify_all()

    def _pinned(self, name, count):
        """This slot's pinned float64 host buffer `name`, at least `count` long (grown, never shrunk)."""
        buf = self._tls.pinned.get(name)
        if buf is None or buf.numel() < count:
            buf = self._torch.empty(max(count, 1 << 16), dtype=self._torch.float64, pin_memory=True)
            self._tls.pinned[name] = buf
        return buf[:count]

    def _stage_in(self, name, arr, dev):
        """Host array -> this slot's pinned buffer -> device (on the current stream).  The
        pinned buffer is reused by the slot's next request only after this one has synchronised."""
        a = np.ascontiguousarray(arr).view(np.float64).reshape(-1)
        h = self._pinned(name, a.size)
        h.numpy()[:] = a
        return h.to(dev, non_blocking=True)

    def _result(self, req, pot, fld, ier, stream):
        n = len(req.source)
        hp, hf = self._pinned("pot", 2 * n), self._pinned("fld", 6 * n)
        with self._torch.cuda.stream(stream):
            hp.copy_(pot.reshape(-1), non_blocking=True)
            hf.copy_(fld.reshape(-1), non_blocking=True)
        stream.synchronize()
        return Result(pot=hp.numpy().view(np.complex128).reshape(n).copy(),
                      fld=hf.numpy().view(np.complex128).reshape(n, 3).copy(), ier=ier, latency_s=0.0,
                      queue_s=0.0, n=n, tag=req.tag)

    def _run_plan(self, req, key, e):
        """A request on the resident plan `e` of its geometry (built by the first request that
        names it; admission counted this request among the plan's users).  Returns None when no
        plan can be built (the request then runs as a plain call)."""
        torch, F = self._torch, self._F
        n = len(req.source)
        dev = torch.device("cuda", self.device)
        try:
            with e.lock:
                if e.failed:
                    return None
                if not e.ready:
                    e.stream = torch.cuda.Stream(device=dev)
                    with torch.cuda.stream(e.stream):
                        src = self._stage_in("src", req.source, dev).reshape(n, 3)
                        form = self._form(req)
                        F.set_precision_thread(-1 if form is None else form)
                        try:
                            e.plan = F.LaplacePlan(req.iprec, src, 1, 0, 1, 1, stream=e.stream.cuda_stream)
                        except RuntimeError:
                            e.failed = True
                            return None
                        finally:
                            F.set_precision_thread(-1)
                        e.q = torch.empty((n, 2), dtype=torch.float64, device=dev)
                        e.pot = torch.empty((n, 2), dtype=torch.float64, device=dev)
                        e.fld = torch.empty((n, 6), dtype=torch.float64, device=dev)
                    e.stream.synchronize()
                    e.bytes = plan_bytes(e.plan.info())
                    with self._cv:
                        self._evict(e.bytes)
                        self._resident += e.bytes
                        self.plans_built += 1
                        e.ready = True
                else:
                    with self._cv:
                        self.plan_hits += 1
                with torch.cuda.stream(e.stream):
                    e.q.copy_(self._stage_in("q", np.asarray(req.charge, np.complex128), dev).reshape(n, 2),
                              non_blocking=True)
                    ier = e.plan.execute(charge=e.q, pot=e.pot, fld=e.fld, use_graph=True,
                                         stream=e.stream.cuda_stream)
                return self._result(req, e.pot, e.fld, ier, e.stream)
        finally:
            with self._cv:
                e.users -= 1
                if e.failed and e.users == 0 and self._plans.get(key) is e:
                    del self._plans[key]
                if self._resident > self.plan_budget:
                    self._evict(0)   # plans that were in use when the budget was passed

    def _run(self, req, entry=None):
        torch, F = self._torch, self._F
        n = len(req.source)
        dev = torch.device("cuda", self.device)
        if entry is not None:
            res = self._run_plan(req, self._plan_key(req), entry)
            if res is not None:
                return res
        stream = self._tls.stream
        with torch.cuda.stream(stream):
            src = self._stage_in("src", req.source, dev).reshape(n, 3)
            chg = self._stage_in("q", np.asarray(req.charge, np.complex128), dev).reshape(n, 2)
            pot = torch.empty((n, 2), dtype=torch.float64, device=dev)
            fld = torch.empty((n, 6), dtype=torch.float64, device=dev)
            if req.kernel == "helmholtz":
                ier = F.hfmm3dparttarg_device(req.iprec, req.zk, src, chg, None, None, pot, fld,
                                              stream=stream.cuda_stream)
            else:
                form = req.precision if req.precision is not None else self.precision
                F.set_precision_thread(-1 if form is None else form)
                try:
                    ier = F.lfmm3dparttarg_device(req.iprec, src, chg, None, None, pot, fld,
                                                  stream=stream.cuda_stream)
                finally:
                    F.set_precision_thread(-1)
        return self._result(req, pot, fld, ier, stream)

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for w in self._workers:
            w.join()
        with self._cv:
            for e in self._plans.values():
                if e.plan is not None:
                    e.plan.close()
            self._plans.clear()
            self._resident = 0

    def stats(self):
        with self._cv:
            done = list(self._done)
        if not done:
            return {}
        lat = np.array([r.latency_s for r in done])
        return {"requests": len(done), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
                "p99_ms": 1e3 * float(np.percentile(lat, 99)), "points": int(sum(r.n for r in done)),
                "plan_hits": self.plan_hits, "plans_built": self.plans_built, "plans_evicted": self.plans_evicted,
                "resident_plan_bytes": self._resident}


def _points(rng, n):
    g = rng.integers(3)
    if g == 0:
        return rng.random((n, 3))
    if g == 1:
        pts = []
        while sum(len(p) for p in pts) < n:
            u = rng.random(n)
            r = 0.1 / np.sqrt(np.maximum(u ** (-2 / 3) - 1, 1e-300))
            v = rng.normal(size=(n, 3))
            v *= (r / np.linalg.norm(v, axis=1))[:, None]
            pts.append(v[r < 1])
        return np.concatenate(pts)[:n]
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None] * rng.uniform(0.2, 1, 3)


def make_request_stream(count, seed=0, geometries=0):
    """Synthetic requests of the serving workload: 70% Laplace, 30% Helmholtz with zk
    uniform in [1, 20]; N log-uniform in [1e3, 1e6]; iprec uniform in {0, 1, 2};
    geometry uniform among a unit cube, a Plummer sphere (scale 0.1, radius cut 1) and
    an ellipsoid surface with semi-axes uniform in [0.2, 1]; charges in [-1, 1]^2.
    geometries > 0: every Laplace request takes its sources and iprec from a pool of that
    many source sets (drawn the same way) and names it as its `geometry`, with charges of
    its own, as repeated solves on fixed geometries do."""
    rng = np.random.default_rng(seed)
    pool = []
    if geometries:
        prng = np.random.default_rng(seed + 1000)
        for _ in range(geometries):
            n = int(10 ** prng.uniform(3, 6))
            pool.append((_points(prng, n), int(prng.integers(0, 3))))
    out = []
    for i in range(count):
        n = int(10 ** rng.uniform(3, 6))
        src = _points(rng, n)
        q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        helm = rng.random() < 0.3
        iprec = int(rng.integers(0, 3))
        zk = float(rng.uniform(1, 20)) if helm else 0.0
        if pool and not helm:
            g = int(rng.integers(len(pool)))
            src, iprec = pool[g]
            q = rng.uniform(-1, 1, len(src)) + 1j * rng.uniform(-1, 1, len(src))
            out.append(Request("laplace", src, q, iprec=iprec, tag=i, geometry=g))
            continue
        out.append(Request("helmholtz" if helm else "laplace", src, q, iprec=iprec, zk=zk, tag=i))
    return out


def run_stream(server, requests, rate_hz, seed=1):
    """Submit `requests` with Poisson arrivals at rate_hz; wait for all; return stats."""
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    futs = []
    t_next = t0
    for req in requests:
        t_next += rng.exponential(1.0 / rate_hz) if math.isfinite(rate_hz) else 0.0
        delay = t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        futs.append(server.submit(req))
    res = [f.result() for f in futs]
    wall = time.perf_counter() - t0
    lat = np.array([r.latency_s for r in res])
    pts = sum(r.n for r in res)
    return {"rate_hz": rate_hz, "requests": len(res), "points": int(pts), "wall_s": wall,
            "points_per_s": pts / wall, "p50_ms": 1e3 * float(np.percentile(lat, 50)),
            "p99_ms": 1e3 * float(np.percentile(lat, 99)), "max_ier": int(max(r.ier for r in res))}, res
