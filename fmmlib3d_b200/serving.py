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


class FMMServer:
    def __init__(self, slots=4, hbm_budget_bytes=None, device=0, precision=None):
        """precision: arithmetic form of Laplace requests that do not name one (0 FP64, 1 mixed
        for iprec <= 1; None: the process-wide setting)."""
        import torch
        import fmmlib3d_b200 as F
        self._torch, self._F = torch, F
        self.device = device
        self.precision = precision
        if hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget_bytes = int(0.8 * free)
        self.budget = hbm_budget_bytes
        self._cv = threading.Condition()
        self._wait = collections.deque()
        self._in_use = 0
        self._running = 0
        self.max_running = 0       # most requests seen on the GPU at once
        self._closed = False
        self._done = []
        self._workers = [threading.Thread(target=self._worker, daemon=True) for _ in range(slots)]
        for w in self._workers:
            w.start()

    def submit(self, req):
        fut = Future()
        req.submitted = time.perf_counter()
        with self._cv:
            if self._closed:
                raise RuntimeError("server closed")
            self._wait.append((req, fut, projected_bytes(req)))
            self._cv.notify_all()
        return fut

    def _next(self):
        # first waiting request whose footprint fits (a request larger than the
        # whole budget runs alone)
        for i, (req, fut, need) in enumerate(self._wait):
            if self._in_use + need <= self.budget or self._running == 0:
                del self._wait[i]
                return req, fut, need
        return None

    def _worker(self):
        torch = self._torch
        torch.cuda.set_device(self.device)
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
                req, fut, need = item
                self._in_use += need
                self._running += 1
                self.max_running = max(self.max_running, self._running)
            start = time.perf_counter()
            try:
                res = self._run(req)
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

    def _run(self, req):
        torch, F = self._torch, self._F
        n = len(req.source)
        dev = torch.device("cuda", self.device)
        stream = torch.cuda.Stream(device=dev)
        with torch.cuda.stream(stream):
            src = torch.from_numpy(np.ascontiguousarray(req.source, np.float64)).pin_memory().to(dev, non_blocking=True)
            q = np.ascontiguousarray(req.charge, np.complex128).view(np.float64).reshape(n, 2)
            chg = torch.from_numpy(q).pin_memory().to(dev, non_blocking=True)
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
            hp = torch.empty((n, 2), dtype=torch.float64, pin_memory=True)
            hf = torch.empty((n, 6), dtype=torch.float64, pin_memory=True)
            hp.copy_(pot, non_blocking=True)
            hf.copy_(fld, non_blocking=True)
        stream.synchronize()
        return Result(pot=hp.numpy().view(np.complex128).reshape(n).copy(),
                      fld=hf.numpy().view(np.complex128).reshape(n, 3).copy(), ier=ier, latency_s=0.0,
                      queue_s=0.0, n=n, tag=req.tag)

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for w in self._workers:
            w.join()

    def stats(self):
        with self._cv:
            done = list(self._done)
        if not done:
            return {}
        lat = np.array([r.latency_s for r in done])
        return {"requests": len(done), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
                "p99_ms": 1e3 * float(np.percentile(lat, 99)), "points": int(sum(r.n for r in done))}


def make_request_stream(count, seed=0):
    """Synthetic requests of the serving workload: 70% Laplace, 30% Helmholtz with zk
    uniform in [1, 20]; N log-uniform in [1e3, 1e6]; iprec uniform in {0, 1, 2};
    geometry uniform among a unit cube, a Plummer sphere (scale 0.1, radius cut 1) and
    an ellipsoid surface with semi-axes uniform in [0.2, 1]; charges in [-1, 1]^2."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(10 ** rng.uniform(3, 6))
        g = rng.integers(3)
        if g == 0:
            src = rng.random((n, 3))
        elif g == 1:
            pts = []
            while sum(len(p) for p in pts) < n:
                u = rng.random(n)
                r = 0.1 / np.sqrt(np.maximum(u ** (-2 / 3) - 1, 1e-300))
                v = rng.normal(size=(n, 3))
                v *= (r / np.linalg.norm(v, axis=1))[:, None]
                pts.append(v[r < 1])
            src = np.concatenate(pts)[:n]
        else:
            v = rng.normal(size=(n, 3))
            src = v / np.linalg.norm(v, axis=1)[:, None] * rng.uniform(0.2, 1, 3)
        q = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        helm = rng.random() < 0.3
        out.append(Request("helmholtz" if helm else "laplace", src, q, iprec=int(rng.integers(0, 3)),
                           zk=float(rng.uniform(1, 20)) if helm else 0.0, tag=i))
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
