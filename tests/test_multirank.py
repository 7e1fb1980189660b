"""The replica path of bench.py on two CPU ranks (gloo, 127.0.0.1).

An FMM call does not shard, so `bench.py --gpus N` runs N independent replicas:
each rank draws its own seeded inputs, the ranks meet at a barrier around the
timed region, and the reported time is the maximum over ranks.  This test runs
that logic with two gloo ranks: distinct per-rank inputs, the max reduction,
and the Laplace and Helmholtz CPU oracle calls each replica would check against.
"""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        src, q, dq, dv, trg = bench.make_inputs(1000, 500, 2 + rank)
        hs, hq = bench.helm_inputs(800, seed=3 + rank)
        dist.barrier()
        t = bench.reduce_max(dist, 10.0 * (rank + 1), "cpu")
        import oracle
        ier_l = oracle.lfmm3dparttarg(1, src, q[:, 0] + 1j * q[:, 1], None, None, trg)[0]
        ier_h = oracle.hfmm3dparttarg(1, bench.HELM_ZK, hs, hq[:, 0] + 1j * hq[:, 1])[0]
        dist.barrier()
        out.put((rank, float(src[0, 0]), float(hs[0, 0]), t, ier_l, ier_h))
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_max_with_distinct_inputs():
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import oracle
    oracle.lib()  # build before spawning
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, a0, h0, t0, l0, k0), (r1, a1, h1, t1, l1, k1) = res
    assert (r0, r1) == (0, 1)
    assert a0 != a1 and h0 != h1          # each replica has its own seeded inputs
    assert t0 == t1 == 20.0               # the reported time is the max over ranks
    assert l0 == l1 == k0 == k1 == 0
