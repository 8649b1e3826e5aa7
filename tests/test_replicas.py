"""The N>1 path of bench.py: one process per GPU running independent replicas
("replicas only": no field data crosses ranks).  Exercised here with the gloo
backend, world size 2, on CPU; each rank integrates its own replica with the
oracle standing in for the GPU library."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        from compchan3dmpi_b200 import replicas as R
        from chan_cases import make_case
        from oracle import oracle as O
        r = R.init("gloo", timeout_s=60)
        p, x3, jac, inv, var = make_case(nP=(12, 10, 11), quantize=False, istat=2)
        o = O.Oracle(p.with_(device=r.local_rank), x3, jac, inv, threads=1)
        o.upload(var)
        o.step(3)
        checksum = float(np.sum(o.download()))
        R.barrier(r)
        fake_ms = 10.0 + rank          # device time of this rank's timed region
        mx = R.max_over_ranks(r, fake_ms)
        units = R.sum_over_ranks(r, float(p.n_interior * p.stages * 3))
        R.barrier(r)
        q.put((rank, r.world, mx, units, checksum, None))
        R.finalize(r)
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, None, None, None, None, repr(e)))


def test_two_rank_replicas_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=240) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
    res.sort()
    for rank, world, mx, units, checksum, err in res:
        assert err is None, err
        assert world == 2
        assert mx == 11.0                      # max over ranks of the device time
    assert res[0][3] == res[1][3] and res[0][3] > 0   # whole-job units = sum over ranks
    assert res[0][4] == res[1][4]              # independent replicas integrate identically


def test_single_rank_is_identity():
    from compchan3dmpi_b200 import replicas as R
    r = R.Ranks()
    assert R.max_over_ranks(r, 3.5) == 3.5 and R.sum_over_ranks(r, 2.0) == 2.0
    R.barrier(r)
    R.finalize(r)
