"""World-size-2 gloo test of the multi-GPU exchange (reproblas_b200.distributed) on the
CPU: each rank reduces its shard (with the oracle restatement standing in for the GPU
kernel), the states are all-gathered and merged with the binned addition, and both ranks
must hold the bits of the single-process reduction of the whole vector."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_merge(fold, count, gathered, out, reverse=False):
    from _ffi import port, ptr
    P = port()
    g = gathered.numpy()
    o = out.numpy()
    order = range(count - 1, -1, -1) if reverse else range(count)
    for i in order:
        st = np.ascontiguousarray(g[i * 2 * fold:(i + 1) * 2 * fold])
        P.dbdbadd(fold, ptr(st), ptr(o))


def _worker(rank, world, port, n, fold, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from _ffi import port as oport, ptr, binned_zeros
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "rbdist", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                               "reproblas_b200", "distributed.py"))
    rbdist = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rbdist)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(42)
        x = np.exp2(rng.uniform(-200, 200, n)) * rng.choice([-1.0, 1.0], n)
        y = rng.standard_normal(n)
        start, length = rbdist.shard(n, rank, world)
        st = binned_zeros(fold)
        oport().dbddot(fold, length, ptr(x[start:]), 1, ptr(y[start:]), 1, ptr(st))
        merged = rbdist.allgather_merge(torch.from_numpy(st), fold, merge=_oracle_merge)
        rev = rbdist.allgather_merge(torch.from_numpy(st), fold,
                                     merge=lambda f, c, g, o: _oracle_merge(f, c, g, o, True))
        q.put((rank, merged.numpy().tobytes(), rev.numpy().tobytes()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_allgather_merge_matches_single_process(world):
    from _ffi import port, ptr, binned_zeros
    n, fold = 100003, 3
    rng = np.random.default_rng(42)
    x = np.exp2(rng.uniform(-200, 200, n)) * rng.choice([-1.0, 1.0], n)
    y = rng.standard_normal(n)
    want = binned_zeros(fold)
    port().dbddot(fold, n, ptr(x), 1, ptr(y), 1, ptr(want))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, p, n, fold, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, merged, rev in got:
        assert merged == want.tobytes(), rank
        assert rev == want.tobytes(), rank


def test_shard_covers_range():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "rbdist", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                               "reproblas_b200", "distributed.py"))
    rbdist = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rbdist)
    for n in (0, 1, 7, 1000, 2 ** 28 + 5):
        for world in (1, 2, 3, 8):
            parts = [rbdist.shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0
            for (s0, l0), (s1, _) in zip(parts, parts[1:]):
                assert s0 + l0 == s1
            assert sum(l for _, l in parts) == n
