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


def _load_rbdist():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "rbdist", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                               "reproblas_b200", "distributed.py"))
    rbdist = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rbdist)
    return rbdist


def _oracle_merge_kind(kind, reverse):
    """CPU stand-in for rb_<kind>_states: the oracle's merge of each record, in order or
    reversed."""
    def merge(fold, count, gathered, out):
        from _ffi import port, ptr
        P = port()
        g, o = gathered.numpy(), out.numpy()
        n = len(o)
        order = range(count - 1, -1, -1) if reverse else range(count)
        for i in order:
            rec = np.ascontiguousarray(g[i * n:(i + 1) * n])
            if kind in ("z", "c", "s"):
                getattr(P, {"z": "zbzbadd", "c": "cbcbadd", "s": "sbsbadd"}[kind])(fold, ptr(rec), ptr(o))
            elif kind in ("dsq", "ssq"):
                body = o[1:].copy()
                add = P.dbdbaddsq if kind == "dsq" else P.sbsbaddsq
                o[0] = add(fold, float(rec[0]), ptr(np.ascontiguousarray(rec[1:])), float(o[0]), ptr(body))
                o[1:] = body
    return merge


def _kind_worker(rank, world, port, n, fold, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from _ffi import port as oport, ptr, binned_zeros
    from _data import gen, gen_complex
    rbdist = _load_rbdist()
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = oport()
        start, length = rbdist.shard(n, rank, world)
        out = {}
        # complex dot: double_complex_binned records
        x, y = gen_complex("loguniform", n, 5), gen_complex("normal", n, 6)
        st = binned_zeros(fold, "z")
        P.zbzdotc(fold, length, ptr(x[start:]), 1, ptr(y[start:]), 1, ptr(st))
        for rev in (False, True):
            m = rbdist.allgather_merge(torch.from_numpy(st), fold, kind="z",
                                       merge=_oracle_merge_kind("z", rev))
            out[("z", rev)] = m.numpy().tobytes()
        # 2-norm: [scale, double_binned] records
        v = gen("loguniform", n, 7)
        rec = np.zeros(1 + 2 * fold)
        body = binned_zeros(fold)
        rec[0] = P.dbdssq(fold, length, ptr(v[start:]), 1, 0.0, ptr(body))
        rec[1:] = body
        for rev in (False, True):
            m = rbdist.allgather_merge(torch.from_numpy(rec), fold, kind="dsq",
                                       merge=_oracle_merge_kind("dsq", rev))
            out[("dsq", rev)] = m.numpy().tobytes()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_allgather_merge_complex_and_scaled_states(world):
    """Complex dot states and the scaled sum-of-squares records of dnrm2 through the same
    exchange: every rank holds the single-process bits, for both merge orders."""
    from _ffi import port, ptr, binned_zeros
    from _data import gen, gen_complex
    n, fold = 50021, 3
    P = port()
    x, y = gen_complex("loguniform", n, 5), gen_complex("normal", n, 6)
    want_z = binned_zeros(fold, "z")
    P.zbzdotc(fold, n, ptr(x), 1, ptr(y), 1, ptr(want_z))
    v = gen("loguniform", n, 7)
    body = binned_zeros(fold)
    want_dsq = np.zeros(1 + 2 * fold)
    want_dsq[0] = P.dbdssq(fold, n, ptr(v), 1, 0.0, ptr(body))
    want_dsq[1:] = body
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = _free_port()
    procs = [ctx.Process(target=_kind_worker, args=(r, world, p, n, fold, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, out in got:
        for rev in (False, True):
            assert out[("z", rev)] == want_z.tobytes(), (rank, rev)
            assert out[("dsq", rev)] == want_dsq.tobytes(), (rank, rev)


def test_record_lengths_and_kind_check():
    rbdist = _load_rbdist()
    assert rbdist.record_len("d", 3) == 6 and rbdist.record_len("z", 3) == 12
    assert rbdist.record_len("dsq", 3) == 7 and rbdist.record_len("ssq", 2) == 5
    with pytest.raises(ValueError):
        rbdist.allgather_merge(torch.zeros(5), 3, kind="d")
    with pytest.raises(ValueError):
        rbdist.allgather_merge(torch.zeros(6), 3, kind="q")


def _fp32_worker(rank, world, port, n, fold, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from _ffi import port as oport, ptr, binned_zeros
    from _data import gen, gen_complex
    rbdist = _load_rbdist()
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = oport()
        start, length = rbdist.shard(n, rank, world)
        out = {}
        xs = gen("normal", n, 11, np.float32)
        st = binned_zeros(fold, "s")
        P.sbssum(fold, length, ptr(xs[start:]), 1, ptr(st))
        xc, yc = gen_complex("normal", n, 12, np.complex64), gen_complex("normal", n, 13, np.complex64)
        stc = binned_zeros(fold, "c")
        P.cbcdotu(fold, length, ptr(xc[start:]), 1, ptr(yc[start:]), 1, ptr(stc))
        v = gen("loguniform", n, 14, np.float32)
        rec = np.zeros(1 + 2 * fold, np.float32)
        body = binned_zeros(fold, "s")
        rec[0] = P.sbsssq(fold, length, ptr(v[start:]), 1, 0.0, ptr(body))
        rec[1:] = body
        for rev in (False, True):
            for kind, state in (("s", st), ("c", stc), ("ssq", rec)):
                m = rbdist.allgather_merge(torch.from_numpy(state), fold, kind=kind,
                                           merge=_oracle_merge_kind(kind, rev))
                out[(kind, rev)] = m.numpy().tobytes()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_allgather_merge_fp32_kinds():
    """float, float complex and scaled FP32 records through the exchange with 2 ranks."""
    from _ffi import port, ptr, binned_zeros
    from _data import gen, gen_complex
    n, fold, world = 40009, 3, 2
    P = port()
    want = {}
    xs = gen("normal", n, 11, np.float32)
    st = binned_zeros(fold, "s")
    P.sbssum(fold, n, ptr(xs), 1, ptr(st))
    want["s"] = st.tobytes()
    xc, yc = gen_complex("normal", n, 12, np.complex64), gen_complex("normal", n, 13, np.complex64)
    stc = binned_zeros(fold, "c")
    P.cbcdotu(fold, n, ptr(xc), 1, ptr(yc), 1, ptr(stc))
    want["c"] = stc.tobytes()
    v = gen("loguniform", n, 14, np.float32)
    rec = np.zeros(1 + 2 * fold, np.float32)
    body = binned_zeros(fold, "s")
    rec[0] = P.sbsssq(fold, n, ptr(v), 1, 0.0, ptr(body))
    rec[1:] = body
    want["ssq"] = rec.tobytes()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = _free_port()
    procs = [ctx.Process(target=_fp32_worker, args=(r, world, p, n, fold, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, out in got:
        for (kind, rev), b in out.items():
            assert b == want[kind], (rank, kind, rev)
