"""BLAS1 sweep parity at full size: dsum, ddot, dnrm2, dasum (FP64), ssum, sdot, snrm2, sasum
(FP32), zsum, zdotc, zdotu, dznrm2, dzasum (complex128), csum, scnrm2, scasum (complex64) at
N = 2^10, 2^12, ..., 2^28 elements, folds 2, 3 and 4, for uniform,
normal, log-uniform and ill-conditioned inputs. Every GPU result (binned state, the
sum-of-squares scale, and the converted value of the reproBLAS_r* call) must equal the
reference library bit for bit, and the largest N must give the same bits under 8 grid/block
launch configurations (the reproducibility check of tests/checks/verify_daugsum.c:56-95).

The reference side is the ReproBLAS library compiled from its own sources (oracle/_ref; the
oracle restatement, pinned to it by test_oracle_pin.py, stands in where it is absent). Its
binned states are resumable, so one accumulating pass per (routine, fold) yields the state of
every prefix: the pass adds [2^(2k-2), 2^(2k)) to the state of the previous prefix, which
is the state of a single call over [0, 2^(2k)) (binned sums depend only on the multiset of
deposited values). The reference passes run on host threads while the GPU calls run, and
the inputs are seeded fills whose prefixes are the shorter vectors (oracle/rb_fill.c).
"""
from concurrent.futures import ThreadPoolExecutor

import pytest

from _cmp import same_state, same_value
from _ffi import host_threads, port, ref
from _sweep import (DISTS, FOLDS, GROUPS, LAUNCH_CONFIGS, LOGN, NMAX, SSQ, gpu_call, gpu_state,
                    group_inputs, reference_prefixes)
from _sweep import comps as sweep_comps

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("group", list(GROUPS))
@pytest.mark.parametrize("dist", DISTS)
def test_blas1_sweep_bit_exact(cuda, rb, dist, group):
    L = ref() or port()
    x, y = group_inputs(dist, group)
    routines = GROUPS[group]
    jobs = [(r, f) for r in routines for f in FOLDS]
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), host_threads()))) as ex:
        futs = {(r, f): ex.submit(reference_prefixes, L, r, f, x, y) for r, f in jobs}
        X = cuda.from_numpy(x).cuda()
        Y = cuda.from_numpy(y).cuda() if y is not None else None
        got, got_cfg = {}, {}
        for r, f in jobs:
            for lg in LOGN:
                got[(r, f, lg)] = gpu_call(cuda, rb, r, f, 1 << lg, X, Y)
        try:
            for cps, thr in LAUNCH_CONFIGS:
                rb.call("rb_set_launch_config", cps, thr)
                for r, f in jobs:
                    got_cfg[(r, f, cps, thr)] = gpu_state(cuda, rb, r, f, NMAX, X, Y)
        finally:
            rb.call("rb_set_launch_config", 0, 0)
        want = {k: fu.result() for k, fu in futs.items()}
    del X, Y
    bad = []
    for (r, f, lg), (st, scl, val) in got.items():
        wst, wscl, wval = want[(r, f)][lg]
        comps = sweep_comps(r)
        if not same_state(st, wst, f, comps):
            bad.append((r, f, lg, "state"))
        if r in SSQ and scl != wscl:
            bad.append((r, f, lg, "scale", scl, wscl))
        if not same_value(val, wval):
            bad.append((r, f, lg, "value", val, wval))
    for (r, f, cps, thr), (st, scl) in got_cfg.items():
        wst, wscl, _ = want[(r, f)][LOGN[-1]]
        comps = sweep_comps(r)
        if not same_state(st, wst, f, comps) or (r in SSQ and scl != wscl):
            bad.append((r, f, "launch", cps, thr))
    assert not bad, (dist, group, "reference" if ref() else "oracle", bad[:10])
