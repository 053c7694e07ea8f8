"""Failure paths, exercised without a GPU fault (no trap, no bad address, no endless wait):

* a bounded pipeline wait that runs out: the test hook rb_debug_pipeline_fault makes the TMA
  producers of the dgemv and int8-sliced dgemm kernels stop feeding their rings after a few
  stages and shortens the consumers' wait for a stage's data to a few milliseconds. The
  kernels must give up cleanly: status reported (RB_ERR_CUDA, at once for calls that wait
  for their stream, by rb_synchronize for asynchronous ones), the entries they could not
  finish NaN and every other entry exact, copies and tensor-core work drained, TMEM freed
  (the next calls run and return the oracle's bits);
* an allocation that fails: the test hook rb_debug_fail_allocations makes the next workspace
  allocations fail as on an exhausted device; the call reports RB_ERR_ALLOC, a
  value-returning call returns NaN, outputs are untouched, and the next call succeeds.
"""
import math

import numpy as np
import pytest

from _ffi import ptr

pytestmark = pytest.mark.gpu

RB_ERR_CUDA = 2
RB_ERR_ALLOC = 3
STOP_AFTER = 2        # stages each CTA's producer issues before it stops
SHORT_WAIT = 20000    # polls (a few milliseconds) before a consumer gives up


def _nan_or_exact(got, want):
    """Every entry is NaN (not finished) or has exactly the expected bits."""
    nan = np.isnan(got)
    return bool(np.all(nan | (got.view(np.int64) == want.view(np.int64)))), float(nan.mean())


@pytest.mark.parametrize("trans", ["n", "t"])
def test_gemv_pipeline_wait_gives_up(cuda, rb, port, trans):
    m = n = 4096
    rng = np.random.default_rng(41)
    A = rng.uniform(-1, 1, m * n)
    x = rng.uniform(-1, 1, n if trans == "n" else m)
    y = rng.uniform(-1, 1, m if trans == "n" else n)
    want = y.copy()
    port.rdgemv(3, b"r", trans.encode(), m, n, 1.5, ptr(A), n, ptr(x), 1, 0.5, ptr(want), 1)
    Ad, xd = cuda.from_numpy(A).cuda(), cuda.from_numpy(x).cuda()
    lib = rb.lib
    try:
        lib.rb_clear_error()
        lib.rb_debug_pipeline_fault(STOP_AFTER, SHORT_WAIT)
        # host y: the call waits for its stream and reports the give-up itself
        yh = y.copy()
        lib.reproBLAS_rdgemv(3, b"r", trans.encode(), m, n, 1.5, Ad.data_ptr(), n, xd.data_ptr(), 1,
                             0.5, yh.ctypes.data, 1)
        assert lib.rb_get_last_error() == RB_ERR_CUDA
        assert b"timed out" in lib.rb_get_last_error_message()
        ok, frac = _nan_or_exact(yh, want)
        assert ok and frac > 0.5, frac
        lib.rb_clear_error()
        # device y: the call only enqueues; rb_synchronize reports the give-up
        yd = cuda.from_numpy(y.copy()).cuda()
        lib.reproBLAS_rdgemv(3, b"r", trans.encode(), m, n, 1.5, Ad.data_ptr(), n, xd.data_ptr(), 1,
                             0.5, yd.data_ptr(), 1)
        assert lib.rb_get_last_error() == 0
        assert lib.rb_synchronize() == RB_ERR_CUDA
        ok, frac = _nan_or_exact(yd.cpu().numpy(), want)
        assert ok and frac > 0.5, frac
    finally:
        lib.rb_debug_pipeline_fault(-1, 0)
        lib.rb_clear_error()
    # the context stays usable and no stale status is left behind
    assert lib.rb_synchronize() == 0
    yh = y.copy()
    rb.call("reproBLAS_rdgemv", 3, "r", trans, m, n, 1.5, Ad, n, xd, 1, 0.5, yh, 1)
    assert yh.tobytes() == want.tobytes()
    yd = cuda.from_numpy(y.copy()).cuda()
    rb.call("reproBLAS_rdgemv", 3, "r", trans, m, n, 1.5, Ad, n, xd, 1, 0.5, yd, 1)
    assert rb.lib.rb_synchronize() == 0
    assert yd.cpu().numpy().tobytes() == want.tobytes()


def test_int8_pipeline_wait_gives_up(cuda, rb):
    n, S = 512, 4
    rng = np.random.default_rng(42)
    A = cuda.from_numpy(rng.uniform(-1, 1, (n, n))).cuda()
    B = cuda.from_numpy(rng.uniform(-1, 1, (n, n))).cuda()
    C0 = rng.uniform(-1, 1, (n, n))
    C = cuda.from_numpy(C0.copy()).cuda()
    assert rb.call("rb_dgemm_int8", 3, "r", "n", "n", n, n, n, 1.5, A, n, B, n, 0.5, C, n, S) == 0
    want = C.cpu().numpy()
    lib = rb.lib
    try:
        lib.rb_clear_error()
        lib.rb_debug_pipeline_fault(STOP_AFTER, SHORT_WAIT)
        C.copy_(cuda.from_numpy(C0))
        code = lib.rb_dgemm_int8(3, b"r", b"n", b"n", n, n, n, 1.5, A.data_ptr(), n, B.data_ptr(), n,
                                 0.5, C.data_ptr(), n, S)
        assert code == RB_ERR_CUDA and b"timed out" in lib.rb_get_last_error_message()
        ok, frac = _nan_or_exact(C.cpu().numpy(), want)
        assert ok and frac > 0.5, frac
    finally:
        lib.rb_debug_pipeline_fault(-1, 0)
        lib.rb_clear_error()
    # TMEM was freed and the pipeline drained: the next calls run and give the same bits
    for _ in range(2):
        C.copy_(cuda.from_numpy(C0))
        assert rb.call("rb_dgemm_int8", 3, "r", "n", "n", n, n, n, 1.5, A, n, B, n, 0.5, C, n, S) == 0
        assert C.cpu().numpy().tobytes() == want.tobytes()


def test_workspace_allocation_failure(cuda, rb, port):
    n = 100003
    rng = np.random.default_rng(43)
    x, y = rng.standard_normal(n), rng.uniform(-1, 1, n)
    X, Y = cuda.from_numpy(x).cuda(), cuda.from_numpy(y).cuda()
    want = port.rddot(3, n, ptr(x), 1, ptr(y), 1)
    m = 512
    A = rng.uniform(-1, 1, m * m)
    gx, gy = rng.uniform(-1, 1, m), rng.uniform(-1, 1, m)
    gwant = gy.copy()
    port.rdgemv(3, b"r", b"n", m, m, 1.5, ptr(A), m, ptr(gx), 1, 0.5, ptr(gwant), 1)
    lib = rb.lib
    stream = cuda.cuda.Stream()   # no call has used it yet: its workspace is made on first use
    lib.rb_set_stream(stream.cuda_stream)
    try:
        lib.rb_clear_error()
        lib.rb_debug_fail_allocations(1)
        v = lib.reproBLAS_rddot(3, n, X.data_ptr(), 1, Y.data_ptr(), 1)
        assert math.isnan(v) and lib.rb_get_last_error() == RB_ERR_ALLOC
        lib.rb_clear_error()
        # the failed set-up was released: the next call builds the workspace and succeeds
        assert rb.call("reproBLAS_rddot", 3, n, X, 1, Y, 1) == want
        # host operands need the grow-on-demand buffer: its allocation fails, y is untouched
        lib.rb_debug_fail_allocations(1)
        yh = gy.copy()
        lib.reproBLAS_rdgemv(3, b"r", b"n", m, m, 1.5, A.ctypes.data, m, gx.ctypes.data, 1, 0.5,
                             yh.ctypes.data, 1)
        assert lib.rb_get_last_error() == RB_ERR_ALLOC
        assert yh.tobytes() == gy.tobytes()
        lib.rb_clear_error()
        rb.call("reproBLAS_rdgemv", 3, "r", "n", m, m, 1.5, A, m, gx, 1, 0.5, yh, 1)
        assert yh.tobytes() == gwant.tobytes()
    finally:
        lib.rb_debug_fail_allocations(0)
        stream.synchronize()
        lib.rb_set_stream(None)
        lib.rb_clear_error()
