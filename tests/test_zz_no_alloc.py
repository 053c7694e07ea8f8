"""rb_ddot_noalloc: the dot product for callers that may not allocate device memory
(plugins whose host application owns the device-memory budget, latency-critical callers
that cannot afford a possibly synchronising cudaMalloc). Its scratch is a fixed array
inside the library instead of a workspace allocated on first use.

Checked bit for bit against the oracle and against the regular entry points
(binnedBLAS_dbddot, reproBLAS_rddot) over folds, strides (1, 0, 3), sizes (including N <= 0),
a NULL or a pre-filled accumulator Z, a NULL or a device result, the legacy default stream
and an explicit stream; every case runs two calls in a row, since the calls share the
scratch array and the second must not see the first one's leftovers. Once device code is
loaded, the calls take no device memory. This file is collected last so that a run stopping
at the first failure has already run every other test; it also passes alone in a fresh
process.
"""
import numpy as np
import pytest

from _ffi import binned_zeros, ptr

pytestmark = pytest.mark.gpu

FOLDS = (2, 3, 5, 8)
SIZES = (-1, 0, 1, 33, 100003, 1000003)
INCS = (1, 0, 3)


def _host_inputs(n, inc, seed):
    rng = np.random.default_rng(seed)
    m = max(1, n * max(inc, 1))
    x = np.exp2(rng.uniform(-200, 200, m)) * rng.choice([-1.0, 1.0], m)
    y = rng.standard_normal(m)
    return x, y


def _seed_state(port, fold, seed):
    """A non-empty binned state to accumulate into (the state of a short dot)."""
    rng = np.random.default_rng(seed)
    a, b = rng.uniform(-1e3, 1e3, 50), rng.uniform(-1, 1, 50)
    z = binned_zeros(fold)
    port.dbddot(fold, 50, ptr(a), 1, ptr(b), 1, ptr(z))
    return z


def _check_case(cuda, rb, port, fold, n, inc, mode, stream, seed):
    """One rb_ddot_noalloc call against the oracle and the regular entry points.
    mode: "Z+result", "Z" (result NULL) or "result" (Z NULL)."""
    x, y = _host_inputs(n, inc, seed)
    X, Y = cuda.from_numpy(x).cuda(), cuda.from_numpy(y).cuda()
    z0 = _seed_state(port, fold, seed + 1)
    want = z0.copy()
    port.dbddot(fold, n, ptr(x), inc, ptr(y), inc, ptr(want))
    want_val = port.ddbconv(fold, ptr(want))
    fresh = binned_zeros(fold)
    port.dbddot(fold, n, ptr(x), inc, ptr(y), inc, ptr(fresh))
    fresh_val = port.ddbconv(fold, ptr(fresh))

    Z = cuda.from_numpy(z0.copy()).cuda() if "Z" in mode else None
    res = cuda.full((1,), -7.0, dtype=cuda.float64, device="cuda") if "result" in mode else None
    s = stream.cuda_stream if stream is not None else None
    code = rb.call("rb_ddot_noalloc", fold, n, X, inc, Y, inc, Z, res, s)
    (stream or cuda.cuda.default_stream()).synchronize()
    assert code == 0, (fold, n, inc, mode)
    tag = (fold, n, inc, mode, stream is not None)
    if Z is not None:
        assert Z.cpu().numpy().tobytes() == want.tobytes(), tag
        # the regular accumulate-into entry point gives the same bits
        Zr = cuda.from_numpy(z0.copy()).cuda()
        rb.call("binnedBLAS_dbddot", fold, n, X, inc, Y, inc, Zr)
        assert Zr.cpu().numpy().tobytes() == want.tobytes(), tag
    if res is not None:
        got = res.item()
        if Z is not None:
            assert got == want_val, tag
        else:
            assert got == fresh_val, tag
            assert got == rb.call("reproBLAS_rddot", fold, n, X, inc, Y, inc), tag


@pytest.mark.parametrize("fold", FOLDS)
def test_noalloc_matches_oracle_and_regular_entry_points(cuda, rb, port, fold):
    stream = cuda.cuda.Stream()
    seed = 100 * fold
    for n in SIZES:
        for inc in INCS:
            for mode in ("Z+result", "Z", "result"):
                for st in (None, stream):
                    # two calls in a row on different data
                    _check_case(cuda, rb, port, fold, n, inc, mode, st, seed)
                    _check_case(cuda, rb, port, fold, n, inc, mode, st, seed + 50)
                    seed += 1


def test_noalloc_takes_no_device_memory(cuda, rb):
    """After the first call at each fold (which may load device code), calls allocate
    nothing: the free device memory is unchanged across a run of calls."""
    n = 1 << 20
    rng = np.random.default_rng(9)
    X = cuda.from_numpy(rng.standard_normal(n)).cuda()
    Y = cuda.from_numpy(rng.standard_normal(n)).cuda()
    Z = cuda.zeros(16, dtype=cuda.float64, device="cuda")
    res = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    for fold in FOLDS:
        assert rb.call("rb_ddot_noalloc", fold, n, X, 1, Y, 1, Z, res, None) == 0
    cuda.cuda.synchronize()
    free_before = cuda.cuda.mem_get_info()[0]
    for _ in range(3):
        for fold in FOLDS:
            Z.zero_()
            assert rb.call("rb_ddot_noalloc", fold, n, X, 1, Y, 1, Z, res, None) == 0
            # stride 3 over a third of X (in bounds), stride 0 on Y
            assert rb.call("rb_ddot_noalloc", fold, n // 3, X, 3, Y, 0, None, res, None) == 0
    cuda.cuda.synchronize()
    assert cuda.cuda.mem_get_info()[0] == free_before


def test_noalloc_rejects_host_inputs_misalignment_and_oversized_launch(cuda, rb):
    x = np.ones(16)
    code = rb.lib.rb_ddot_noalloc(3, 16, x.ctypes.data, 1, x.ctypes.data, 1, None, None, None)
    assert code == 1 and b"device memory" in rb.lib.rb_get_last_error_message()
    rb.lib.rb_clear_error()
    X = cuda.ones(1 << 22, dtype=cuda.float64, device="cuda")
    out = cuda.zeros(16, dtype=cuda.float64, device="cuda")
    # Z and result must be 8-byte aligned device memory
    for zp, rp in ((out.data_ptr() + 4, None), (None, out.data_ptr() + 4), (x.ctypes.data, None)):
        code = rb.lib.rb_ddot_noalloc(3, 64, X.data_ptr(), 1, X.data_ptr(), 1, zp, rp, None)
        assert code == 1 and b"aligned" in rb.lib.rb_get_last_error_message()
        rb.lib.rb_clear_error()
    code = rb.lib.rb_ddot_noalloc(1, 64, X.data_ptr(), 1, X.data_ptr(), 1, None, None, None)
    assert code == 1
    rb.lib.rb_clear_error()
    try:
        # 16 CTAs of 32 threads on every SM needs more records than the 128 KiB hold at fold 8
        rb.lib.rb_set_launch_config(16, 32)
        code = rb.lib.rb_ddot_noalloc(8, 1 << 22, X.data_ptr(), 1, X.data_ptr(), 1, None, None, None)
        assert code == 1 and b"scratch holds at most" in rb.lib.rb_get_last_error_message()
    finally:
        rb.lib.rb_set_launch_config(0, 0)
        rb.lib.rb_clear_error()
