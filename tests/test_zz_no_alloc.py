"""rb_ddot_noalloc: the dot product for callers that may not allocate device memory
(plugins whose host application owns the device-memory budget, latency-critical callers
that cannot afford a possibly synchronising cudaMalloc). Its scratch is a fixed array
inside the library instead of a workspace allocated on first use.

Checked against the regular entry points (binnedBLAS_dbddot, reproBLAS_rddot) bit for bit
on two calls in a row, since the calls share that array and the second one must not see
the first one's leftovers. This file is collected last so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(cuda, n, seed):
    rng = np.random.default_rng(seed)
    x = np.exp2(rng.uniform(-200, 200, n)) * rng.choice([-1.0, 1.0], n)
    y = rng.standard_normal(n)
    return cuda.from_numpy(x).cuda(), cuda.from_numpy(y).cuda()


def test_noalloc_matches_regular_entry_points_twice(cuda, rb):
    for call, (n, seed, off) in enumerate([(1000003, 1, 0), (333331, 2, 1)]):
        X, Y = _inputs(cuda, n + off, seed)
        X, Y = X[off:], Y[off:]
        # regular entry points
        zr = cuda.zeros(6, dtype=cuda.float64, device="cuda")
        rb.call("binnedBLAS_dbddot", 3, n, X, 1, Y, 1, zr)
        dr = rb.call("reproBLAS_rddot", 3, n, X, 1, Y, 1)
        # allocation-free entry point, accumulating into a device state and converting
        zn = cuda.zeros(6, dtype=cuda.float64, device="cuda")
        res = cuda.full((1,), -1.0, dtype=cuda.float64, device="cuda")
        free_before = cuda.cuda.mem_get_info()[0]
        code = rb.call("rb_ddot_noalloc", 3, n, X, 1, Y, 1, zn, res, None)
        cuda.cuda.synchronize()
        assert code == 0
        if call == 1:
            # no device memory was taken by the second call
            assert cuda.cuda.mem_get_info()[0] == free_before
        assert zn.cpu().numpy().tobytes() == zr.cpu().numpy().tobytes(), call
        assert res.item() == dr, call


def test_noalloc_rejects_host_inputs_and_oversized_launch(cuda, rb):
    x = np.ones(16)
    code = rb.lib.rb_ddot_noalloc(3, 16, x.ctypes.data, 1, x.ctypes.data, 1, None, None, None)
    assert code == 1 and b"device memory" in rb.lib.rb_get_last_error_message()
    rb.lib.rb_clear_error()
    X = cuda.ones(1 << 22, dtype=cuda.float64, device="cuda")
    try:
        # 16 CTAs of 32 threads on every SM needs more records than the 128 KiB hold at fold 8
        rb.lib.rb_set_launch_config(16, 32)
        code = rb.lib.rb_ddot_noalloc(8, 1 << 22, X.data_ptr(), 1, X.data_ptr(), 1, None, None, None)
        assert code == 1 and b"scratch holds at most" in rb.lib.rb_get_last_error_message()
    finally:
        rb.lib.rb_set_launch_config(0, 0)
        rb.lib.rb_clear_error()
