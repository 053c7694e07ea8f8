"""The batched ragged form: many segment dot products / sums and small dgemm instances in
one persistent launch run as a CUDA graph. Every result must equal the per-instance plain
call bit for bit, for every schedule the autotuner may pick."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


class Problem:
    def __init__(self, cuda, rb, nseg, max_log2, ngemm, seed, dot=True, with_states=False, fold=3):
        rng = np.random.default_rng(seed)
        self.cuda, self.rb, self.fold = cuda, rb, fold
        lens = np.floor(np.exp2(rng.uniform(0, max_log2, nseg))).astype(np.int64)
        lens[::17] = 0                                   # empty segments too
        offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int64)
        total = int(lens.sum()) + 1
        self.lens, self.offs = lens.astype(np.int32), offs
        self.X = dev(cuda, rng.standard_normal(total))
        self.Y = dev(cuda, rng.standard_normal(total)) if dot else None
        self.results = cuda.zeros(nseg, dtype=cuda.float64, device="cuda")
        self.states = None
        if with_states:
            st = np.zeros(nseg * 2 * fold)
            self.states = dev(cuda, st)
        self.inst = (rb.DgemmInstance * max(ngemm, 1))()
        self.mats = []
        for g in range(ngemm):
            m, n, k = (int(v) for v in rng.integers(16, 257, 3))
            order = "rc"[g % 2]; ta = "nt"[(g // 2) % 2]; tb = "nt"[(g // 4) % 2]
            alpha, beta = [(1.5, 0.5), (1.0, 1.0), (2.0, 0.0), (0.0, 3.0)][g % 4]
            if order == "r":
                lda = k if ta == "n" else m; ldb = n if tb == "n" else k; ldc = n
            else:
                lda = m if ta == "n" else k; ldb = k if tb == "n" else n; ldc = m
            A = dev(cuda, rng.uniform(-1, 1, m * k)); B = dev(cuda, rng.uniform(-1, 1, k * n))
            C0 = rng.uniform(-1, 1, m * n); C = dev(cuda, C0)
            self.mats.append((order, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, C0))
            d = self.inst[g]
            d.order, d.transa, d.transb = order.encode(), ta.encode(), tb.encode()
            d.m, d.n, d.k, d.alpha, d.beta = m, n, k, alpha, beta
            d.A, d.lda, d.B, d.ldb, d.C, d.ldc = A.data_ptr(), lda, B.data_ptr(), ldb, C.data_ptr(), ldc
        self.plan = rb.lib.rb_batch_plan_create(
            fold, nseg, self.offs.ctypes.data, self.lens.ctypes.data, self.X.data_ptr(),
            self.Y.data_ptr() if dot else None, self.results.data_ptr(),
            self.states.data_ptr() if with_states else None, ngemm, ctypes.addressof(self.inst))
        rb.check()
        assert self.plan

    def expected_segments(self, times=1):
        rb, cuda, f = self.rb, self.cuda, self.fold
        out = np.zeros(len(self.lens))
        st = np.zeros(len(self.lens) * 2 * f)
        for i, (o, l) in enumerate(zip(self.offs, self.lens)):
            xs = self.X[o:]
            if self.states is not None:
                z = cuda.zeros(2 * f, dtype=cuda.float64, device="cuda")
                for _ in range(times):
                    if self.Y is not None:
                        rb.call("binnedBLAS_dbddot", f, int(l), xs, 1, self.Y[o:], 1, z)
                    else:
                        rb.call("binnedBLAS_dbdsum", f, int(l), xs, 1, z)
                st[i * 2 * f:(i + 1) * 2 * f] = z.cpu().numpy()
                zz = z.cpu().numpy()
                # conversion through a one-element sum of the state's value is not the same
                # operation; compare states, and results against the state's conversion below
                out[i] = np.nan
            elif self.Y is not None:
                out[i] = rb.call("reproBLAS_rddot", f, int(l), xs, 1, self.Y[o:], 1)
            else:
                out[i] = rb.call("reproBLAS_rdsum", f, int(l), xs, 1)
        return out, st

    def expected_gemms(self, times=1):
        outs = []
        for (order, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, C0) in self.mats:
            Cw = dev(self.cuda, C0)
            for _ in range(times):
                self.rb.call("reproBLAS_rdgemm", self.fold, order, ta, tb, m, n, k, alpha, A, lda, B,
                             ldb, beta, Cw, ldc)
            outs.append(Cw.cpu().numpy())
        return outs

    def gemm_outputs(self):
        return [t[12].cpu().numpy() for t in self.mats]

    def reset_gemms(self):
        for t in self.mats:
            t[12].copy_(self.cuda.from_numpy(t[14]))

    def destroy(self):
        self.rb.lib.rb_batch_plan_destroy(self.plan)


def test_batched_matches_per_instance_calls(cuda, rb):
    P = Problem(cuda, rb, nseg=300, max_log2=16, ngemm=24, seed=1)
    try:
        want_seg, _ = P.expected_segments()
        want_c = P.expected_gemms()
        assert rb.call("rb_batch_plan_run", P.plan, None) == 0
        cuda.cuda.synchronize()
        assert P.results.cpu().numpy().tobytes() == want_seg.tobytes()
        for got, want in zip(P.gemm_outputs(), want_c):
            assert got.tobytes() == want.tobytes()
        # every schedule gives the same bits
        for tile in (0, 1, 2, 3, 4):
            for chunk, small in ((256, 0), (1 << 13, 512), (1 << 15, 1 << 20)):
                P.reset_gemms()
                P.results.zero_()
                assert rb.call("rb_batch_plan_set_config", P.plan, tile, chunk, small, 0) == 0
                assert rb.call("rb_batch_plan_run", P.plan, None) == 0
                cuda.cuda.synchronize()
                assert P.results.cpu().numpy().tobytes() == want_seg.tobytes(), (tile, chunk, small)
                for got, want in zip(P.gemm_outputs(), want_c):
                    assert got.tobytes() == want.tobytes(), (tile, chunk, small)
    finally:
        P.destroy()


def test_autotune_and_graph_replay(cuda, rb):
    P = Problem(cuda, rb, nseg=200, max_log2=15, ngemm=12, seed=2)
    try:
        want_seg, _ = P.expected_segments()
        want_c1 = P.expected_gemms(1)
        want_c2 = P.expected_gemms(2)
        before = [c.copy() for c in P.gemm_outputs()]
        assert rb.call("rb_batch_plan_autotune", P.plan, 2) == 0
        info = [ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong(),
                ctypes.c_int(), ctypes.c_int(), ctypes.c_int()]
        rb.lib.rb_batch_plan_info(P.plan, *[ctypes.byref(v) for v in info])
        assert info[5].value > 0 and info[6].value == 0          # tried, none rejected
        for got, b in zip(P.gemm_outputs(), before):             # outputs restored
            assert got.tobytes() == b.tobytes()
        assert rb.call("rb_batch_plan_run", P.plan, None) == 0
        assert rb.call("rb_batch_plan_run", P.plan, None) == 0   # graph replay
        cuda.cuda.synchronize()
        assert P.results.cpu().numpy().tobytes() == want_seg.tobytes()
        for got, want in zip(P.gemm_outputs(), want_c2):
            assert got.tobytes() == want.tobytes()
        assert any(a.tobytes() != b.tobytes() for a, b in zip(want_c1, want_c2))
    finally:
        P.destroy()


def test_sums_and_states_accumulate(cuda, rb):
    P = Problem(cuda, rb, nseg=150, max_log2=14, ngemm=0, seed=3, dot=False, with_states=True)
    try:
        _, want_st = P.expected_segments(times=2)
        for _ in range(2):
            assert rb.call("rb_batch_plan_run", P.plan, None) == 0
        cuda.cuda.synchronize()
        assert P.states.cpu().numpy().tobytes() == want_st.tobytes()
    finally:
        P.destroy()
