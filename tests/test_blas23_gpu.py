"""GPU parity of the binned dgemv / plain binned dgemm through the C ABI: bit-identical to
the reference fixtures and to the oracle restatement, all orders and transposes, alpha/beta
special values, folds 2..8, strides, binned (accumulating) entry points, and the benchmark
shapes (gemv 4096x4096, 16384x1024, 1024x16384; dgemm 2048^3 sampled)."""
import numpy as np
import pytest

from _cmp import from_hex, same_bits, same_state
from _data import blas23_operands
from _ffi import binned_zeros, ptr, ref

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def test_golden_blas23(cuda, rb, golden):
    for c in golden["blas23"]:
        for on_dev in (True, False):
            if c["kind"] == "gemv":
                A, xv, yv = blas23_operands(c["seed"], c["M"] * c["N"], 64, 64)
                if on_dev:
                    Y = dev(cuda, yv)
                    rb.call("reproBLAS_rdgemv", 3, c["order"], c["ta"], c["M"], c["N"], 1.5,
                            dev(cuda, A), c["lda"], dev(cuda, xv), 1, 0.5, Y, 1)
                    out = Y.cpu().numpy()
                else:
                    out = yv.copy()
                    rb.call("reproBLAS_rdgemv", 3, c["order"], c["ta"], c["M"], c["N"], 1.5, A,
                            c["lda"], xv, 1, 0.5, out, 1)
            else:
                A, B, C = blas23_operands(c["seed"], c["M"] * c["K"], c["K"] * c["N"], c["M"] * c["N"])
                if on_dev:
                    Cd = dev(cuda, C)
                    rb.call("reproBLAS_rdgemm", 3, c["order"], c["ta"], c["tb"], c["M"], c["N"],
                            c["K"], 1.5, dev(cuda, A), c["lda"], dev(cuda, B), c["ldb"], 0.5, Cd, c["ldc"])
                    out = Cd.cpu().numpy()
                else:
                    out = C.copy()
                    rb.call("reproBLAS_rdgemm", 3, c["order"], c["ta"], c["tb"], c["M"], c["N"],
                            c["K"], 1.5, A, c["lda"], B, c["ldb"], 0.5, out, c["ldc"])
            assert same_bits(out, from_hex(c["out"], np.float64)), (c["kind"], c["order"], c["ta"], on_dev)


AB = [(1.5, 0.5), (1.0, 1.0), (0.0, 2.0), (2.0, 0.0), (1.0, 0.0), (-3.0, 1.0)]


@pytest.mark.parametrize("fold", [2, 3, 4, 6, 8])
def test_gemv_vs_oracle(cuda, rb, port, fold):
    rng = np.random.default_rng(fold)
    for (M, N) in [(1, 1), (7, 33), (33, 7), (255, 512), (64, 1500)]:
        for order in "rc":
            for ta in "nt":
                for alpha, beta in AB[fold % 3::2]:
                    lda = (N if order == "r" else M) + 3
                    rows = M if order == "r" else N
                    A = np.exp2(rng.uniform(-30, 30, rows * lda)) * rng.choice([-1.0, 1.0], rows * lda)
                    lenx = N if ta == "n" else M
                    leny = M if ta == "n" else N
                    x = rng.standard_normal(lenx * 2)
                    y = rng.standard_normal(leny * 3)
                    want = y.copy()
                    port.rdgemv(fold, order.encode(), ta.encode(), M, N, alpha, ptr(A), lda,
                                ptr(x), 2, beta, ptr(want), 3)
                    Y = dev(cuda, y)
                    rb.call("reproBLAS_rdgemv", fold, order, ta, M, N, alpha, dev(cuda, A), lda,
                            dev(cuda, x), 2, beta, Y, 3)
                    assert same_bits(Y.cpu().numpy(), want), (M, N, order, ta, alpha, beta)


@pytest.mark.parametrize("fold", [2, 3, 5, 8])
def test_gemm_vs_oracle(cuda, rb, port, fold):
    rng = np.random.default_rng(100 + fold)
    for (M, N, K) in [(1, 1, 1), (5, 7, 9), (33, 65, 31), (70, 40, 130)]:
        for order in "rc":
            for ta in "nt":
                for tb in "nt":
                    alpha, beta = AB[(M + N + K + fold) % len(AB)]
                    A = np.exp2(rng.uniform(-20, 20, M * K)) * rng.choice([-1.0, 1.0], M * K)
                    B = rng.uniform(-1, 1, K * N)
                    C = rng.standard_normal(M * N)
                    if order == "r":
                        lda = K if ta == "n" else M; ldb = N if tb == "n" else K; ldc = N
                    else:
                        lda = M if ta == "n" else K; ldb = K if tb == "n" else N; ldc = M
                    want = C.copy()
                    port.rdgemm(fold, order.encode(), ta.encode(), tb.encode(), M, N, K, alpha,
                                ptr(A), lda, ptr(B), ldb, beta, ptr(want), ldc)
                    Cd = dev(cuda, C)
                    rb.call("reproBLAS_rdgemm", fold, order, ta, tb, M, N, K, alpha, dev(cuda, A),
                            lda, dev(cuda, B), ldb, beta, Cd, ldc)
                    assert same_bits(Cd.cpu().numpy(), want), (M, N, K, order, ta, tb, alpha, beta)


def test_binned_entry_points_accumulate(cuda, rb, port):
    rng = np.random.default_rng(7)
    fold = 3
    M, N, K = 37, 29, 300
    A = rng.standard_normal(M * K); B = rng.standard_normal(K * N)
    # two K-halves accumulated into the same binned C equal the whole product
    want = binned_zeros(fold, n=M * N)
    port.dbdgemm(fold, b"r", b"n", b"n", M, N, K, 1.5, ptr(A), K, ptr(B), N, ptr(want), N)
    Cb = dev(cuda, binned_zeros(fold, n=M * N))
    A2 = A.reshape(M, K)
    B2 = B.reshape(K, N)
    for k0, k1 in [(0, 111), (111, K)]:
        a = np.ascontiguousarray(A2[:, k0:k1]); b = np.ascontiguousarray(B2[k0:k1, :])
        rb.call("binnedBLAS_dbdgemm", fold, "r", "n", "n", M, N, k1 - k0, 1.5, dev(cuda, a), k1 - k0,
                dev(cuda, b), N, Cb, N)
    assert same_bits(Cb.cpu().numpy(), want)
    # binned gemv into existing states (host states this time)
    x = rng.standard_normal(K)
    pre = binned_zeros(fold, n=M)
    for i in range(M):
        port.dbdconv(fold, float(i) - 3.5, ptr(pre[i * 2 * fold:]))
    want = pre.copy()
    port.dbdgemv(fold, b"r", b"n", M, K, 0.75, ptr(A), K, ptr(x), 1, ptr(want), 1)
    got = pre.copy()
    rb.call("binnedBLAS_dbdgemv", fold, "r", "n", M, K, 0.75, A, K, x, 1, got, 1)
    assert same_bits(got, want)


@pytest.mark.parametrize("shape", [(4096, 4096), (16384, 1024), (1024, 16384)])
@pytest.mark.parametrize("ta", ["n", "t"])
def test_gemv_benchmark_shapes(cuda, rb, port, shape, ta):
    """dgemv configuration: uniform(-1,1), alpha 1.5, beta 0.5, fold 3, row-major; checked
    against the reference library (the oracle where it is absent)."""
    M, N = shape
    rng = np.random.default_rng(M + N)
    A = rng.uniform(-1, 1, M * N)
    x = rng.uniform(-1, 1, N if ta == "n" else M)
    y = rng.uniform(-1, 1, M if ta == "n" else N)
    want = y.copy()
    (ref() or port).rdgemv(3, b"r", ta.encode(), M, N, 1.5, ptr(A), N, ptr(x), 1, 0.5,
                           ptr(want), 1)
    Y = dev(cuda, y)
    rb.call("reproBLAS_rdgemv", 3, "r", ta, M, N, 1.5, dev(cuda, A), N, dev(cuda, x), 1, 0.5, Y, 1)
    assert same_bits(Y.cpu().numpy(), want)


# Column-reduction shapes (row-major, Trans: N outputs, M-long reductions). Even N takes the
# TMA-fed kernel, whose thread groups per output (2, 4, 8) these shapes vary, odd N (odd lda)
# the register-streaming kernel with its row groups (1, 2, 4, 8).
@pytest.mark.parametrize("shape", [(2, 2), (2, 3), (64, 8192), (64, 8191), (4096, 4096),
                                   (3000, 600), (3000, 601), (20000, 3001), (5000, 130)])
def test_gemv_column_reduction_shapes(cuda, rb, port, shape):
    M, N = shape
    rng = np.random.default_rng(7 * M + N)
    A = np.exp2(rng.uniform(-25, 25, M * N)) * rng.choice([-1.0, 1.0], M * N)
    x = rng.uniform(-1, 1, M)
    y = rng.uniform(-1, 1, N)
    want = y.copy()
    port.rdgemv(3, b"r", b"t", M, N, 1.5, ptr(A), N, ptr(x), 1, 0.5, ptr(want), 1)
    Y = dev(cuda, y)
    rb.call("reproBLAS_rdgemv", 3, "r", "t", M, N, 1.5, dev(cuda, A), N, dev(cuda, x), 1, 0.5, Y, 1)
    assert same_bits(Y.cpu().numpy(), want)
    # binned form into existing states, fold 5
    fold = 5
    wantb = binned_zeros(fold, n=N)
    port.dbdgemv(fold, b"r", b"t", M, N, 0.75, ptr(A), N, ptr(x), 1, ptr(wantb), 1)
    Yb = dev(cuda, binned_zeros(fold, n=N))
    rb.call("binnedBLAS_dbdgemv", fold, "r", "t", M, N, 0.75, dev(cuda, A), N, dev(cuda, x), 1, Yb, 1)
    assert same_bits(Yb.cpu().numpy(), wantb)


def test_gemm_2048_sampled(cuda, rb, port):
    """Plain binned dgemm, M=N=K=2048, uniform(-1,1), alpha 1.5, beta 0.5, fold 3: 512 sampled
    entries equal the reference library's (the oracle's where it is absent) binned(beta*C_ij)
    + binned dot of row and column; the column-major transposed formulation of the same product
    gives identical bits."""
    L = ref() or port
    n = 2048
    rng = np.random.default_rng(2048)
    A = rng.uniform(-1, 1, n * n); B = rng.uniform(-1, 1, n * n); C = rng.uniform(-1, 1, n * n)
    Cd = dev(cuda, C)
    rb.call("reproBLAS_rdgemm", 3, "r", "n", "n", n, n, n, 1.5, dev(cuda, A), n, dev(cuda, B), n,
            0.5, Cd, n)
    got = Cd.cpu().numpy().reshape(n, n)
    A2 = A.reshape(n, n); B2 = B.reshape(n, n); C2 = C.reshape(n, n)
    for _ in range(512):
        i, j = int(rng.integers(0, n)), int(rng.integers(0, n))
        a = np.ascontiguousarray(A2[i, :]) * 1.5
        b = np.ascontiguousarray(B2[:, j])
        st = binned_zeros(3)
        L.dbdconv(3, C2[i, j] * 0.5, ptr(st))
        L.dbddot(3, n, ptr(a), 1, ptr(b), 1, ptr(st))
        assert L.ddbconv(3, ptr(st)) == got[i, j], (i, j)
    # C^T = B^T A^T in column-major with both operands transposed
    Ct = dev(cuda, np.ascontiguousarray(C2.T))
    rb.call("reproBLAS_rdgemm", 3, "c", "t", "t", n, n, n, 1.5, dev(cuda, A), n, dev(cuda, B), n,
            0.5, Ct, n)
    assert same_bits(Ct.cpu().numpy().reshape(n, n).T, got)


@pytest.mark.parametrize("ta", ["n", "t"])
def test_gemv_x_layouts(cuda, rb, port, ta):
    """x read in place (unit stride, aligned), through a gathered copy (stride 3, or unit
    stride at an odd 8-byte offset), alpha 1 and not, fold 2 and 3."""
    M, N = 1000, 1200
    rng = np.random.default_rng(11)
    A = rng.uniform(-1, 1, M * N)
    lx, ly = (N, M) if ta == "n" else (M, N)
    buf = rng.uniform(-1, 1, 3 * lx + 1)
    y0 = rng.uniform(-1, 1, ly)
    dA = dev(cuda, A)
    dbuf = dev(cuda, buf)
    for fold in (2, 3):
        for alpha in (1.0, 1.5):
            for off, inc in ((0, 1), (1, 1), (0, 3)):
                xs = buf[off:off + (lx - 1) * inc + 1]
                want = y0.copy()
                port.rdgemv(fold, b"r", ta.encode(), M, N, alpha, ptr(A), N, ptr(xs), inc, 0.5,
                            ptr(want), 1)
                Y = dev(cuda, y0)
                rb.call("reproBLAS_rdgemv", fold, "r", ta, M, N, alpha, dA, N, dbuf[off:], inc, 0.5, Y, 1)
                assert same_bits(Y.cpu().numpy(), want), (fold, alpha, off, inc)
