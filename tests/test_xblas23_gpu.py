"""GPU parity of the FP32 real, FP64 complex and FP32 complex gemv / gemm (reproBLAS_r[szc]gemv,
r[szc]gemm, binnedBLAS_sbsgemv, zbzgemv, cbcgemv, sbsgemm, zbzgemm, cbcgemm) through the C
ABI: bit-identical to the reference fixtures and to the oracle, every order and transpose
(n, t, c), folds 2..8, strides, leading dimensions, host and device operands, binned forms
accumulating into non-empty states, and non-finite values."""
import numpy as np
import pytest

from _cmp import from_hex, same_bits, same_state, same_value
from _data import XREAL, gen, gen_complex, xblas23_case_operands
from _xblas import comps, lib_gemm, lib_gemv, rb_gemm, rb_gemv, real_view, state_len
import hashlib

pytestmark = pytest.mark.gpu


def _h(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def dview(cuda, t, a):
    """Device copy of a real or complex numpy array as a real tensor."""
    return dev(cuda, real_view(t, a))


def host_of(t, d, like):
    """numpy array of like's dtype from a real device tensor."""
    return d.cpu().numpy().view(like.dtype)


def _ops(t, n, seed, dist):
    if t == "s":
        return gen(dist, n, seed, np.float32)
    return gen_complex(dist, n, seed, np.complex128 if t == "z" else np.complex64)


def _states(port, t, fold, count, rng):
    n = state_len(t, fold)
    z = np.zeros(count * n, XREAL[t])
    for i in range(count):
        if t == "s":
            port.sbsconv(fold, float(np.float32(rng.standard_normal())), z[i * n:].ctypes.data)
        else:
            v = rng.standard_normal(2).astype(XREAL[t])
            getattr(port, t + "b" + t + "conv")(fold, v.ctypes.data, z[i * n:].ctypes.data)
    return z


def _same_states(a, b, t, fold, count):
    n = state_len(t, fold)
    return all(same_state(a[i * n:(i + 1) * n], b[i * n:(i + 1) * n], fold, comps(t))
               for i in range(count))


def test_golden_xblas23(cuda, rb, golden):
    bad = []
    for c in golden["xblas23"]:
        t, fold = c["t"], c["fold"]
        ops = xblas23_case_operands(c)
        al, be = complex(*c["alpha"]), complex(*c["beta"])
        if c["kind"] == "gemv":
            A, xv, yv = ops
            y = dview(cuda, t, yv)
            rb_gemv(rb, t, fold, c["order"], c["ta"], c["M"], c["N"], al, dview(cuda, t, A), c["lda"],
                    dview(cuda, t, xv), 1, be, y, 1)
            z = dev(cuda, np.zeros(len(yv) * state_len(t, fold), XREAL[t]))
            rb_gemv(rb, t, fold, c["order"], c["ta"], c["M"], c["N"], al, dview(cuda, t, A), c["lda"],
                    dview(cuda, t, xv), 1, be, z, 1, binned=True)
        else:
            A, B, C = ops
            y = dview(cuda, t, C)
            rb_gemm(rb, t, fold, c["order"], c["ta"], c["tb"], c["M"], c["N"], c["K"], al,
                    dview(cuda, t, A), c["lda"], dview(cuda, t, B), c["ldb"], be, y, c["ldc"])
            z = dev(cuda, np.zeros(len(C) * state_len(t, fold), XREAL[t]))
            rb_gemm(rb, t, fold, c["order"], c["ta"], c["tb"], c["M"], c["N"], c["K"], al,
                    dview(cuda, t, A), c["lda"], dview(cuda, t, B), c["ldb"], be, z, c["ldc"],
                    binned=True)
        if not same_bits(y.cpu().numpy(), from_hex(c["out"], XREAL[t])):
            bad.append(("value", c["kind"], t, c["order"], c["ta"], c.get("tb")))
        if _h(z.cpu().numpy()) != c["states_hash"]:
            bad.append(("states", c["kind"], t, c["order"], c["ta"], c.get("tb")))
    assert not bad, bad


# (M, N) shapes: small, one long reduction (rows kernel split over warps; cols kernel row
# chunks merged by the last CTA), many outputs
GEMV_SHAPES = [(1, 1), (3, 70), (37, 53), (300, 17), (17, 2000), (2000, 300), (640, 640)]


@pytest.mark.parametrize("t", ["s", "z", "c"])
def test_xgemv_vs_oracle(cuda, rb, port, t):
    rng = np.random.default_rng(300 + ord(t))
    trial = 0
    for M, N in GEMV_SHAPES:
        for order in "rc":
            for ta in "ntc":
                trial += 1
                fold = [2, 3, 4, 5, 6, 7, 8][trial % 7]
                dist = ["uniform", "normal", "loguniform", "illcond"][trial % 4]
                Rs, Cs = (M, N) if order == "r" else (N, M)
                lda = Cs + (trial % 3)
                A = _ops(t, Rs * lda, trial, dist)
                lenx, leny = (N, M) if ta == "n" else (M, N)
                incx, incy = 1 + trial % 2, 1 + (trial // 2) % 2
                X = _ops(t, lenx * incx, trial + 1, dist)
                Y = _ops(t, leny * incy, trial + 2, "normal")
                al = [1.0, 1.5 - 0.25j, 0.0, -2.0 + 0.5j][trial % 4]
                be = [0.5 + 0.5j, 1.0, 0.0, -0.75][(trial // 4) % 4]
                if t == "s":
                    al, be = complex(al).real, complex(be).real
                want = Y.copy()
                lib_gemv(port, t, fold, order, ta, M, N, al, A, lda, X, incx, be, want, incy)
                host = trial % 3 == 0   # host operands on every third case
                if host:
                    got = Y.copy()
                    rb_gemv(rb, t, fold, order, ta, M, N, al, A, lda, X, incx, be, got, incy)
                else:
                    gd = dview(cuda, t, Y)
                    rb_gemv(rb, t, fold, order, ta, M, N, al, dview(cuda, t, A), lda,
                            dview(cuda, t, X), incx, be, gd, incy)
                    got = host_of(t, gd, Y)
                assert same_value(real_view(t, got), real_view(t, want)), (t, M, N, order, ta, fold, dist, host)
                # binned form into non-empty states
                zs = _states(port, t, fold, leny * incy, rng)
                zw = zs.copy()
                lib_gemv(port, t, fold, order, ta, M, N, al, A, lda, X, incx, be, zw, incy, binned=True)
                zd = dev(cuda, zs)
                rb_gemv(rb, t, fold, order, ta, M, N, al, dview(cuda, t, A), lda, dview(cuda, t, X),
                        incx, be, zd, incy, binned=True)
                assert _same_states(zd.cpu().numpy(), zw, t, fold, leny * incy), (t, M, N, order, ta, fold)


# (M, N, K): tile edges of the 32x32 / 16x32 / 16x16 CTA tiles and the 16 / 32 K tiles
GEMM_SHAPES = [(1, 1, 1), (5, 7, 3), (17, 33, 31), (33, 17, 70), (48, 40, 129)]


@pytest.mark.parametrize("t", ["s", "z", "c"])
def test_xgemm_vs_oracle(cuda, rb, port, t):
    rng = np.random.default_rng(400 + ord(t))
    trial = 0
    for M, N, K in GEMM_SHAPES:
        for order in "rc":
            for ta in "ntc":
                for tb in "ntc":
                    trial += 1
                    fold = [2, 3, 4, 5, 6, 7, 8][trial % 7]
                    dist = ["uniform", "normal", "loguniform", "illcond"][trial % 4]
                    am, an = (M, K) if ta == "n" else (K, M)
                    bm, bn = (K, N) if tb == "n" else (N, K)
                    if order == "r":
                        lda, ldb, ldc = an + trial % 2, bn, N + (trial // 2) % 2
                    else:
                        lda, ldb, ldc = am, bm + trial % 2, M + (trial // 2) % 2
                    A = _ops(t, (am if order == "r" else an) * lda, trial, dist)
                    B = _ops(t, (bm if order == "r" else bn) * ldb, trial + 7, dist)
                    C = _ops(t, (M if order == "r" else N) * ldc, trial + 9, "normal")
                    al = [1.0, 1.5 - 0.25j, 0.0, -2.0 + 0.5j][trial % 4]
                    be = [0.5 + 0.5j, 1.0, 0.0, -0.75][(trial // 4) % 4]
                    if t == "s":
                        al, be = complex(al).real, complex(be).real
                    want = C.copy()
                    lib_gemm(port, t, fold, order, ta, tb, M, N, K, al, A, lda, B, ldb, be, want, ldc)
                    if trial % 4 == 0:
                        got = C.copy()
                        rb_gemm(rb, t, fold, order, ta, tb, M, N, K, al, A, lda, B, ldb, be, got, ldc)
                    else:
                        gd = dview(cuda, t, C)
                        rb_gemm(rb, t, fold, order, ta, tb, M, N, K, al, dview(cuda, t, A), lda,
                                dview(cuda, t, B), ldb, be, gd, ldc)
                        got = host_of(t, gd, C)
                    assert same_value(real_view(t, got), real_view(t, want)), (t, M, N, K, order, ta, tb, fold)
                    if trial % 3 == 0:
                        zs = _states(port, t, fold, len(C), rng)
                        zw = zs.copy()
                        lib_gemm(port, t, fold, order, ta, tb, M, N, K, al, A, lda, B, ldb, be, zw, ldc,
                                 binned=True)
                        zd = dev(cuda, zs)
                        rb_gemm(rb, t, fold, order, ta, tb, M, N, K, al, dview(cuda, t, A), lda,
                                dview(cuda, t, B), ldb, be, zd, ldc, binned=True)
                        assert _same_states(zd.cpu().numpy(), zw, t, fold, len(C)), (t, M, N, K, order, ta, tb)


@pytest.mark.parametrize("t", ["s", "z", "c"])
def test_xblas23_special_values(cuda, rb, port, t):
    """Infinities and NaN in A and x: the affected outputs take the reference's class."""
    rng = np.random.default_rng(500 + ord(t))
    for trial in range(12):
        order, ta = "rc"[trial % 2], "ntc"[trial % 3]
        M, N = 40, 90
        Rs, Cs = (M, N) if order == "r" else (N, M)
        A = _ops(t, Rs * Cs, trial, "uniform")
        for _ in range(3):
            v = [np.inf, -np.inf, np.nan][int(rng.integers(0, 3))]
            i = int(rng.integers(0, Rs * Cs))
            if t == "s":
                A[i] = v
            else:
                A[i] = complex(v, 0.5) if trial % 2 else complex(0.5, v)
        lenx, leny = (N, M) if ta == "n" else (M, N)
        X = _ops(t, lenx, trial + 1, "uniform")
        Y = _ops(t, leny, trial + 2, "uniform")
        al = 1.5 if t == "s" else 1.5 - 0.25j
        want = Y.copy()
        lib_gemv(port, t, 3, order, ta, M, N, al, A, Cs, X, 1, 0.5, want, 1)
        gd = dview(cuda, t, Y)
        rb_gemv(rb, t, 3, order, ta, M, N, al, dview(cuda, t, A), Cs, dview(cuda, t, X), 1, 0.5, gd, 1)
        assert same_value(real_view(t, host_of(t, gd, Y)), real_view(t, want)), (t, order, ta)
        # gemm with the same A as op(A) (M x K = 40 x 90 row-major view)
        if order == "r" and ta == "n":
            B = _ops(t, 90 * 7, trial + 3, "uniform")
            C = _ops(t, 40 * 7, trial + 4, "uniform")
            want = C.copy()
            lib_gemm(port, t, 3, "r", "n", "n", 40, 7, 90, al, A, 90, B, 7, 0.5, want, 7)
            gd = dview(cuda, t, C)
            rb_gemm(rb, t, 3, "r", "n", "n", 40, 7, 90, al, dview(cuda, t, A), 90, dview(cuda, t, B), 7,
                    0.5, gd, 7)
            assert same_value(real_view(t, host_of(t, gd, C)), real_view(t, want)), t


def test_xblas23_errors(cuda, rb):
    """Invalid arguments raise through the error channel; M == 0 or N == 0 touches nothing."""
    A = dev(cuda, np.ones(16, np.float32))
    y = dev(cuda, np.full(4, 7.0, np.float32))
    rb.call("reproBLAS_rsgemv", 3, "r", "n", 0, 4, 1.0, A, 4, A, 1, 0.5, y, 1)
    assert (y.cpu().numpy() == 7.0).all()
    with pytest.raises(rb.ReproBLASError):
        rb.call("reproBLAS_rsgemv", 22, "r", "n", 4, 4, 1.0, A, 4, A, 1, 0.5, y, 1)   # above binned_SBMAXFOLD
    with pytest.raises(rb.ReproBLASError):
        rb.call("reproBLAS_rsgemv", 3, "r", "n", 4, 4, 1.0, A, 2, A, 1, 0.5, y, 1)
    one = np.array([1.0, 0.0], np.float32)
    with pytest.raises(rb.ReproBLASError):
        rb.call("reproBLAS_rcgemm", 3, "r", "n", "n", 2, 2, 2, one, A, 0, A, 2, one, y, 2)


@pytest.mark.parametrize("t", ["s", "z", "c"])
def test_xgemv_extreme_shapes(cuda, rb, port, t):
    """Shapes at the ends of the row split: one row of 200000 elements (every warp of the split
    holds a part of it; the completing warp merges ~190 parts), 3 rows of 100000, and 300000
    rows of 3 elements (many rows per warp); both reductions, value form."""
    for M, N in [(1, 200000), (3, 100000), (300000, 3)]:
        for ta in "nc":
            A = _ops(t, M * N, M + N, "normal")
            lenx, leny = (N, M) if ta == "n" else (M, N)
            X = _ops(t, lenx, 7, "loguniform")
            Y = _ops(t, leny, 8, "normal")
            al = 1.5 if t == "s" else 1.5 - 0.25j
            want = Y.copy()
            lib_gemv(port, t, 3, "r", ta, M, N, al, A, N, X, 1, 0.5, want, 1)
            gd = dview(cuda, t, Y)
            rb_gemv(rb, t, 3, "r", ta, M, N, al, dview(cuda, t, A), N, dview(cuda, t, X), 1, 0.5, gd, 1)
            assert same_value(real_view(t, host_of(t, gd, Y)), real_view(t, want)), (t, M, N, ta)
            # twice in a row: the row tickets are back at zero after a call
            gd2 = dview(cuda, t, Y)
            rb_gemv(rb, t, 3, "r", ta, M, N, al, dview(cuda, t, A), N, dview(cuda, t, X), 1, 0.5, gd2, 1)
            assert same_value(real_view(t, host_of(t, gd2, Y)), real_view(t, want)), (t, M, N, ta, 2)
