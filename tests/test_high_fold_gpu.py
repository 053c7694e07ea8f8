"""GPU parity at the folds above the register-resident kernels (2..8): every fold the
reference accepts, up to binned_DBMAXFOLD = 52 (FP64 and double complex) and
binned_SBMAXFOLD = 21 (FP32 and float complex) (include/binned.h:123,131). Checked bit for
bit against the oracle (pinned to the reference at these folds by test_oracle_pin.py) at
folds 9, 16 and 52 / 9 and 21: every BLAS1 reduction and its binned form, accumulation into
device and host states, strides, host inputs, launch shapes, gemv / gemm of every element
type, order and transpose, binned gemv / gemm into non-empty states, the state merges, a
manual-layout form; folds past the maximum are rejected."""
import math

import numpy as np
import pytest

from _cmp import same_bits, same_state, same_value
from _data import XREAL, gen, gen_complex
from _ffi import binned_zeros, ptr
from _xblas import comps, lib_gemm, lib_gemv, rb_gemm, rb_gemv, real_view, state_len

pytestmark = pytest.mark.gpu

DFOLDS = (9, 16, 52)
SFOLDS = (9, 21)


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("fold", DFOLDS)
def test_fp64_reductions(cuda, rb, port, fold):
    n = 70001
    x, y = gen("loguniform", n, fold), gen("normal", n, fold + 1)
    X, Y = dev(cuda, x), dev(cuda, y)
    # sum, asum, dot: binned states and values
    for name, pname, args_g, args_p in (
            ("dbdsum", "dbdsum", (X, 1), (ptr(x), 1)),
            ("dbdasum", "dbdasum", (X, 1), (ptr(x), 1)),
            ("dbddot", "dbddot", (X, 1, Y, 1), (ptr(x), 1, ptr(y), 1))):
        want = binned_zeros(fold)
        getattr(port, pname)(fold, n, *args_p, ptr(want))
        z = dev(cuda, binned_zeros(fold))
        rb.call("binnedBLAS_" + name, fold, n, *args_g, z)
        assert same_bits(z.cpu().numpy(), want), (name, fold)
    assert same_value(rb.call("reproBLAS_rdsum", fold, n, X, 1), port.rdsum(fold, n, ptr(x), 1))
    assert same_value(rb.call("reproBLAS_rddot", fold, n, X, 1, Y, 1),
                      port.rddot(fold, n, ptr(x), 1, ptr(y), 1))
    assert same_value(rb.call("reproBLAS_rdasum", fold, n, X, 1), port.rdasum(fold, n, ptr(x), 1))
    # scaled sum of squares and the 2-norm, on data whose reference result does not depend on
    # the decomposition (see test_reference_ssq_order_dependence_at_high_folds)
    s = x if fold < 28 else y
    S = X if fold < 28 else Y
    want = binned_zeros(fold)
    wscl = port.dbdssq(fold, n, ptr(s), 1, 0.0, ptr(want))
    z = dev(cuda, binned_zeros(fold))
    scl = rb.call("binnedBLAS_dbdssq", fold, n, S, 1, 0.0, z)
    assert same_bits(z.cpu().numpy(), want) and scl == wscl
    assert same_value(rb.call("reproBLAS_rdnrm2", fold, n, S, 1), port.rdnrm2(fold, n, ptr(s), 1))
    # accumulation into a device state over two calls, and into a host state
    whole = binned_zeros(fold)
    port.dbddot(fold, n, ptr(x), 1, ptr(y), 1, ptr(whole))
    z = dev(cuda, binned_zeros(fold))
    rb.call("binnedBLAS_dbddot", fold, 12345, X, 1, Y, 1, z)
    rb.call("binnedBLAS_dbddot", fold, n - 12345, X[12345:], 1, Y[12345:], 1, z)
    assert same_bits(z.cpu().numpy(), whole)
    zh = binned_zeros(fold)
    rb.call("binnedBLAS_dbddot", fold, n, x, 1, y, 1, zh)   # host inputs and state
    assert same_bits(zh, whole)
    # strides
    want = binned_zeros(fold)
    port.dbddot(fold, n // 3, ptr(x), 3, ptr(y), 2, ptr(want))
    z = dev(cuda, binned_zeros(fold))
    rb.call("binnedBLAS_dbddot", fold, n // 3, X, 3, Y, 2, z)
    assert same_bits(z.cpu().numpy(), want)


@pytest.mark.parametrize("fold", DFOLDS)
def test_complex128_reductions(cuda, rb, port, fold):
    n = 30011
    xz, yz = gen_complex("loguniform", n, fold), gen_complex("normal", n, fold + 1)
    X, Y = dev(cuda, xz.view(np.float64)), dev(cuda, yz.view(np.float64))
    for name, args_g, args_p in (("zbzsum", (X, 1), (ptr(xz), 1)),
                                 ("zbzdotc", (X, 1, Y, 1), (ptr(xz), 1, ptr(yz), 1)),
                                 ("zbzdotu", (X, 1, Y, 1), (ptr(xz), 1, ptr(yz), 1))):
        want = binned_zeros(fold, "z")
        getattr(port, name)(fold, n, *args_p, ptr(want))
        z = dev(cuda, binned_zeros(fold, "z"))
        rb.call("binnedBLAS_" + name, fold, n, *args_g, z)
        assert same_bits(z.cpu().numpy(), want), (name, fold)
    o = dev(cuda, np.zeros(2))
    w = np.zeros(2)
    rb.call("reproBLAS_rzdotc_sub", fold, n, X, 1, Y, 1, o)
    port.rzdotc_sub(fold, n, ptr(xz), 1, ptr(yz), 1, ptr(w))
    assert same_value(o.cpu().numpy(), w)
    # |re| + |im| and the scaled sum of squares of the components
    want = binned_zeros(fold)
    port.dbzasum(fold, n, ptr(xz), 1, ptr(want))
    z = dev(cuda, binned_zeros(fold))
    rb.call("binnedBLAS_dbzasum", fold, n, X, 1, z)
    assert same_bits(z.cpu().numpy(), want)
    sz, SZ = (xz, X) if fold < 28 else (yz, Y)
    want = binned_zeros(fold)
    wscl = port.dbzssq(fold, n, ptr(sz), 1, 0.0, ptr(want))
    z = dev(cuda, binned_zeros(fold))
    scl = rb.call("binnedBLAS_dbzssq", fold, n, SZ, 1, 0.0, z)
    assert same_bits(z.cpu().numpy(), want) and scl == wscl
    assert same_value(rb.call("reproBLAS_rdznrm2", fold, n, SZ, 1), port.rdznrm2(fold, n, ptr(sz), 1))


@pytest.mark.parametrize("fold", SFOLDS)
def test_fp32_reductions(cuda, rb, port, fold):
    n = 50021
    x, y = gen("loguniform", n, fold, np.float32), gen("normal", n, fold + 1, np.float32)
    X, Y = dev(cuda, x), dev(cuda, y)
    for name, args_g, args_p in (("sbssum", (X, 1), (ptr(x), 1)),
                                 ("sbsasum", (X, 1), (ptr(x), 1)),
                                 ("sbsdot", (X, 1, Y, 1), (ptr(x), 1, ptr(y), 1))):
        want = binned_zeros(fold, "s")
        getattr(port, name)(fold, n, *args_p, ptr(want))
        z = dev(cuda, binned_zeros(fold, "s"))
        rb.call("binnedBLAS_" + name, fold, n, *args_g, z)
        assert same_state(z.cpu().numpy(), want, fold), (name, fold)
    assert same_value(np.float32(rb.call("reproBLAS_rssum", fold, n, X, 1)),
                      np.float32(port.rssum(fold, n, ptr(x), 1)))
    assert same_value(np.float32(rb.call("reproBLAS_rsdot", fold, n, X, 1, Y, 1)),
                      np.float32(port.rsdot(fold, n, ptr(x), 1, ptr(y), 1)))
    # the FP32 scaled sum of squares on normal values (wide exponent ranges make the
    # reference's result depend on its decomposition from fold 11 on)
    want = binned_zeros(fold, "s")
    wscl = port.sbsssq(fold, n, ptr(y), 1, 0.0, ptr(want))
    z = dev(cuda, binned_zeros(fold, "s"))
    scl = rb.call("binnedBLAS_sbsssq", fold, n, Y, 1, 0.0, z)
    assert same_bits(z.cpu().numpy(), want) and scl == wscl
    assert same_value(np.float32(rb.call("reproBLAS_rsnrm2", fold, n, Y, 1)),
                      np.float32(port.rsnrm2(fold, n, ptr(y), 1)))
    # float complex sum and dots (calls of up to 256 elements are where the reference's own
    # float-complex dots stay canonical; the oracle computes the documented sum at any length)
    xc, yc = gen_complex("normal", n, fold, np.complex64), gen_complex("uniform", n, fold + 1, np.complex64)
    XC, YC = dev(cuda, xc.view(np.float32)), dev(cuda, yc.view(np.float32))
    for name, args_g, args_p in (("cbcsum", (XC, 1), (ptr(xc), 1)),
                                 ("cbcdotc", (XC, 1, YC, 1), (ptr(xc), 1, ptr(yc), 1)),
                                 ("cbcdotu", (XC, 1, YC, 1), (ptr(xc), 1, ptr(yc), 1))):
        want = binned_zeros(fold, "c")
        getattr(port, name)(fold, n, *args_p, ptr(want))
        z = dev(cuda, binned_zeros(fold, "c"))
        rb.call("binnedBLAS_" + name, fold, n, *args_g, z)
        assert same_state(z.cpu().numpy(), want, fold, comps=2), (name, fold)
    want = binned_zeros(fold, "s")
    wscl = port.sbcssq(fold, n, ptr(xc), 1, 0.0, ptr(want))
    z = dev(cuda, binned_zeros(fold, "s"))
    scl = rb.call("binnedBLAS_sbcssq", fold, n, XC, 1, 0.0, z)
    assert same_bits(z.cpu().numpy(), want) and scl == wscl


def test_launch_shapes_and_special_values(cuda, rb, port):
    """The run-time fold kernels give the same bits under every launch shape, and classify
    Inf / NaN as the reference does."""
    fold = 16
    n = (1 << 20) + 77
    x, y = gen("loguniform", n, 5), gen("illcond", n, 6)
    X, Y = dev(cuda, x), dev(cuda, y)
    want = binned_zeros(fold)
    port.dbddot(fold, n, ptr(x), 1, ptr(y), 1, ptr(want))
    try:
        for cps, thr in ((1, 32), (2, 128), (4, 256), (16, 32), (3, 224)):
            rb.call("rb_set_launch_config", cps, thr)
            z = dev(cuda, binned_zeros(fold))
            rb.call("binnedBLAS_dbddot", fold, n, X, 1, Y, 1, z)
            assert same_bits(z.cpu().numpy(), want), (cps, thr)
    finally:
        rb.call("rb_set_launch_config", 0, 0)
    rng = np.random.default_rng(3)
    for _ in range(20):
        m = int(rng.integers(1, 5000))
        v = rng.uniform(-1, 1, m)
        for _ in range(int(rng.integers(1, 3))):
            v[int(rng.integers(0, m))] = rng.choice([np.inf, -np.inf, np.nan])
        assert same_value(rb.call("reproBLAS_rdsum", 20, m, dev(cuda, v), 1), port.rdsum(20, m, ptr(v), 1))


@pytest.mark.parametrize("fold", (9, 52))
def test_dgemv_dgemm(cuda, rb, port, fold):
    rng = np.random.default_rng(fold)
    M, N, K = 37, 53, 41
    for order in "rc":
        for ta in "nt":
            lda = N if order == "r" else M
            A = rng.uniform(-1, 1, M * N)
            lx, ly = (N, M) if ta == "n" else (M, N)
            x, y = rng.uniform(-1, 1, lx), rng.uniform(-1, 1, ly)
            want = y.copy()
            port.rdgemv(fold, order.encode(), ta.encode(), M, N, 1.5, ptr(A), lda, ptr(x), 1, 0.5,
                        ptr(want), 1)
            yd = dev(cuda, y)
            rb.call("reproBLAS_rdgemv", fold, order, ta, M, N, 1.5, dev(cuda, A), lda, dev(cuda, x), 1,
                    0.5, yd, 1)
            assert same_bits(yd.cpu().numpy(), want), ("gemv", order, ta)
            # binned form into non-empty states
            st = np.zeros(ly * 2 * fold)
            for i in range(ly):
                port.dbdconv(fold, float(rng.standard_normal()), ptr(st[i * 2 * fold:]))
            want = st.copy()
            port.dbdgemv(fold, order.encode(), ta.encode(), M, N, 1.5, ptr(A), lda, ptr(x), 1,
                         ptr(want), 1)
            sd = dev(cuda, st)
            rb.call("binnedBLAS_dbdgemv", fold, order, ta, M, N, 1.5, dev(cuda, A), lda,
                    dev(cuda, x), 1, sd, 1)
            assert same_bits(sd.cpu().numpy(), want), ("dbdgemv", order, ta)
            for tb in "nt":
                if order == "r":
                    lda, ldb, ldc = (K if ta == "n" else M), (N if tb == "n" else K), N
                else:
                    lda, ldb, ldc = (M if ta == "n" else K), (K if tb == "n" else N), M
                A = rng.uniform(-1, 1, M * K)
                B = rng.uniform(-1, 1, K * N)
                C = rng.uniform(-1, 1, M * N)
                want = C.copy()
                port.rdgemm(fold, order.encode(), ta.encode(), tb.encode(), M, N, K, 1.5, ptr(A),
                            lda, ptr(B), ldb, 0.5, ptr(want), ldc)
                got = C.copy()   # host operands
                rb.call("reproBLAS_rdgemm", fold, order, ta, tb, M, N, K, 1.5, A, lda, B, ldb, 0.5,
                        got, ldc)
                assert same_bits(got, want), ("gemm", order, ta, tb)


@pytest.mark.parametrize("t,fold", [("s", 9), ("s", 21), ("z", 9), ("z", 52), ("c", 21)])
def test_xgemv_xgemm(cuda, rb, port, t, fold):
    rng = np.random.default_rng(fold + ord(t))
    rt = XREAL[t]
    nc = comps(t)

    def mat(n):
        v = rng.uniform(-1, 1, n * nc).astype(rt)
        return v if t == "s" else v.view(np.complex128 if t == "z" else np.complex64)

    M, N, K = 29, 23, 31
    alpha, beta = (1.5, 0.5) if t == "s" else (complex(1.5, -0.25), complex(0.5, 0.25))
    for order in "rc":
        for ta in ("n", "t") + (("c",) if t != "s" else ()):
            if order == "c" and ta == "c":
                continue   # the reference's column-major A^H x differs (documented); covered elsewhere
            lda = N if order == "r" else M
            A = mat(M * N)
            lx, ly = (N, M) if ta == "n" else (M, N)
            x, y = mat(lx), mat(ly)
            want = y.copy()
            lib_gemv(port, t, fold, order, ta, M, N, alpha, A, lda, x, 1, beta, want, 1)
            yd = dev(cuda, real_view(t, y))
            rb_gemv(rb, t, fold, order, ta, M, N, alpha, dev(cuda, real_view(t, A)), lda,
                    dev(cuda, real_view(t, x)), 1, beta, yd, 1)
            assert same_bits(yd.cpu().numpy().view(y.dtype), want), ("gemv", t, order, ta)
        tbs = ("n", "t") + (("c",) if t != "s" else ())
        for ta in ("n", "t"):
            for tb in tbs:
                if order == "r":
                    lda, ldb, ldc = (K if ta == "n" else M), (N if tb == "n" else K), N
                else:
                    lda, ldb, ldc = (M if ta == "n" else K), (K if tb == "n" else N), M
                A, B, C = mat(M * K), mat(K * N), mat(M * N)
                al = alpha if (t == "s" or order == "r" or ta == "n") else complex(1.25, 1.25)
                want = C.copy()
                lib_gemm(port, t, fold, order, ta, tb, M, N, K, al, A, lda, B, ldb, beta, want, ldc)
                got = C.copy()
                rb_gemm(rb, t, fold, order, ta, tb, M, N, K, al, A, lda, B, ldb, beta, got, ldc)
                assert same_bits(got, want), ("gemm", t, order, ta, tb)
        # binned gemm into non-empty states
        A, B = mat(M * K), mat(K * N)
        st = np.zeros(M * N * state_len(t, fold), rt)
        for i in range(M * N):
            if t == "s":
                port.sbsconv(fold, float(np.float32(rng.standard_normal())), st[i * state_len(t, fold):].ctypes.data)
            else:
                v = rng.standard_normal(2).astype(rt)
                getattr(port, t + "b" + t + "conv")(fold, v.ctypes.data, st[i * state_len(t, fold):].ctypes.data)
        want = st.copy()
        ld = (K, N, N) if order == "r" else (M, K, M)
        lib_gemm(port, t, fold, order, "n", "n", M, N, K, alpha, A, ld[0], B, ld[1], 0.0, want, ld[2],
                 binned=True)
        got = st.copy()
        rb_gemm(rb, t, fold, order, "n", "n", M, N, K, alpha, A, ld[0], B, ld[1], 0.0, got, ld[2],
                binned=True)
        assert same_bits(got, want), ("binned gemm", t, order)


@pytest.mark.parametrize("kind,fold", [("d", 16), ("d", 52), ("z", 52), ("s", 21), ("c", 9),
                                       ("dsq", 52), ("ssq", 21)])
def test_state_merges(cuda, rb, port, kind, fold):
    """rb_*_states at high folds equal the oracle's merges of the same states."""
    rng = np.random.default_rng(fold)
    count = 37
    base = {"d": "d", "dsq": "d", "z": "z", "s": "s", "ssq": "s", "c": "c"}[kind]
    dt = np.float64 if base in "dz" else np.float32
    n = 3001
    states = []
    scales = []
    for i in range(count):
        z = binned_zeros(fold, base)
        if base == "d":
            v = gen("loguniform", n, 100 + i)
            if kind == "dsq":
                scales.append(port.dbdssq(fold, n, ptr(v), 1, 0.0, ptr(z)))
            else:
                port.dbdsum(fold, n, ptr(v), 1, ptr(z))
        elif base == "s":
            v = gen("loguniform", n, 100 + i, np.float32)
            if kind == "ssq":
                scales.append(port.sbsssq(fold, n, ptr(v), 1, 0.0, ptr(z)))
            else:
                port.sbssum(fold, n, ptr(v), 1, ptr(z))
        elif base == "z":
            v = gen_complex("normal", n, 100 + i)
            port.zbzsum(fold, n, ptr(v), 1, ptr(z))
        else:
            v = gen_complex("normal", n, 100 + i, np.complex64)
            port.cbcsum(fold, n, ptr(v), 1, ptr(z))
        states.append(z)
    if kind in ("dsq", "ssq"):
        recs = [np.concatenate([np.array([s], dt), z]) for s, z in zip(scales, states)]
        want_s, want = dt(0), binned_zeros(fold, base)
        for s, z in zip(scales, states):
            f = port.dbdbaddsq if kind == "dsq" else port.sbsbaddsq
            want_s = f(fold, s, ptr(z), want_s, ptr(want))
        packed = np.concatenate(recs)
        out = dev(cuda, np.concatenate([np.zeros(1, dt), binned_zeros(fold, base)]))
        name = "rb_dbdbaddsq_states" if kind == "dsq" else "rb_sbsbaddsq_states"
        assert rb.call(name, fold, count, dev(cuda, packed), out) == 0
        got = out.cpu().numpy()
        assert got[0] == dt(want_s) and same_bits(got[1:], want)
        return
    want = binned_zeros(fold, base)
    merge = {"d": port.dbdbadd, "s": port.sbsbadd, "z": port.zbzbadd, "c": port.cbcbadd}[base]
    for z in states:
        merge(fold, ptr(z), ptr(want))
    out = dev(cuda, binned_zeros(fold, base))
    name = {"d": "rb_dbdbadd_states", "s": "rb_sbsbadd_states", "z": "rb_zbzbadd_states",
            "c": "rb_cbcbadd_states"}[base]
    assert rb.call(name, fold, count, dev(cuda, np.concatenate(states)), out) == 0
    assert same_bits(out.cpu().numpy(), want)


def test_manual_form_and_limits(cuda, rb, port):
    fold = 20
    n = 9999
    x, y = gen("normal", n, 1), gen("loguniform", n, 2)
    want = binned_zeros(fold)
    port.dbddot(fold, n, ptr(x), 1, ptr(y), 1, ptr(want))
    # binnedBLAS_dmddot with primaries and carries in separate strided device arrays
    pri = dev(cuda, np.zeros(3 * fold))
    car = dev(cuda, np.zeros(2 * fold))
    rb.call("binnedBLAS_dmddot", fold, n, dev(cuda, x), 1, dev(cuda, y), 1, pri, 3, car, 2)
    got = np.concatenate([pri.cpu().numpy()[::3], car.cpu().numpy()[::2]])
    assert same_bits(got, want)
    # folds past binned_DBMAXFOLD / binned_SBMAXFOLD are rejected
    lib = rb.lib
    lib.rb_clear_error()
    v = lib.reproBLAS_rddot(53, n, dev(cuda, x).data_ptr(), 1, dev(cuda, y).data_ptr(), 1)
    assert math.isnan(v) and lib.rb_get_last_error() == 1
    lib.rb_clear_error()
    xf = dev(cuda, x.astype(np.float32))
    v = lib.reproBLAS_rssum(22, n, xf.data_ptr(), 1)
    assert math.isnan(v) and lib.rb_get_last_error() == 1
    lib.rb_clear_error()
    assert not math.isnan(lib.reproBLAS_rssum(21, n, xf.data_ptr(), 1))
