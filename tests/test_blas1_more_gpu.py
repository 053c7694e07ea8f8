"""GPU parity of the absolute sums (dasum, sasum, dzasum, scasum) and of the zdotu, cdotc and
cdotu dots through the C ABI: bit-identical to the reference fixtures and to the oracle
restatement, for binned (accumulating) and value-returning forms, every fold, strides,
offsets, host pointers and non-finite values.

The float complex dots are compared with the canonical binned state (the reference's own
state whenever its calls stay within the FP32 endurance; tests/golden/make_golden.py)."""
import numpy as np
import pytest

from _cmp import from_hex, same_state, same_value
from _data import gen, gen_complex
from _ffi import binned_zeros, ptr

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def as_real(a):
    return a.view(np.float64 if a.dtype == np.complex128 else np.float32)


BINNED = [("dbdasum", "d", 1, 1), ("sbsasum", "s", 1, 1), ("dbzasum", "d", 1, 1),
          ("sbcasum", "s", 1, 1), ("zbzdotu", "z", 2, 2), ("cbcdotc", "c", 2, 2),
          ("cbcdotu", "c", 2, 2)]


def test_golden_asum_dots(cuda, rb, golden):
    bad = []
    for c in golden["blas1_more"]:
        dist, n, fold = c["dist"], c["n"], c["fold"]
        x, xf = gen(dist, n, 11), gen(dist, n, 11, np.float32)
        xz, yz = gen_complex(dist, n, 11), gen_complex(dist, n, 12)
        xc, yc = gen_complex(dist, n, 11, np.complex64), gen_complex(dist, n, 12, np.complex64)
        ins = {"dbdasum": (x,), "sbsasum": (xf,), "dbzasum": (xz,), "sbcasum": (xc,),
               "zbzdotu": (xz, yz), "cbcdotc": (xc, yc), "cbcdotu": (xc, yc)}
        for name, kind, nin, comps in BINNED:
            z = dev(cuda, binned_zeros(fold, kind))
            args = []
            for a in ins[name]:
                args += [dev(cuda, as_real(a) if a.dtype.kind == "c" else a), 1]
            rb.call("binnedBLAS_" + name, fold, n, *args, z)
            dt = np.float64 if kind in "dz" else np.float32
            if not same_state(host(z), from_hex(c[name], dt), fold, comps):
                bad.append((name, dist, n, fold))
        vals = {"rdasum": (rb.call("reproBLAS_rdasum", fold, n, dev(cuda, x), 1), np.float64),
                "rsasum": (rb.call("reproBLAS_rsasum", fold, n, dev(cuda, xf), 1), np.float32),
                "rdzasum": (rb.call("reproBLAS_rdzasum", fold, n, dev(cuda, as_real(xz)), 1), np.float64),
                "rscasum": (rb.call("reproBLAS_rscasum", fold, n, dev(cuda, as_real(xc)), 1), np.float32)}
        for k, (v, dt) in vals.items():
            if not same_value(np.asarray(v, dt), from_hex(c[k], dt)[0]):
                bad.append((k, dist, n, fold))
        for k, fn, dt, a, b in [("rzdotu", "reproBLAS_rzdotu_sub", np.float64, xz, yz),
                                ("rdotc", "reproBLAS_rcdotc_sub", np.float32, xc, yc),
                                ("rdotu", "reproBLAS_rcdotu_sub", np.float32, xc, yc)]:
            o = dev(cuda, np.zeros(2, dt))
            rb.call(fn, fold, n, dev(cuda, as_real(a)), 1, dev(cuda, as_real(b)), 1, o)
            if not same_value(host(o), from_hex(c[k], dt)):
                bad.append((k, dist, n, fold))
    assert not bad, bad[:10]


@pytest.mark.parametrize("fold", [2, 3, 5, 8])
def test_asum_dots_vs_oracle(cuda, rb, port, fold):
    """Edge sizes around the warp tiles, strides 1/2/3, odd element offsets, accumulation
    into a non-empty state, device and host pointers."""
    rng = np.random.default_rng(40 + fold)
    for n in [0, 1, 5, 63, 64, 65, 255, 256, 257, 1023, 4097, 70001]:
        inc = int(rng.integers(1, 4))
        off = int(rng.integers(0, 2))
        dist = ["uniform", "normal", "loguniform", "illcond"][n % 4]
        m = n * inc + 2
        bx = gen(dist, m, n + 1)
        bf = gen(dist, m, n + 1, np.float32)
        bz, byz = gen_complex(dist, m, n + 2), gen_complex(dist, m, n + 3)
        bc, byc = gen_complex(dist, m, n + 2, np.complex64), gen_complex(dist, m, n + 3, np.complex64)
        seeds = {"d": gen("normal", 3, n), "s": gen("normal", 3, n, np.float32)}
        ins = {"dbdasum": (bx,), "sbsasum": (bf,), "dbzasum": (bz,), "sbcasum": (bc,),
               "zbzdotu": (bz, byz), "cbcdotc": (bc, byc), "cbcdotu": (bc, byc)}
        for name, kind, nin, comps in BINNED:
            want = binned_zeros(fold, kind)
            if kind in "ds":
                # start from a non-empty state
                (port.dbdsum if kind == "d" else port.sbssum)(fold, 3, ptr(seeds[kind]), 1, ptr(want))
            got0 = want.copy()
            pargs, dargs, hargs = [], [], []
            for a in ins[name]:
                pargs += [ptr(a[off:]), inc]
                r = as_real(a) if a.dtype.kind == "c" else a
                step = 2 if a.dtype.kind == "c" else 1
                dargs += [dev(cuda, r)[step * off:], inc]
                hargs += [np.ascontiguousarray(r[step * off:]), inc]
            getattr(port, name)(fold, n, *pargs, ptr(want))
            z = dev(cuda, got0)
            rb.call("binnedBLAS_" + name, fold, n, *dargs, z)
            assert same_state(host(z), want, fold, comps), (name, n, inc, off, "device")
            zh = got0.copy()
            rb.call("binnedBLAS_" + name, fold, n, *hargs, zh)
            assert same_state(zh, want, fold, comps), (name, n, inc, off, "host")
        assert same_value(rb.call("reproBLAS_rdasum", fold, n, dev(cuda, bx)[off:], inc),
                          port.rdasum(fold, n, ptr(bx[off:]), inc))
        assert same_value(np.float32(rb.call("reproBLAS_rsasum", fold, n, dev(cuda, bf)[off:], inc)),
                          np.float32(port.rsasum(fold, n, ptr(bf[off:]), inc)))
        assert same_value(rb.call("reproBLAS_rdzasum", fold, n, dev(cuda, as_real(bz))[2 * off:], inc),
                          port.rdzasum(fold, n, ptr(bz[off:]), inc))
        assert same_value(np.float32(rb.call("reproBLAS_rscasum", fold, n, dev(cuda, as_real(bc))[2 * off:], inc)),
                          np.float32(port.rscasum(fold, n, ptr(bc[off:]), inc)))
        for fn, pfn, dt, a, b in [("reproBLAS_rzdotu_sub", port.rzdotu_sub, np.float64, bz, byz),
                                  ("reproBLAS_rcdotc_sub", port.rcdotc_sub, np.float32, bc, byc),
                                  ("reproBLAS_rcdotu_sub", port.rcdotu_sub, np.float32, bc, byc)]:
            want = np.zeros(2, dt)
            pfn(fold, n, ptr(a[off:]), inc, ptr(b[off:]), inc, ptr(want))
            o = dev(cuda, np.zeros(2, dt))
            rb.call(fn, fold, n, dev(cuda, as_real(a))[2 * off:], inc, dev(cuda, as_real(b))[2 * off:], inc, o)
            assert same_value(host(o), want), (fn, n, inc, off)


def test_asum_dots_special_values(cuda, rb, port):
    rng = np.random.default_rng(17)
    for trial in range(60):
        n = int(rng.integers(1, 3000))
        x = rng.uniform(-1, 1, n)
        for _ in range(int(rng.integers(1, 4))):
            x[int(rng.integers(0, n))] = rng.choice([np.inf, -np.inf, np.nan])
        assert same_value(rb.call("reproBLAS_rdasum", 3, n, dev(cuda, x), 1), port.rdasum(3, n, ptr(x), 1))
        xz = np.empty(n, np.complex128)
        xz.real = x
        xz.imag = np.roll(x, 5)
        yz = np.empty(n, np.complex128)
        yz.real = rng.uniform(-1, 1, n)
        yz.imag = rng.uniform(-1, 1, n)
        assert same_value(rb.call("reproBLAS_rdzasum", 3, n, dev(cuda, as_real(xz)), 1),
                          port.rdzasum(3, n, ptr(xz), 1))
        want = np.zeros(2)
        port.rzdotu_sub(3, n, ptr(xz), 1, ptr(yz), 1, ptr(want))
        o = dev(cuda, np.zeros(2))
        rb.call("reproBLAS_rzdotu_sub", 3, n, dev(cuda, as_real(xz)), 1, dev(cuda, as_real(yz)), 1, o)
        assert same_value(host(o), want)
        xc, yc = xz.astype(np.complex64), yz.astype(np.complex64)
        for fn, pfn in (("reproBLAS_rcdotc_sub", port.rcdotc_sub), ("reproBLAS_rcdotu_sub", port.rcdotu_sub)):
            want = np.zeros(2, np.float32)
            pfn(3, n, ptr(xc), 1, ptr(yc), 1, ptr(want))
            o = dev(cuda, np.zeros(2, np.float32))
            rb.call(fn, 3, n, dev(cuda, as_real(xc)), 1, dev(cuda, as_real(yc)), 1, o)
            assert same_value(host(o), want), fn


def test_golden_ssq_more(cuda, rb, golden):
    """FP32 and complex scaled sums of squares and the 2-norms built on them."""
    bad = []
    for c in golden["blas1_more"]:
        dist, n, fold = c["dist"], c["n"], c["fold"]
        xf = gen(dist, n, 11, np.float32)
        xz, xc = gen_complex(dist, n, 11), gen_complex(dist, n, 11, np.complex64)
        for name, kind, x, dt in [("sbsssq", "s", xf, np.float32), ("dbzssq", "d", as_real(xz), np.float64),
                                  ("sbcssq", "s", as_real(xc), np.float32)]:
            z = dev(cuda, binned_zeros(fold, kind))
            sc = rb.call("binnedBLAS_" + name, fold, n, dev(cuda, x), 1, 0.0, z)
            if not same_state(host(z), from_hex(c[name], dt), fold):
                bad.append((name, dist, n, fold))
            if not same_value(np.asarray(sc, dt), from_hex(c[name + "_scale"], dt)[0]):
                bad.append((name + "_scale", dist, n, fold))
        for name, x, dt in [("rsnrm2", xf, np.float32), ("rdznrm2", as_real(xz), np.float64),
                            ("rscnrm2", as_real(xc), np.float32)]:
            v = rb.call("reproBLAS_" + name, fold, n, dev(cuda, x), 1)
            if not same_value(np.asarray(v, dt), from_hex(c[name], dt)[0]):
                bad.append((name, dist, n, fold))
    assert not bad, bad[:10]


@pytest.mark.parametrize("fold", [2, 3, 6])
def test_ssq_more_vs_oracle(cuda, rb, port, fold):
    """Scaled sums of squares into scaled non-empty states, strides, offsets, device and host
    pointers; and the 2-norms."""
    rng = np.random.default_rng(70 + fold)
    for n in [0, 1, 5, 64, 257, 1023, 4097, 70001]:
        inc = int(rng.integers(1, 4))
        off = int(rng.integers(0, 2))
        dist = ["uniform", "normal", "loguniform", "illcond", "huge", "tiny"][n % 6]
        m = n * inc + 2
        bf = gen(dist, m, n + 1, np.float32)
        bz = gen_complex(dist, m, n + 2)
        bc = gen_complex(dist, m, n + 2, np.complex64)
        pre = gen("normal", 4, n)
        for name, kind, arr, seedf in [("sbsssq", "s", bf, "sbsssq"), ("dbzssq", "d", bz, "dbdssq"),
                                       ("sbcssq", "s", bc, "sbsssq")]:
            want = binned_zeros(fold, kind)
            p0 = pre.astype(np.float32) if kind == "s" else pre
            s0 = getattr(port, seedf)(fold, 4, ptr(p0), 1, 0.0, ptr(want))
            start = want.copy()
            sw = getattr(port, name)(fold, n, ptr(arr[off:]), inc, s0, ptr(want))
            r = as_real(arr) if arr.dtype.kind == "c" else arr
            step = 2 if arr.dtype.kind == "c" else 1
            z = dev(cuda, start)
            sg = rb.call("binnedBLAS_" + name, fold, n, dev(cuda, r)[step * off:], inc, s0, z)
            assert same_state(host(z), want, fold) and same_value(sg, sw), (name, n, inc, off, "device")
            zh = start.copy()
            sh = rb.call("binnedBLAS_" + name, fold, n, np.ascontiguousarray(r[step * off:]), inc, s0, zh)
            assert same_state(zh, want, fold) and same_value(sh, sw), (name, n, inc, off, "host")
        for name, arr in [("rsnrm2", bf), ("rdznrm2", bz), ("rscnrm2", bc)]:
            r = as_real(arr) if arr.dtype.kind == "c" else arr
            step = 2 if arr.dtype.kind == "c" else 1
            got = rb.call("reproBLAS_" + name, fold, n, dev(cuda, r)[step * off:], inc)
            want = getattr(port, name)(fold, n, ptr(arr[off:]), inc)
            assert same_value(got, want), (name, n, inc, off)


def test_ssq_more_special_values(cuda, rb, port):
    rng = np.random.default_rng(23)
    for trial in range(60):
        n = int(rng.integers(1, 3000))
        x = rng.uniform(-1, 1, n)
        for _ in range(int(rng.integers(1, 4))):
            x[int(rng.integers(0, n))] = rng.choice([np.inf, -np.inf, np.nan])
        xf = x.astype(np.float32)
        assert same_value(np.float32(rb.call("reproBLAS_rsnrm2", 3, n, dev(cuda, xf), 1)),
                          np.float32(port.rsnrm2(3, n, ptr(xf), 1)))
        xz = np.empty(n, np.complex128)
        xz.real = x
        xz.imag = np.roll(x, 7)
        assert same_value(rb.call("reproBLAS_rdznrm2", 3, n, dev(cuda, as_real(xz)), 1),
                          port.rdznrm2(3, n, ptr(xz), 1))
        xc = xz.astype(np.complex64)
        assert same_value(np.float32(rb.call("reproBLAS_rscnrm2", 3, n, dev(cuda, as_real(xc)), 1)),
                          np.float32(port.rscnrm2(3, n, ptr(xc), 1)))


def test_amax_family(cuda, rb, port):
    """binnedBLAS_[dszc]amax and amaxm: device and host pointers, strides, infinities and
    NaN (NaN anywhere gives NaN, as in the oracle)."""
    rng = np.random.default_rng(31)
    for trial in range(40):
        n = int(rng.integers(0, 70000)) if trial % 4 else int(rng.integers(0, 70))
        inc = int(rng.integers(1, 4))
        dist = ["uniform", "normal", "loguniform", "illcond"][trial % 4]
        x, y = gen(dist, n * inc + 1, trial), gen(dist, n * inc + 1, trial + 1)
        if n and trial % 3 == 0:
            x[int(rng.integers(0, n)) * inc] = [np.inf, -np.inf, np.nan][trial % 9 // 3]
        xf, yf = x.astype(np.float32), y.astype(np.float32)
        xz, yz = gen_complex(dist, n * inc + 1, trial), gen_complex(dist, n * inc + 1, trial + 2)
        if n and trial % 3 == 1:
            xz[int(rng.integers(0, n)) * inc] = complex(np.nan, 1.0)
        xc, yc = xz.astype(np.complex64), yz.astype(np.complex64)
        for src in ("dev", "host"):
            d = (lambda a: dev(cuda, as_real(a) if a.dtype.kind == "c" else a)) if src == "dev" else \
                (lambda a: np.ascontiguousarray(as_real(a) if a.dtype.kind == "c" else a))
            assert same_value(rb.call("binnedBLAS_damax", n, d(x), inc), port.damax(n, ptr(x), inc))
            assert same_value(np.float32(rb.call("binnedBLAS_samax", n, d(xf), inc)),
                              np.float32(port.samax(n, ptr(xf), inc)))
            assert same_value(rb.call("binnedBLAS_damaxm", n, d(x), inc, d(y), inc),
                              port.damaxm(n, ptr(x), inc, ptr(y), inc))
            assert same_value(np.float32(rb.call("binnedBLAS_samaxm", n, d(xf), inc, d(yf), inc)),
                              np.float32(port.samaxm(n, ptr(xf), inc, ptr(yf), inc)))
            for name, a, b, dt in [("zamax_sub", xz, None, np.float64), ("camax_sub", xc, None, np.float32),
                                   ("zamaxm_sub", xz, yz, np.float64), ("camaxm_sub", xc, yc, np.float32)]:
                want = np.zeros(2, dt)
                pargs = [n, ptr(a), inc] + ([ptr(b), inc] if b is not None else [])
                getattr(port, name)(*pargs, ptr(want))
                got = np.zeros(2, dt)
                gargs = [n, d(a), inc] + ([d(b), inc] if b is not None else [])
                out = dev(cuda, got) if src == "dev" else got
                rb.call("binnedBLAS_" + name, *gargs, out)
                got = host(out) if src == "dev" else got
                assert same_value(got, want), (name, n, inc, src)
