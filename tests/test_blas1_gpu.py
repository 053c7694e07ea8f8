"""GPU parity of the BLAS1 reductions through the C ABI: bit-identical to the reference
(committed fixtures generated by the compiled reference) and to the oracle restatement,
for device and host pointers, every fold 2..8, edge sizes, strides, misalignment,
special values, accumulate-into-state, 8 launch shapes and input permutations."""
import numpy as np
import pytest

from _cmp import from_hex, same_bits, same_state, same_value
from _data import gen, gen_complex
from _ffi import binned_zeros, ptr

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def run_all_device(cuda, rb, fold, x, y, xf, yf, xz, yz, xc):
    """Every BLAS1 routine on device inputs; returns a dict of numpy results."""
    n = len(x)
    out = {}
    X, Y, XF, YF = dev(cuda, x), dev(cuda, y), dev(cuda, xf), dev(cuda, yf)
    XZ, YZ, XC = dev(cuda, xz), dev(cuda, yz), dev(cuda, xc)
    z = dev(cuda, binned_zeros(fold)); rb.call("binnedBLAS_dbdsum", fold, n, X, 1, z); out["dbdsum"] = host(z)
    out["rdsum"] = rb.call("reproBLAS_rdsum", fold, n, X, 1)
    z = dev(cuda, binned_zeros(fold)); rb.call("binnedBLAS_dbddot", fold, n, X, 1, Y, 1, z); out["dbddot"] = host(z)
    out["rddot"] = rb.call("reproBLAS_rddot", fold, n, X, 1, Y, 1)
    z = dev(cuda, binned_zeros(fold)); s = rb.call("binnedBLAS_dbdssq", fold, n, X, 1, 0.0, z)
    out["dbdssq"] = host(z); out["dbdssq_scale"] = s
    out["rdnrm2"] = rb.call("reproBLAS_rdnrm2", fold, n, X, 1)
    z = dev(cuda, binned_zeros(fold, "s")); rb.call("binnedBLAS_sbssum", fold, n, XF, 1, z); out["sbssum"] = host(z)
    out["rssum"] = rb.call("reproBLAS_rssum", fold, n, XF, 1)
    z = dev(cuda, binned_zeros(fold, "s")); rb.call("binnedBLAS_sbsdot", fold, n, XF, 1, YF, 1, z); out["sbsdot"] = host(z)
    out["rsdot"] = rb.call("reproBLAS_rsdot", fold, n, XF, 1, YF, 1)
    z = dev(cuda, binned_zeros(fold, "z")); rb.call("binnedBLAS_zbzsum", fold, n, XZ, 1, z); out["zbzsum"] = host(z)
    o = dev(cuda, np.zeros(2)); rb.call("reproBLAS_rzsum_sub", fold, n, XZ, 1, o); out["rzsum"] = host(o)
    z = dev(cuda, binned_zeros(fold, "z")); rb.call("binnedBLAS_zbzdotc", fold, n, XZ, 1, YZ, 1, z); out["zbzdotc"] = host(z)
    o = dev(cuda, np.zeros(2)); rb.call("reproBLAS_rzdotc_sub", fold, n, XZ, 1, YZ, 1, o); out["rzdotc"] = host(o)
    z = dev(cuda, binned_zeros(fold, "c")); rb.call("binnedBLAS_cbcsum", fold, n, XC, 1, z); out["cbcsum"] = host(z)
    o = dev(cuda, np.zeros(2, np.float32)); rb.call("reproBLAS_rcsum_sub", fold, n, XC, 1, o); out["rcsum"] = host(o)
    return out


def check_against(c, out, fold):
    bad = []
    for k, dt, comps in [("dbdsum", np.float64, 1), ("dbddot", np.float64, 1), ("dbdssq", np.float64, 1),
                         ("sbssum", np.float32, 1), ("sbsdot", np.float32, 1), ("zbzsum", np.float64, 2),
                         ("zbzdotc", np.float64, 2), ("cbcsum", np.float32, 2)]:
        if not same_state(out[k], from_hex(c[k], dt), fold, comps):
            bad.append(k)
    for k, dt in [("rdsum", np.float64), ("rddot", np.float64), ("dbdssq_scale", np.float64),
                  ("rdnrm2", np.float64), ("rssum", np.float32), ("rsdot", np.float32),
                  ("rzsum", np.float64), ("rzdotc", np.float64), ("rcsum", np.float32)]:
        ref = from_hex(c[k], dt)
        got = np.asarray(out[k], dtype=dt).reshape(ref.shape)
        if not same_value(got, ref):
            bad.append(k)
    return bad


def test_golden_blas1_device(cuda, rb, golden):
    bad = []
    for c in golden["blas1"]:
        dist, n, fold = c["dist"], c["n"], c["fold"]
        out = run_all_device(cuda, rb, fold, gen(dist, n, 11), gen(dist, n, 12),
                             gen(dist, n, 11, np.float32), gen(dist, n, 12, np.float32),
                             gen_complex(dist, n, 11), gen_complex(dist, n, 12),
                             gen_complex(dist, n, 11, np.complex64))
        b = check_against(c, out, fold)
        if b:
            bad.append((dist, n, fold, b))
    assert not bad, bad[:8]


def test_golden_blas1_host_pointers(cuda, rb, golden):
    """The same calls with host (pageable) inputs and host accumulators."""
    bad = []
    for c in golden["blas1"][::7]:
        dist, n, fold = c["dist"], c["n"], c["fold"]
        x, y = gen(dist, n, 11), gen(dist, n, 12)
        z = binned_zeros(fold); rb.call("binnedBLAS_dbddot", fold, n, x, 1, y, 1, z)
        if not same_state(z, from_hex(c["dbddot"], np.float64), fold): bad.append(("dbddot", dist, n, fold))
        if not same_value(rb.call("reproBLAS_rddot", fold, n, x, 1, y, 1), from_hex(c["rddot"], np.float64)[0]):
            bad.append(("rddot", dist, n, fold))
        xz = gen_complex(dist, n, 11)
        o = np.zeros(2); rb.call("reproBLAS_rzsum_sub", fold, n, xz, 1, o)
        if not same_value(o, from_hex(c["rzsum"], np.float64)): bad.append(("rzsum", dist, n, fold))
        xf = gen(dist, n, 11, np.float32)
        if not same_value(np.float32(rb.call("reproBLAS_rssum", fold, n, xf, 1)), from_hex(c["rssum"], np.float32)[0]):
            bad.append(("rssum", dist, n, fold))
    assert not bad, bad


def test_pinned_host_and_staging_chunks(cuda, rb, port):
    """Host inputs longer than one 32 MiB staging chunk (5 chunks), pinned and pageable."""
    n = (5 << 22) + 12345
    x = gen("loguniform", n, 3)
    y = gen("normal", n, 4)
    want = binned_zeros(3); port.dbddot(3, n, ptr(x), 1, ptr(y), 1, ptr(want))
    for pinned in (False, True):
        if pinned:
            xp = cuda.from_numpy(x).pin_memory(); yp = cuda.from_numpy(y).pin_memory()
        else:
            xp, yp = x, y
        z = binned_zeros(3)
        rb.call("binnedBLAS_dbddot", 3, n, xp, 1, yp, 1, z)
        assert same_bits(z, want), pinned
        assert same_value(rb.call("reproBLAS_rddot", 3, n, xp, 1, yp, 1), port.rddot(3, n, ptr(x), 1, ptr(y), 1))


def test_dsum_config_permutations(cuda, rb, golden):
    """reproBLAS_dsum, fold 3, N = 2^20 (sine and uniform(-1,1), seed 0): bit-identical to
    the reference under the permutations of verify_daugsum.c:155-215."""
    for c in golden["dsum_config"]:
        x = gen(c["dist"], c["n"], c["seed"])
        want = from_hex(c["dbdsum"], np.float64)
        rng = np.random.default_rng(1)
        perms = [x, x[::-1], np.sort(x), np.sort(x)[::-1], x[np.argsort(np.abs(x))],
                 x[np.argsort(-np.abs(x))], x[rng.permutation(len(x))], x[rng.permutation(len(x))],
                 x[rng.permutation(len(x))]]
        for p in perms:
            z = dev(cuda, binned_zeros(3))
            rb.call("binnedBLAS_dbdsum", 3, len(p), dev(cuda, p), 1, z)
            assert same_bits(host(z), want)
            assert same_value(rb.call("reproBLAS_dsum", len(p), dev(cuda, p), 1),
                              from_hex(c["rdsum"], np.float64)[0])


LAUNCH_CONFIGS = [(1, 32), (1, 256), (2, 64), (2, 128), (4, 256), (8, 96), (16, 32), (3, 224)]


@pytest.mark.parametrize("dist", ["loguniform", "normal", "illcond"])
def test_launch_config_invariance(cuda, rb, port, dist):
    n = (1 << 20) + 77
    x, y = gen(dist, n, 5), gen(dist, n, 6)
    xz, yz = gen_complex(dist, n, 5), gen_complex(dist, n, 6)
    xf = gen(dist, n, 5, np.float32)
    X, Y, XZ, YZ, XF = dev(cuda, x), dev(cuda, y), dev(cuda, xz), dev(cuda, yz), dev(cuda, xf)
    want_dot = binned_zeros(3); port.dbddot(3, n, ptr(x), 1, ptr(y), 1, ptr(want_dot))
    want_ssq = binned_zeros(3); want_scl = port.dbdssq(3, n, ptr(x), 1, 0.0, ptr(want_ssq))
    want_zd = binned_zeros(3, "z"); port.zbzdotc(3, n, ptr(xz), 1, ptr(yz), 1, ptr(want_zd))
    want_s = binned_zeros(3, "s"); port.sbssum(3, n, ptr(xf), 1, ptr(want_s))
    try:
        for cps, thr in LAUNCH_CONFIGS:
            rb.call("rb_set_launch_config", cps, thr)
            z = dev(cuda, binned_zeros(3)); rb.call("binnedBLAS_dbddot", 3, n, X, 1, Y, 1, z)
            assert same_bits(host(z), want_dot), (cps, thr)
            z = dev(cuda, binned_zeros(3)); s = rb.call("binnedBLAS_dbdssq", 3, n, X, 1, 0.0, z)
            assert same_bits(host(z), want_ssq) and s == want_scl, (cps, thr)
            z = dev(cuda, binned_zeros(3, "z")); rb.call("binnedBLAS_zbzdotc", 3, n, XZ, 1, YZ, 1, z)
            assert same_bits(host(z), want_zd), (cps, thr)
            z = dev(cuda, binned_zeros(3, "s")); rb.call("binnedBLAS_sbssum", 3, n, XF, 1, z)
            assert same_bits(host(z), want_s), (cps, thr)
    finally:
        rb.call("rb_set_launch_config", 0, 0)


@pytest.mark.parametrize("fold", [2, 3, 4, 5, 6, 7, 8])
def test_edge_sizes_strides_alignment(cuda, rb, port, fold):
    sizes = [0, 1, 2, 31, 33, 255, 256, 257, 1023, 1025, 2047, 2049, 4099, 65537]
    for n in sizes:
        for inc in (1, 2):
            for off in (0, 1):
                base_x = gen("loguniform", n * inc + 2, n + 1)
                base_y = gen("normal", n * inc + 2, n + 2)
                X, Y = dev(cuda, base_x), dev(cuda, base_y)
                xs = base_x[off:]
                ys = base_y[off:]
                want = binned_zeros(fold); port.dbddot(fold, n, ptr(xs), inc, ptr(ys), inc, ptr(want))
                z = dev(cuda, binned_zeros(fold))
                rb.call("binnedBLAS_dbddot", fold, n, X[off:], inc, Y[off:], inc, z)
                assert same_bits(host(z), want), (n, inc, off)
                want = binned_zeros(fold); port.dbdsum(fold, n, ptr(xs), inc, ptr(want))
                z = dev(cuda, binned_zeros(fold))
                rb.call("binnedBLAS_dbdsum", fold, n, X[off:], inc, z)
                assert same_bits(host(z), want), (n, inc, off)
                xf = base_x.astype(np.float32)
                want = binned_zeros(fold, "s"); port.sbsdot(fold, n, ptr(xf[off:]), inc, ptr(xf[off:]), inc, ptr(want))
                XF = dev(cuda, xf)
                z = dev(cuda, binned_zeros(fold, "s"))
                rb.call("binnedBLAS_sbsdot", fold, n, XF[off:], inc, XF[off:], inc, z)
                assert same_state(host(z), want, fold), (n, inc, off)


@pytest.mark.parametrize("fold", [2, 3, 5, 8])
def test_complex_edge_sizes_strides_alignment(cuda, rb, port, fold):
    """Complex sums and dots around the vector body's warp tiles (128 and 256 complex
    elements), with unit and double strides, and float complex at an odd element offset
    (an 8-byte head before the 16-byte aligned body)."""
    sizes = [0, 1, 2, 63, 64, 65, 127, 128, 129, 255, 256, 257, 4095, 4097, 65537]
    for n in sizes:
        for inc in (1, 2):
            for off in (0, 1):
                bx = gen_complex("loguniform", n * inc + 2, n + 3)
                by = gen_complex("normal", n * inc + 2, n + 4)
                X, Y = dev(cuda, bx.view(np.float64)), dev(cuda, by.view(np.float64))
                xs, ys = bx[off:], by[off:]
                want = binned_zeros(fold, "z"); port.zbzsum(fold, n, ptr(xs), inc, ptr(want))
                z = dev(cuda, binned_zeros(fold, "z"))
                rb.call("binnedBLAS_zbzsum", fold, n, X[2 * off:], inc, z)
                assert same_bits(host(z), want), ("zsum", n, inc, off)
                want = binned_zeros(fold, "z")
                port.zbzdotc(fold, n, ptr(xs), inc, ptr(ys), inc, ptr(want))
                z = dev(cuda, binned_zeros(fold, "z"))
                rb.call("binnedBLAS_zbzdotc", fold, n, X[2 * off:], inc, Y[2 * off:], inc, z)
                assert same_bits(host(z), want), ("zdotc", n, inc, off)
                bc = bx.astype(np.complex64)
                want = binned_zeros(fold, "c"); port.cbcsum(fold, n, ptr(bc[off:]), inc, ptr(want))
                XC = dev(cuda, bc.view(np.float32))
                z = dev(cuda, binned_zeros(fold, "c"))
                rb.call("binnedBLAS_cbcsum", fold, n, XC[2 * off:], inc, z)
                assert same_state(host(z), want, fold, comps=2), ("csum", n, inc, off)


def test_accumulate_resume(cuda, rb, port):
    """binnedBLAS_* add into the caller's state: two halves equal the whole."""
    n = 300001
    x, y = gen("loguniform", n, 8), gen("loguniform", n, 9)
    X, Y = dev(cuda, x), dev(cuda, y)
    whole = binned_zeros(3); port.dbddot(3, n, ptr(x), 1, ptr(y), 1, ptr(whole))
    for k in (0, 1, 1000, 150000, n):
        z = dev(cuda, binned_zeros(3))
        rb.call("binnedBLAS_dbddot", 3, k, X, 1, Y, 1, z)
        rb.call("binnedBLAS_dbddot", 3, n - k, X[k:], 1, Y[k:], 1, z)
        assert same_bits(host(z), whole), k
    # host accumulator carried across calls
    z = binned_zeros(3)
    rb.call("binnedBLAS_dbddot", 3, 1234, X, 1, Y, 1, z)
    rb.call("binnedBLAS_dbddot", 3, n - 1234, X[1234:], 1, Y[1234:], 1, z)
    assert same_bits(z, whole)
    # sum of squares carried with its scale
    a = binned_zeros(3); sa = port.dbdssq(3, n, ptr(x), 1, 0.0, ptr(a))
    z = dev(cuda, binned_zeros(3))
    s = rb.call("binnedBLAS_dbdssq", 3, 5000, X, 1, 0.0, z)
    s = rb.call("binnedBLAS_dbdssq", 3, n - 5000, X[5000:], 1, s, z)
    assert same_bits(host(z), a) and s == sa


def test_special_values(cuda, rb, port, golden):
    for c in golden["special"]:
        x = from_hex(c["x"], np.float64)
        X = dev(cuda, x)
        ones = dev(cuda, np.ones_like(x))
        n = len(x)
        assert same_value(rb.call("reproBLAS_rdsum", 3, n, X, 1), from_hex(c["rdsum"], np.float64)[0])
        assert same_value(rb.call("reproBLAS_rddot", 3, n, X, 1, ones, 1), from_hex(c["rddot"], np.float64)[0])
        assert same_value(rb.call("reproBLAS_rdnrm2", 3, n, X, 1), from_hex(c["rdnrm2"], np.float64)[0])
    rng = np.random.default_rng(17)
    for trial in range(60):
        n = int(rng.integers(1, 20000))
        x = rng.uniform(-1, 1, n)
        for _ in range(int(rng.integers(1, 4))):
            x[int(rng.integers(0, n))] = rng.choice([np.inf, -np.inf, np.nan])
        y = rng.uniform(-1, 1, n)
        X, Y = dev(cuda, x), dev(cuda, y)
        assert same_value(rb.call("reproBLAS_rdsum", 3, n, X, 1), port.rdsum(3, n, ptr(x), 1))
        assert same_value(rb.call("reproBLAS_rddot", 3, n, X, 1, Y, 1), port.rddot(3, n, ptr(x), 1, ptr(y), 1))
        assert same_value(rb.call("reproBLAS_rdnrm2", 3, n, X, 1), port.rdnrm2(3, n, ptr(x), 1))


def test_large_ddot_and_split_property(cuda, rb, port):
    """N = 2^26: equal to the oracle, and equal to the host merge (binned_dbdbadd, the
    operation binnedMPI_DBDBADD applies) of the states of 7 uneven GPU shards."""
    n = 1 << 26
    x, y = gen("normal", n, 21), gen("uniform", n, 22)
    X, Y = dev(cuda, x), dev(cuda, y)
    want = binned_zeros(3); port.dbddot(3, n, ptr(x), 1, ptr(y), 1, ptr(want))
    z = dev(cuda, binned_zeros(3)); rb.call("binnedBLAS_dbddot", 3, n, X, 1, Y, 1, z)
    assert same_bits(host(z), want)
    cuts = [0, 1, 999, 1 << 20, 5 << 20, 40 << 20, n - 3, n]
    merged = binned_zeros(3)
    for a, b in zip(cuts[:-1], cuts[1:]):
        part = dev(cuda, binned_zeros(3))
        rb.call("binnedBLAS_dbddot", 3, b - a, X[a:], 1, Y[a:], 1, part)
        hp = host(part)
        port.dbdbadd(3, ptr(hp), ptr(merged))
    assert same_bits(merged, want)
