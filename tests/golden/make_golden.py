"""Generate the golden fixtures in this directory from the ReproBLAS reference library
itself, compiled from its own sources by `make -C oracle ref` (oracle/_ref/).

Inputs are regenerated from (distribution, n, seed) by tests/_data.py; the fixture stores
a SHA-256 of each input so that a change in the generator is detected rather than
silently compared. Outputs are the reference's binned states and converted results.

Usage: python tests/golden/make_golden.py   (needs oracle/_ref/libreproblas_ref.so)
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from _ffi import ref, ptr, binned_zeros  # noqa: E402
from _data import gen, gen_complex, blas23_operands  # noqa: E402
from _data import XREAL, xblas23_cases, xblas23_case_operands, xscalar  # noqa: E402

DISTS = ["uniform", "normal", "loguniform", "illcond", "sine", "bigsmall", "huge", "tiny"]
NS = [1, 7, 1000, 4095, 20000]
FOLDS = [2, 3, 4]


def h(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def hexb(a):
    return np.ascontiguousarray(a).tobytes().hex()


def ref_chunked(fn, fold, n, x, y, chunk=256):
    """The reference's float complex dot applied to consecutive calls of `chunk` elements
    accumulating into one state."""
    z = binned_zeros(fold, "c")
    for o in range(0, n, chunk):
        m = min(chunk, n - o)
        fn(fold, m, ptr(x[o:]), 1, ptr(y[o:]), 1, ptr(z))
    return z


def cconv(R, fold, z):
    """binned_ccbconv_sub through the reference's float conversion of each component."""
    out = np.zeros(2, np.float32)
    for k in range(2):
        comp = np.concatenate([z[k:2 * fold:2], z[2 * fold + k::2]]).astype(np.float32)
        out[k] = R.ssbconv(fold, ptr(comp))
    return out


def main():
    R = ref()
    if R is None:
        sys.exit("oracle/_ref/libreproblas_ref.so not built (make -C oracle ref)")
    cases = []
    for dist in DISTS:
        for n in NS:
            x = gen(dist, n, 11)
            y = gen(dist, n, 12)
            xf = gen(dist, n, 11, np.float32)
            yf = gen(dist, n, 12, np.float32)
            xz = gen_complex(dist, n, 11)
            yz = gen_complex(dist, n, 12)
            xc = gen_complex(dist, n, 11, np.complex64)
            hashes = {"x": h(x), "y": h(y), "xf": h(xf), "yf": h(yf), "xz": h(xz),
                      "yz": h(yz), "xc": h(xc)}
            for fold in FOLDS:
                c = {"dist": dist, "n": n, "fold": fold, "hash": hashes}
                z = binned_zeros(fold); R.dbdsum(fold, n, ptr(x), 1, ptr(z)); c["dbdsum"] = hexb(z)
                c["rdsum"] = hexb(np.float64(R.rdsum(fold, n, ptr(x), 1)))
                z = binned_zeros(fold); R.dbddot(fold, n, ptr(x), 1, ptr(y), 1, ptr(z)); c["dbddot"] = hexb(z)
                c["rddot"] = hexb(np.float64(R.rddot(fold, n, ptr(x), 1, ptr(y), 1)))
                z = binned_zeros(fold); s = R.dbdssq(fold, n, ptr(x), 1, 0.0, ptr(z))
                c["dbdssq"] = hexb(z); c["dbdssq_scale"] = hexb(np.float64(s))
                c["rdnrm2"] = hexb(np.float64(R.rdnrm2(fold, n, ptr(x), 1)))
                z = binned_zeros(fold, "s"); R.sbssum(fold, n, ptr(xf), 1, ptr(z)); c["sbssum"] = hexb(z)
                c["rssum"] = hexb(np.float32(R.rssum(fold, n, ptr(xf), 1)))
                z = binned_zeros(fold, "s"); R.sbsdot(fold, n, ptr(xf), 1, ptr(yf), 1, ptr(z)); c["sbsdot"] = hexb(z)
                c["rsdot"] = hexb(np.float32(R.rsdot(fold, n, ptr(xf), 1, ptr(yf), 1)))
                z = binned_zeros(fold, "z"); R.zbzsum(fold, n, ptr(xz), 1, ptr(z)); c["zbzsum"] = hexb(z)
                o = np.zeros(2); R.rzsum_sub(fold, n, ptr(xz), 1, ptr(o)); c["rzsum"] = hexb(o)
                z = binned_zeros(fold, "z"); R.zbzdotc(fold, n, ptr(xz), 1, ptr(yz), 1, ptr(z)); c["zbzdotc"] = hexb(z)
                o = np.zeros(2); R.rzdotc_sub(fold, n, ptr(xz), 1, ptr(yz), 1, ptr(o)); c["rzdotc"] = hexb(o)
                z = binned_zeros(fold, "c"); R.cbcsum(fold, n, ptr(xc), 1, ptr(z)); c["cbcsum"] = hexb(z)
                o = np.zeros(2, np.float32); R.rcsum_sub(fold, n, ptr(xc), 1, ptr(o)); c["rcsum"] = hexb(o)
                cases.append(c)

    # Absolute sums and the remaining complex dots, same inputs (plus the float complex y)
    more = []
    for dist in DISTS:
        for n in NS:
            x = gen(dist, n, 11)
            xf = gen(dist, n, 11, np.float32)
            xz, yz = gen_complex(dist, n, 11), gen_complex(dist, n, 12)
            xc, yc = gen_complex(dist, n, 11, np.complex64), gen_complex(dist, n, 12, np.complex64)
            hashes = {"x": h(x), "xf": h(xf), "xz": h(xz), "yz": h(yz), "xc": h(xc), "yc": h(yc)}
            for fold in FOLDS:
                c = {"dist": dist, "n": n, "fold": fold, "hash": hashes}
                z = binned_zeros(fold); R.dbdasum(fold, n, ptr(x), 1, ptr(z)); c["dbdasum"] = hexb(z)
                c["rdasum"] = hexb(np.float64(R.rdasum(fold, n, ptr(x), 1)))
                z = binned_zeros(fold, "s"); R.sbsasum(fold, n, ptr(xf), 1, ptr(z)); c["sbsasum"] = hexb(z)
                c["rsasum"] = hexb(np.float32(R.rsasum(fold, n, ptr(xf), 1)))
                z = binned_zeros(fold); R.dbzasum(fold, n, ptr(xz), 1, ptr(z)); c["dbzasum"] = hexb(z)
                c["rdzasum"] = hexb(np.float64(R.rdzasum(fold, n, ptr(xz), 1)))
                z = binned_zeros(fold, "s"); R.sbcasum(fold, n, ptr(xc), 1, ptr(z)); c["sbcasum"] = hexb(z)
                c["rscasum"] = hexb(np.float32(R.rscasum(fold, n, ptr(xc), 1)))
                z = binned_zeros(fold, "z"); R.zbzdotu(fold, n, ptr(xz), 1, ptr(yz), 1, ptr(z)); c["zbzdotu"] = hexb(z)
                o = np.zeros(2); R.rzdotu_sub(fold, n, ptr(xz), 1, ptr(yz), 1, ptr(o)); c["rzdotu"] = hexb(o)
                # float complex dots: the reference deposits 1024 values per component between
                # renormalisations in its 512-element blocks, twice the FP32 endurance, and its
                # state then depends on where a call starts; within 256-element calls it is the
                # canonical state that any correct order produces, which is what is stored
                for nm, fn in (("cbcdotc", R.cbcdotc), ("cbcdotu", R.cbcdotu)):
                    z = ref_chunked(fn, fold, n, xc, yc)
                    c[nm] = hexb(z)
                    c["r" + nm[3:]] = hexb(cconv(R, fold, z))
                z = binned_zeros(fold, "s"); sc = R.sbsssq(fold, n, ptr(xf), 1, 0.0, ptr(z))
                c["sbsssq"] = hexb(z); c["sbsssq_scale"] = hexb(np.float32(sc))
                z = binned_zeros(fold); sc = R.dbzssq(fold, n, ptr(xz), 1, 0.0, ptr(z))
                c["dbzssq"] = hexb(z); c["dbzssq_scale"] = hexb(np.float64(sc))
                z = binned_zeros(fold, "s"); sc = R.sbcssq(fold, n, ptr(xc), 1, 0.0, ptr(z))
                c["sbcssq"] = hexb(z); c["sbcssq_scale"] = hexb(np.float32(sc))
                c["rsnrm2"] = hexb(np.float32(R.rsnrm2(fold, n, ptr(xf), 1)))
                c["rdznrm2"] = hexb(np.float64(R.rdznrm2(fold, n, ptr(xz), 1)))
                c["rscnrm2"] = hexb(np.float32(R.rscnrm2(fold, n, ptr(xc), 1)))
                more.append(c)

    # The dsum configuration quoted by the benchmark: N = 2^20, fold 3, sine and uniform
    cfg0 = []
    for dist in ["sine", "uniform"]:
        x = gen(dist, 1 << 20, 0)
        z = binned_zeros(3); R.dbdsum(3, 1 << 20, ptr(x), 1, ptr(z))
        cfg0.append({"dist": dist, "n": 1 << 20, "seed": 0, "hash": h(x), "dbdsum": hexb(z),
                     "rdsum": hexb(np.float64(R.rdsum(3, 1 << 20, ptr(x), 1)))})

    # Inf / NaN vectors (the reference's validate_internal_daugsum Inf/NaN fills, N=255)
    special = []
    rng = np.random.default_rng(3)
    for k in range(12):
        x = rng.uniform(-1, 1, 255)
        pos = rng.choice(255, size=1 + k % 3, replace=False)
        vals = [np.inf, -np.inf, np.nan][k % 3:] + [np.inf, -np.inf, np.nan][:k % 3]
        for p, v in zip(pos, vals):
            x[p] = v
        y = np.ones(255)
        special.append({"x": hexb(x),
                        "rdsum": hexb(np.float64(R.rdsum(3, 255, ptr(x), 1))),
                        "rddot": hexb(np.float64(R.rddot(3, 255, ptr(x), 1, ptr(y), 1))),
                        "rdnrm2": hexb(np.float64(R.rdnrm2(3, 255, ptr(x), 1)))})

    # Small gemv / gemm (all orders and transposes), alpha 1.5, beta 0.5, fold 3.
    # Operands are regenerated from blas23_operands(seed) and checked by hash.
    blas23 = []
    seed = 1000
    for order in "rc":
        for ta in "nt":
            M, N = 37, 53
            A, xv, yv = blas23_operands(seed, M * N, 64, 64)
            lda = N if order == "r" else M
            yo = yv.copy()
            R.rdgemv(3, order.encode(), ta.encode(), M, N, 1.5, ptr(A), lda, ptr(xv), 1, 0.5, ptr(yo), 1)
            blas23.append({"kind": "gemv", "order": order, "ta": ta, "M": M, "N": N, "lda": lda,
                           "seed": seed, "hash": h(np.concatenate([A, xv, yv])), "out": hexb(yo)})
            seed += 1
            for tb in "nt":
                M, N, K = 19, 23, 41
                A, B, C = blas23_operands(seed, M * K, K * N, M * N)
                if order == "r":
                    lda = K if ta == "n" else M; ldb = N if tb == "n" else K; ldc = N
                else:
                    lda = M if ta == "n" else K; ldb = K if tb == "n" else N; ldc = M
                Co = C.copy()
                R.rdgemm(3, order.encode(), ta.encode(), tb.encode(), M, N, K, 1.5, ptr(A), lda,
                         ptr(B), ldb, 0.5, ptr(Co), ldc)
                blas23.append({"kind": "gemm", "order": order, "ta": ta, "tb": tb, "M": M, "N": N,
                               "K": K, "lda": lda, "ldb": ldb, "ldc": ldc, "seed": seed,
                               "hash": h(np.concatenate([A, B, C])), "out": hexb(Co)})
                seed += 1

    # s / z / c gemv and gemm (xblas23_cases in tests/_data.py): the value form (r*gemv /
    # r*gemm) and the binned form accumulating into empty states (stored as a hash).
    xblas23 = []
    for c in xblas23_cases():
        t, fold = c["t"], c["fold"]
        b = {"s": "sbs", "z": "zbz", "c": "cbc"}[t]
        comps = 1 if t == "s" else 2
        al, be = xscalar(t, complex(*c["alpha"])), xscalar(t, complex(*c["beta"]))
        sa = al if t == "s" else ptr(al)
        sb = be if t == "s" else ptr(be)
        ops = xblas23_case_operands(c)
        e = dict(c)
        e["hash"] = h(np.concatenate([o.view(XREAL[t]) for o in ops]))
        order, ta = c["order"].encode(), c["ta"].encode()
        if c["kind"] == "gemv":
            A, xv, yv = ops
            yo = yv.copy()
            getattr(R, "r%sgemv" % t)(fold, order, ta, c["M"], c["N"], sa, ptr(A), c["lda"],
                                     ptr(xv), 1, sb, ptr(yo), 1)
            zs = np.zeros(len(yv) * 2 * fold * comps, XREAL[t])
            getattr(R, b + "gemv")(fold, order, ta, c["M"], c["N"], sa, ptr(A), c["lda"], ptr(xv),
                                   1, ptr(zs), 1)
        else:
            A, B, C = ops
            yo = C.copy()
            tb = c["tb"].encode()
            getattr(R, "r%sgemm" % t)(fold, order, ta, tb, c["M"], c["N"], c["K"], sa, ptr(A),
                                     c["lda"], ptr(B), c["ldb"], sb, ptr(yo), c["ldc"])
            zs = np.zeros(len(C) * 2 * fold * comps, XREAL[t])
            getattr(R, b + "gemm")(fold, order, ta, tb, c["M"], c["N"], c["K"], sa, ptr(A),
                                   c["lda"], ptr(B), c["ldb"], ptr(zs), c["ldc"])
        e["out"] = hexb(yo)
        e["states_hash"] = h(zs)
        xblas23.append(e)

    out = {"generator": "tests/golden/make_golden.py", "reference": "ReproBLAS v2.1.0 "
           "compiled by oracle/Makefile (gcc -std=c99 -O3 -march=x86-64-v3)",
           "blas1": cases, "blas1_more": more, "dsum_config": cfg0, "special": special,
           "blas23": blas23, "xblas23": xblas23}
    with open(os.path.join(HERE, "reference_golden.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", len(cases), "blas1 cases,", len(special), "special,", len(blas23), "blas2/3,",
          len(xblas23), "s/z/c blas2/3")


if __name__ == "__main__":
    main()
