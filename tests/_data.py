"""Seeded synthetic inputs with the value distributions the reference's tests and the
benchmark configurations use (uniform, normal, log-uniform magnitudes, ill-conditioned
cancelling pairs, sine)."""
import numpy as np


def gen(dist, n, seed=0, dtype=np.float64):
    rng = np.random.default_rng(seed)
    if dist == "uniform":
        x = rng.uniform(-1.0, 1.0, n)
    elif dist == "normal":
        x = rng.standard_normal(n)
    elif dist == "loguniform":
        lim = 300 if dtype == np.float64 else 100
        x = np.exp2(rng.uniform(-lim, lim, n)) * rng.choice([-1.0, 1.0], n)
    elif dist == "illcond":
        # (x, -x) pairs plus n/16 entries of magnitude 1e-12, shuffled
        half = n // 2
        a = rng.uniform(-1.0, 1.0, half)
        x = np.concatenate([a, -a, np.zeros(n - 2 * half)])
        k = n // 16
        idx = rng.choice(n, size=k, replace=False)
        x[idx] = 1e-12 * rng.choice([-1.0, 1.0], k)
        x = x[rng.permutation(n)]
    elif dist == "sine":
        x = np.sin(2 * np.pi * np.arange(n) / n)
    elif dist == "bigsmall":
        # the reference's "small + grow*big" style fill (big = 2^27, small = 2^-27)
        x = rng.uniform(-1.0, 1.0, n) * 2.0 ** -27
        x[:: max(1, n // 7)] *= 2.0 ** 54
    elif dist == "huge":
        # magnitudes near the overflow threshold: exercises bin index 0 and scaled conversion
        x = rng.uniform(0.5, 1.0, n) * 2.0 ** 1020 * rng.choice([-1.0, 1.0], n)
    elif dist == "tiny":
        # subnormal and near-subnormal magnitudes
        x = rng.uniform(-1.0, 1.0, n) * 2.0 ** -1060
    else:
        raise ValueError(dist)
    with np.errstate(over="ignore"):
        return np.ascontiguousarray(x.astype(dtype))


def gen_complex(dist, n, seed=0, dtype=np.complex128):
    base = np.float64 if dtype == np.complex128 else np.float32
    re = gen(dist, n, seed, base)
    im = gen(dist, n, seed + 7919, base)
    out = np.empty(n, dtype=dtype)
    out.real = re
    out.imag = im
    return out


def blas23_operands(seed, *sizes):
    """uniform(-1, 1) operands for the small gemv/gemm fixtures, one generator per case."""
    rng = np.random.default_rng(seed)
    return [rng.uniform(-1.0, 1.0, n) for n in sizes]


# ---- FP32 real / FP64 complex / FP32 complex gemv and gemm (types "s", "z", "c") ----------
XDTYPE = {"s": np.float32, "z": np.complex128, "c": np.complex64}
XREAL = {"s": np.float32, "z": np.float64, "c": np.float32}


def xblas23_operands(t, seed, *sizes):
    """uniform(-1, 1) operands of element type t (complex: independent real and imaginary
    parts), one generator per case."""
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        if t == "s":
            out.append(rng.uniform(-1.0, 1.0, n).astype(np.float32))
        else:
            v = rng.uniform(-1.0, 1.0, 2 * n).astype(XREAL[t])
            out.append(np.ascontiguousarray(v).view(XDTYPE[t]))
    return out


def xscalar(t, v):
    """alpha / beta as the C ABI takes them: a float for "s", else two reals."""
    v = complex(v)
    if t == "s":
        return np.float32(v.real)
    return np.array([v.real, v.imag], XREAL[t])


def xblas23_cases():
    """Parameters of the small s / z / c gemv and gemm fixtures: every order and transpose
    (n, t, c), fold 3 and one other fold. Complex alpha is (1.5, -0.25), except for column-
    major gemm with op(A) transposed, where the reference multiplies by (ar, ai) with ai in
    place of ar in the imaginary part (zbzgemm.ccog:655,754,799,850); there alpha =
    (1.25, 1.25), for which that product is the same. Column-major conjugate-transpose gemv
    is square (the reference's blocks assume M == N there)."""
    cases = []
    seed = 3000
    for t in "szc":
        for order in "rc":
            for ta in "ntc":
                M, N = (45, 45) if (order == "c" and ta == "c") else (37, 53)
                lda = N if order == "r" else M
                for fold in (3, 5 if t == "s" else 4):
                    cases.append({"kind": "gemv", "t": t, "order": order, "ta": ta, "M": M, "N": N,
                                  "lda": lda, "fold": fold, "alpha": [1.5, -0.25 if t != "s" else 0.0],
                                  "beta": [0.5, 0.25 if t != "s" else 0.0], "seed": seed})
                    seed += 1
                for tb in "ntc":
                    M, N, K = 11, 13, 41
                    if order == "r":
                        lda = K if ta == "n" else M
                        ldb = N if tb == "n" else K
                        ldc = N
                    else:
                        lda = M if ta == "n" else K
                        ldb = K if tb == "n" else N
                        ldc = M
                    al = [1.5, -0.25]
                    if t == "s":
                        al = [1.5, 0.0]
                    elif order == "c" and ta != "n":
                        al = [1.25, 1.25]
                    cases.append({"kind": "gemm", "t": t, "order": order, "ta": ta, "tb": tb,
                                  "M": M, "N": N, "K": K, "lda": lda, "ldb": ldb, "ldc": ldc,
                                  "fold": 3, "alpha": al,
                                  "beta": [0.5, 0.25 if t != "s" else 0.0], "seed": seed})
                    seed += 1
    return cases


def xblas23_case_operands(c):
    """The operands of one xblas23_cases() entry: (A, x, y) for gemv, (A, B, C) for gemm."""
    t = c["t"]
    if c["kind"] == "gemv":
        M, N = c["M"], c["N"]
        nt = c["ta"] == "n"
        return xblas23_operands(t, c["seed"], M * N, N if nt else M, M if nt else N)
    M, N, K = c["M"], c["N"], c["K"]
    return xblas23_operands(t, c["seed"], M * K, K * N, M * N)
