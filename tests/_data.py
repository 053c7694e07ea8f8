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
