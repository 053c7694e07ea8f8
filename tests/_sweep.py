"""Shared pieces of the BLAS1 sweep parity tests: the sweep's sizes, folds, distributions and
routine groups, the seeded inputs, the reference-side prefix pass and the GPU calls."""
import ctypes
import math

import numpy as np

from _ffi import binned_zeros, fill

LOGN = list(range(10, 29, 2))        # 2^10 .. 2^28 in powers of 4
NMAX = 1 << LOGN[-1]
FOLDS = (2, 3, 4)
DISTS = ("uniform", "normal", "loguniform", "illcond")
LAUNCH_CONFIGS = [(1, 32), (1, 256), (2, 64), (2, 128), (4, 256), (8, 96), (16, 32), (3, 224)]
# The float-complex dots are left out: the reference's cmcdotc / cmcdotu deposit 1024 values
# per component between renormalisations (cmcdotc.ccog:36), twice the FP32 endurance, so at
# these lengths its state is not the canonical one.
GROUPS = {"real64": ("dsum", "ddot", "dnrm2", "dasum"),
          "real32": ("ssum", "sdot", "snrm2", "sasum"),
          "complex": ("zsum", "zdotc", "zdotu", "dznrm2", "dzasum"),
          "complex64": ("csum", "scnrm2", "scasum")}

# routine: (state kind, bytes per element of x, binned routine (oracle/reference short name),
#           form, reproBLAS_r* routine)
ROUTINES = {
    "dsum": ("d", 8, "dbdsum", "sum", "rdsum"),
    "ddot": ("d", 8, "dbddot", "dot", "rddot"),
    "dnrm2": ("d", 8, "dbdssq", "ssq", "rdnrm2"),
    "dasum": ("d", 8, "dbdasum", "sum", "rdasum"),
    "ssum": ("s", 4, "sbssum", "sum", "rssum"),
    "sdot": ("s", 4, "sbsdot", "dot", "rsdot"),
    "snrm2": ("s", 4, "sbsssq", "ssq", "rsnrm2"),
    "sasum": ("s", 4, "sbsasum", "sum", "rsasum"),
    "zsum": ("z", 16, "zbzsum", "sum", "rzsum_sub"),
    "zdotc": ("z", 16, "zbzdotc", "dot", "rzdotc_sub"),
    "zdotu": ("z", 16, "zbzdotu", "dot", "rzdotu_sub"),
    "dznrm2": ("d", 16, "dbzssq", "ssq", "rdznrm2"),
    "dzasum": ("d", 16, "dbzasum", "sum", "rdzasum"),
    "csum": ("c", 8, "cbcsum", "sum", "rcsum_sub"),
    "scnrm2": ("s", 8, "sbcssq", "ssq", "rscnrm2"),
    "scasum": ("s", 8, "sbcasum", "sum", "rscasum"),
}
KIND = {r: v[:2] for r, v in ROUTINES.items()}
SSQ = tuple(r for r, v in ROUTINES.items() if v[3] == "ssq")


def comps(routine):
    """Components of the routine's binned state (2 for a complex result)."""
    return 2 if ROUTINES[routine][0] in "zc" else 1


def _at(buf, i, esize):
    return ctypes.c_void_p(buf.ctypes.data + i * esize)


def _value(L, routine, fold, st, scale):
    """The reproBLAS_r* result from the binned state, as the reference converts it:
    rdsum.c / rdasum.c / rdzasum.c (ddbconv), rdnrm2.c:31 / rdznrm2.c (scale * sqrt of
    ddbconv), rssum.c / rsasum.c / rscasum.c (ssbconv), rsnrm2.c / rscnrm2.c (the float scale
    times the double sqrt of ssbconv, rounded to float), rzsum_sub.c / rz dot subs (ddmconv per
    component, binned_zzbconv_sub) and rcsum_sub.c (ssmconv per component,
    binned_ccbconv_sub)."""
    kind = ROUTINES[routine][0]
    sp = ctypes.c_void_p(st.ctypes.data)
    if kind == "d":
        v = L.ddbconv(fold, sp)
        return np.float64(scale * math.sqrt(v) if routine in SSQ else v)
    if kind == "s":
        v = L.ssbconv(fold, sp)
        return np.float32(scale * math.sqrt(v) if routine in SSQ else v)
    es = st.itemsize
    car = st.ctypes.data + 2 * fold * es
    conv = L.ddmconv if kind == "z" else L.ssmconv
    re = conv(fold, sp, 2, ctypes.c_void_p(car), 2)
    im = conv(fold, ctypes.c_void_p(st.ctypes.data + es), 2, ctypes.c_void_p(car + es), 2)
    return np.array([re, im], dtype=st.dtype)


def reference_prefixes(L, routine, fold, x, y, logn=LOGN):
    """{log2 N: (state, scale, value)} of the library L (the reference or the oracle) over
    every prefix 2^logn[i], by one accumulating pass: each step adds [previous prefix, this
    prefix) to the state, which then is the state of a single call over the prefix."""
    kind, es, name, form, _ = ROUTINES[routine]
    fn = getattr(L, name)
    st = binned_zeros(fold, kind)
    sp = ctypes.c_void_p(st.ctypes.data)
    scale = 0.0
    prev = 0
    out = {}
    for lg in logn:
        n = 1 << lg
        k = n - prev
        if form == "sum":
            fn(fold, k, _at(x, prev, es), 1, sp)
        elif form == "dot":
            fn(fold, k, _at(x, prev, es), 1, _at(y, prev, es), 1, sp)
        else:
            scale = fn(fold, k, _at(x, prev, es), 1, scale, sp)
        out[lg] = (st.copy(), scale, _value(L, routine, fold, st, scale))
        prev = n
    return out


def _state_buffer(cuda, routine, fold):
    kind = ROUTINES[routine][0]
    dt = cuda.float32 if kind in "sc" else cuda.float64
    return cuda.zeros(len(binned_zeros(fold, kind)), dtype=dt, device="cuda")


def gpu_state(cuda, rb, routine, fold, n, X, Y):
    """The binned state (and scale) of one fresh binnedBLAS_* call."""
    _, _, name, form, _ = ROUTINES[routine]
    z = _state_buffer(cuda, routine, fold)
    scale = 0.0
    if form == "sum":
        rb.call("binnedBLAS_" + name, fold, n, X, 1, z)
    elif form == "dot":
        rb.call("binnedBLAS_" + name, fold, n, X, 1, Y, 1, z)
    else:
        scale = rb.call("binnedBLAS_" + name, fold, n, X, 1, 0.0, z)
    return z.cpu().numpy(), scale


def gpu_call(cuda, rb, routine, fold, n, X, Y):
    """(state, scale, value) of one fresh binnedBLAS_* call and one reproBLAS_r* call."""
    kind, _, _, form, rname = ROUTINES[routine]
    st, scale = gpu_state(cuda, rb, routine, fold, n, X, Y)
    args = (X, 1, Y, 1) if form == "dot" else (X, 1)
    if kind in "zc":
        o = cuda.zeros(2, dtype=cuda.float64 if kind == "z" else cuda.float32, device="cuda")
        rb.call("reproBLAS_" + rname, fold, n, *args, o)
        v = o.cpu().numpy()
    else:
        v = rb.call("reproBLAS_" + rname, fold, n, *args)
        v = np.float64(v) if kind == "d" else np.float32(v)
    return st, scale, v


def group_inputs(dist, group, nmax=NMAX):
    """Host inputs of one routine group: nmax reals, or nmax complex elements (2 nmax
    values; the ill-conditioned pairs are then complex pairs (z, -z)). A group without a
    dot product gets no y."""
    seeds = {"uniform": 101, "normal": 202, "loguniform": 303, "illcond": 404}[dist]
    if group == "real32":
        return (fill(dist, seeds, nmax, np.float32), fill(dist, seeds + 1, nmax, np.float32))
    if group == "real64":
        return fill(dist, seeds, nmax), fill(dist, seeds + 1, nmax)
    if group == "complex64":
        return fill(dist, seeds, 2 * nmax, np.float32, unit=2), None
    return fill(dist, seeds, 2 * nmax, unit=2), fill(dist, seeds + 1, 2 * nmax, unit=2)
