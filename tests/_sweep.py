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
GROUPS = {"real64": ("dsum", "ddot", "dnrm2"), "real32": ("ssum", "sdot"),
          "complex": ("zsum", "zdotc")}
# state kind and bytes per element of the routine's x (and y)
KIND = {"dsum": ("d", 8), "ddot": ("d", 8), "dnrm2": ("d", 8), "ssum": ("s", 4),
        "sdot": ("s", 4), "zsum": ("z", 16), "zdotc": ("z", 16)}


def _at(buf, i, esize):
    return ctypes.c_void_p(buf.ctypes.data + i * esize)


def reference_prefixes(L, routine, fold, x, y, logn=LOGN):
    """{log2 N: (state, scale, value)} of the library L (the reference or the oracle) over
    every prefix 2^logn[i], by one accumulating pass: each step adds [previous prefix, this
    prefix) to the state, which then is the state of a single call over the prefix."""
    kind, es = KIND[routine]
    st = binned_zeros(fold, kind)
    sp = ctypes.c_void_p(st.ctypes.data)
    scale = 0.0
    prev = 0
    out = {}
    for lg in logn:
        n = 1 << lg
        k = n - prev
        if routine == "dsum":
            L.dbdsum(fold, k, _at(x, prev, es), 1, sp)
        elif routine == "ddot":
            L.dbddot(fold, k, _at(x, prev, es), 1, _at(y, prev, es), 1, sp)
        elif routine == "dnrm2":
            scale = L.dbdssq(fold, k, _at(x, prev, es), 1, scale, sp)
        elif routine == "ssum":
            L.sbssum(fold, k, _at(x, prev, es), 1, sp)
        elif routine == "sdot":
            L.sbsdot(fold, k, _at(x, prev, es), 1, _at(y, prev, es), 1, sp)
        elif routine == "zsum":
            L.zbzsum(fold, k, _at(x, prev, es), 1, sp)
        else:
            L.zbzdotc(fold, k, _at(x, prev, es), 1, _at(y, prev, es), 1, sp)
        # the conversions of reproBLAS_r* (rdsum.c, rddot.c, rdnrm2.c:31, rssum.c, rsdot.c,
        # rzsum_sub.c / rzdotc_sub.c through binned_zzbconv_sub = ddmconv per component)
        if kind == "d":
            v = L.ddbconv(fold, sp)
            if routine == "dnrm2":
                v = scale * math.sqrt(v)
            val = np.float64(v)
        elif kind == "s":
            val = np.float32(L.ssbconv(fold, sp))
        else:
            c = ctypes.c_void_p(st.ctypes.data + 2 * fold * 8)
            re = L.ddmconv(fold, sp, 2, c, 2)
            im = L.ddmconv(fold, ctypes.c_void_p(st.ctypes.data + 8), 2,
                           ctypes.c_void_p(st.ctypes.data + 2 * fold * 8 + 8), 2)
            val = np.array([re, im])
        out[lg] = (st.copy(), scale, val)
        prev = n
    return out


def gpu_call(cuda, rb, routine, fold, n, X, Y):
    """(state, scale, value) of one fresh binnedBLAS_* call and one reproBLAS_r* call."""
    kind, _ = KIND[routine]
    dt = cuda.float32 if kind == "s" else cuda.float64
    z = cuda.zeros(len(binned_zeros(fold, kind)), dtype=dt, device="cuda")
    scale = 0.0
    if routine == "dsum":
        rb.call("binnedBLAS_dbdsum", fold, n, X, 1, z)
        v = np.float64(rb.call("reproBLAS_rdsum", fold, n, X, 1))
    elif routine == "ddot":
        rb.call("binnedBLAS_dbddot", fold, n, X, 1, Y, 1, z)
        v = np.float64(rb.call("reproBLAS_rddot", fold, n, X, 1, Y, 1))
    elif routine == "dnrm2":
        scale = rb.call("binnedBLAS_dbdssq", fold, n, X, 1, 0.0, z)
        v = np.float64(rb.call("reproBLAS_rdnrm2", fold, n, X, 1))
    elif routine == "ssum":
        rb.call("binnedBLAS_sbssum", fold, n, X, 1, z)
        v = np.float32(rb.call("reproBLAS_rssum", fold, n, X, 1))
    elif routine == "sdot":
        rb.call("binnedBLAS_sbsdot", fold, n, X, 1, Y, 1, z)
        v = np.float32(rb.call("reproBLAS_rsdot", fold, n, X, 1, Y, 1))
    else:
        o = cuda.zeros(2, dtype=cuda.float64, device="cuda")
        if routine == "zsum":
            rb.call("binnedBLAS_zbzsum", fold, n, X, 1, z)
            rb.call("reproBLAS_rzsum_sub", fold, n, X, 1, o)
        else:
            rb.call("binnedBLAS_zbzdotc", fold, n, X, 1, Y, 1, z)
            rb.call("reproBLAS_rzdotc_sub", fold, n, X, 1, Y, 1, o)
        v = o.cpu().numpy()
    return z.cpu().numpy(), scale, v


def gpu_state(cuda, rb, routine, fold, n, X, Y):
    """The binned state (and scale) of one fresh binnedBLAS_* call."""
    kind, _ = KIND[routine]
    dt = cuda.float32 if kind == "s" else cuda.float64
    z = cuda.zeros(len(binned_zeros(fold, kind)), dtype=dt, device="cuda")
    scale = 0.0
    name = {"dsum": "dbdsum", "ddot": "dbddot", "dnrm2": "dbdssq", "ssum": "sbssum",
            "sdot": "sbsdot", "zsum": "zbzsum", "zdotc": "zbzdotc"}[routine]
    if routine == "dnrm2":
        scale = rb.call("binnedBLAS_dbdssq", fold, n, X, 1, 0.0, z)
    elif routine in ("ddot", "sdot", "zdotc"):
        rb.call("binnedBLAS_" + name, fold, n, X, 1, Y, 1, z)
    else:
        rb.call("binnedBLAS_" + name, fold, n, X, 1, z)
    return z.cpu().numpy(), scale


def group_inputs(dist, group, nmax=NMAX):
    """Host inputs of one routine group: nmax reals, or nmax complex elements (2 nmax
    doubles; the ill-conditioned pairs are then complex pairs (z, -z))."""
    seeds = {"uniform": 101, "normal": 202, "loguniform": 303, "illcond": 404}[dist]
    if group == "real32":
        return (fill(dist, seeds, nmax, np.float32), fill(dist, seeds + 1, nmax, np.float32))
    if group == "real64":
        return fill(dist, seeds, nmax), fill(dist, seeds + 1, nmax)
    return fill(dist, seeds, 2 * nmax, unit=2), fill(dist, seeds + 1, 2 * nmax, unit=2)
