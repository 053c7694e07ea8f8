"""ctypes bindings used by the tests: the oracle restatement (port), the reference library
compiled from its own sources (ref, optional), and the product's C ABI.

The oracle libraries are test infrastructure; the product library is what is checked.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PORT_SO = os.path.join(ROOT, "oracle", "_build", "librb_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libreproblas_ref.so")
REF_SOURCE_NOTE = os.path.join(ROOT, "oracle", "_ref", "SOURCE")


def reference_tree():
    """The ReproBLAS source tree, or None: $REPROBLAS_SRC, else the tree oracle/_ref was
    compiled from (the build records it in oracle/_ref/SOURCE), when it exists here."""
    cand = os.environ.get("REPROBLAS_SRC")
    if not cand and os.path.exists(REF_SOURCE_NOTE):
        with open(REF_SOURCE_NOTE) as f:
            cand = f.read().strip()
    return cand if cand and os.path.isdir(cand) else None

c_int, c_double, c_float, c_char, c_vp = (ctypes.c_int, ctypes.c_double, ctypes.c_float,
                                          ctypes.c_char, ctypes.c_void_p)


def ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


_SIGS = {
    # name: (restype, argtypes) -- shared by the port (rbo_ prefix) and the reference
    "dbdsum": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "dbddot": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "dbdssq": (c_double, [c_int, c_int, c_vp, c_int, c_double, c_vp]),
    "sbssum": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "sbsdot": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "zbzsum": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "zbzdotc": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "cbcsum": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "dbdasum": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "sbsasum": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "dbzasum": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "sbcasum": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "zbzdotu": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "cbcdotc": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "cbcdotu": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "damax": (c_double, [c_int, c_vp, c_int]),
    "samax": (c_float, [c_int, c_vp, c_int]),
    "damaxm": (c_double, [c_int, c_vp, c_int, c_vp, c_int]),
    "samaxm": (c_float, [c_int, c_vp, c_int, c_vp, c_int]),
    "zamax_sub": (None, [c_int, c_vp, c_int, c_vp]),
    "camax_sub": (None, [c_int, c_vp, c_int, c_vp]),
    "zamaxm_sub": (None, [c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "camaxm_sub": (None, [c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "sbsssq": (c_float, [c_int, c_int, c_vp, c_int, c_float, c_vp]),
    "dbzssq": (c_double, [c_int, c_int, c_vp, c_int, c_double, c_vp]),
    "sbcssq": (c_float, [c_int, c_int, c_vp, c_int, c_float, c_vp]),
    "rsnrm2": (c_float, [c_int, c_int, c_vp, c_int]),
    "rdznrm2": (c_double, [c_int, c_int, c_vp, c_int]),
    "rscnrm2": (c_float, [c_int, c_int, c_vp, c_int]),
    "rdasum": (c_double, [c_int, c_int, c_vp, c_int]),
    "rsasum": (c_float, [c_int, c_int, c_vp, c_int]),
    "rdzasum": (c_double, [c_int, c_int, c_vp, c_int]),
    "rscasum": (c_float, [c_int, c_int, c_vp, c_int]),
    "rzdotu_sub": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "rcdotc_sub": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "rcdotu_sub": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "dbdgemv": (None, [c_int, c_char, c_char, c_int, c_int, c_double, c_vp, c_int, c_vp, c_int,
                       c_vp, c_int]),
    "dbdgemm": (None, [c_int, c_char, c_char, c_char, c_int, c_int, c_int, c_double, c_vp, c_int,
                       c_vp, c_int, c_vp, c_int]),
    "rdsum": (c_double, [c_int, c_int, c_vp, c_int]),
    "rddot": (c_double, [c_int, c_int, c_vp, c_int, c_vp, c_int]),
    "rdnrm2": (c_double, [c_int, c_int, c_vp, c_int]),
    "rssum": (c_float, [c_int, c_int, c_vp, c_int]),
    "rsdot": (c_float, [c_int, c_int, c_vp, c_int, c_vp, c_int]),
    "rzsum_sub": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "rzdotc_sub": (None, [c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp]),
    "rcsum_sub": (None, [c_int, c_int, c_vp, c_int, c_vp]),
    "rdgemv": (None, [c_int, c_char, c_char, c_int, c_int, c_double, c_vp, c_int, c_vp, c_int,
                      c_double, c_vp, c_int]),
    "rdgemm": (None, [c_int, c_char, c_char, c_char, c_int, c_int, c_int, c_double, c_vp, c_int,
                      c_vp, c_int, c_double, c_vp, c_int]),
    "dbdbadd": (None, [c_int, c_vp, c_vp]),
    "dbdconv": (None, [c_int, c_double, c_vp]),
    "ddbconv": (c_double, [c_int, c_vp]),
    "ddmconv": (c_double, [c_int, c_vp, c_int, c_vp, c_int]),
    "dbdbaddsq": (c_double, [c_int, c_double, c_vp, c_double, c_vp]),
    "dbbound": (c_double, [c_int, c_int, c_double, c_double]),
    "dscale": (c_double, [c_double]),
    "dindex": (c_int, [c_double]),
    "sindex": (c_int, [c_float]),
    "sbsbadd": (None, [c_int, c_vp, c_vp]),
    "ssbconv": (c_float, [c_int, c_vp]),
    "ssmconv": (c_float, [c_int, c_vp, c_int, c_vp, c_int]),
}

# gemv / gemm of FP32 real (scalars by value) and complex (scalars by pointer) elements
for _t, _b, _sc in (("s", "sbs", c_float), ("z", "zbz", c_vp), ("c", "cbc", c_vp)):
    _SIGS[_b + "gemv"] = (None, [c_int, c_char, c_char, c_int, c_int, _sc, c_vp, c_int, c_vp,
                                 c_int, c_vp, c_int])
    _SIGS[_b + "gemm"] = (None, [c_int, c_char, c_char, c_char, c_int, c_int, c_int, _sc, c_vp,
                                 c_int, c_vp, c_int, c_vp, c_int])
    _SIGS["r" + _t + "gemv"] = (None, [c_int, c_char, c_char, c_int, c_int, _sc, c_vp, c_int, c_vp,
                                       c_int, _sc, c_vp, c_int])
    _SIGS["r" + _t + "gemm"] = (None, [c_int, c_char, c_char, c_char, c_int, c_int, c_int, _sc, c_vp,
                                       c_int, c_vp, c_int, _sc, c_vp, c_int])
_SIGS["sbsconv"] = (None, [c_int, c_float, c_vp])
_SIGS["zbzconv"] = (None, [c_int, c_vp, c_vp])
_SIGS["zbzbadd"] = (None, [c_int, c_vp, c_vp])
_SIGS["cbcbadd"] = (None, [c_int, c_vp, c_vp])
_SIGS["sbsbaddsq"] = (c_float, [c_int, c_float, c_vp, c_float, c_vp])
_SIGS["cbcconv"] = (None, [c_int, c_vp, c_vp])

# reference-library names for the shared signatures
_REF_NAMES = {
    "dbdsum": "binnedBLAS_dbdsum", "dbddot": "binnedBLAS_dbddot", "dbdssq": "binnedBLAS_dbdssq",
    "sbssum": "binnedBLAS_sbssum", "sbsdot": "binnedBLAS_sbsdot", "zbzsum": "binnedBLAS_zbzsum",
    "zbzdotc": "binnedBLAS_zbzdotc", "cbcsum": "binnedBLAS_cbcsum",
    "dbdgemv": "binnedBLAS_dbdgemv", "dbdgemm": "binnedBLAS_dbdgemm",
    "rdsum": "reproBLAS_rdsum", "rddot": "reproBLAS_rddot", "rdnrm2": "reproBLAS_rdnrm2",
    "rssum": "reproBLAS_rssum", "rsdot": "reproBLAS_rsdot", "rzsum_sub": "reproBLAS_rzsum_sub",
    "rzdotc_sub": "reproBLAS_rzdotc_sub", "rcsum_sub": "reproBLAS_rcsum_sub",
    "rdgemv": "reproBLAS_rdgemv", "rdgemm": "reproBLAS_rdgemm",
    "dbdasum": "binnedBLAS_dbdasum", "sbsasum": "binnedBLAS_sbsasum",
    "dbzasum": "binnedBLAS_dbzasum", "sbcasum": "binnedBLAS_sbcasum",
    "zbzdotu": "binnedBLAS_zbzdotu", "cbcdotc": "binnedBLAS_cbcdotc",
    "cbcdotu": "binnedBLAS_cbcdotu", "rdasum": "reproBLAS_rdasum", "rsasum": "reproBLAS_rsasum",
    "rdzasum": "reproBLAS_rdzasum", "rscasum": "reproBLAS_rscasum",
    "rzdotu_sub": "reproBLAS_rzdotu_sub", "rcdotc_sub": "reproBLAS_rcdotc_sub",
    "rcdotu_sub": "reproBLAS_rcdotu_sub",
    "sbsssq": "binnedBLAS_sbsssq", "dbzssq": "binnedBLAS_dbzssq", "sbcssq": "binnedBLAS_sbcssq",
    "damax": "binnedBLAS_damax", "samax": "binnedBLAS_samax", "damaxm": "binnedBLAS_damaxm",
    "samaxm": "binnedBLAS_samaxm", "zamax_sub": "binnedBLAS_zamax_sub",
    "camax_sub": "binnedBLAS_camax_sub", "zamaxm_sub": "binnedBLAS_zamaxm_sub",
    "camaxm_sub": "binnedBLAS_camaxm_sub",
    "rsnrm2": "reproBLAS_rsnrm2", "rdznrm2": "reproBLAS_rdznrm2", "rscnrm2": "reproBLAS_rscnrm2",
    "dbdbadd": "binned_dbdbadd", "dbdconv": "binned_dbdconv", "ddbconv": "binned_ddbconv", "ddmconv": "binned_ddmconv",
    "dbdbaddsq": "binned_dbdbaddsq", "dbbound": "binned_dbbound", "dscale": "binned_dscale",
    "dindex": "binned_dindex", "sindex": "binned_sindex", "sbsbadd": "binned_sbsbadd",
    "ssbconv": "binned_ssbconv", "ssmconv": "binned_ssmconv",
    "sbsconv": "binned_sbsconv", "zbzconv": "binned_zbzconv", "cbcconv": "binned_cbcconv",
    "zbzbadd": "binned_zbzbadd", "cbcbadd": "binned_cbcbadd", "sbsbaddsq": "binned_sbsbaddsq",
}
for _t, _b in (("s", "sbs"), ("z", "zbz"), ("c", "cbc")):
    _REF_NAMES[_b + "gemv"] = "binnedBLAS_%sgemv" % _b
    _REF_NAMES[_b + "gemm"] = "binnedBLAS_%sgemm" % _b
    _REF_NAMES["r%sgemv" % _t] = "reproBLAS_r%sgemv" % _t
    _REF_NAMES["r%sgemm" % _t] = "reproBLAS_r%sgemm" % _t


class _Lib:
    def __init__(self, path, names):
        self.path = path
        self.lib = ctypes.CDLL(path)
        for key, (res, args) in _SIGS.items():
            fn = getattr(self.lib, names(key))
            fn.restype = res
            fn.argtypes = args
            setattr(self, key, fn)


_port = None
_ref = None


def port():
    global _port
    if _port is None:
        _port = _Lib(PORT_SO, lambda k: "rbo_" + k)
        extra = _port.lib.rbo_exact_dot
        extra.restype = c_double
        extra.argtypes = [c_int, c_vp, c_int, c_vp, c_int]
        _port.exact_dot = extra
        for nm in ("rbo_fill_d", "rbo_fill_s"):
            fn = getattr(_port.lib, nm)
            fn.restype = c_int
            fn.argtypes = [c_int, ctypes.c_ulonglong, ctypes.c_longlong, c_vp, c_int, c_int]
        _port.fill_d = _port.lib.rbo_fill_d
        _port.fill_s = _port.lib.rbo_fill_s
    return _port


FILL_DISTS = {"uniform": 0, "normal": 1, "loguniform": 2, "illcond": 3}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def fill(dist, seed, n, dtype=np.float64, unit=1, out=None):
    """A seeded vector of n values of the given distribution (oracle/rb_fill.c): element i
    depends only on (dist, seed, i), so prefixes of a long vector are the shorter vectors.
    `unit` = 2 builds the ill-conditioned pairs from complex items (z, -z)."""
    out = np.empty(n, dtype) if out is None else out
    f = port().fill_d if out.dtype == np.float64 else port().fill_s
    rc = f(FILL_DISTS[dist], seed, n, out.ctypes.data, unit, min(64, host_threads()))
    assert rc == 0
    return out


def ref():
    """The reference library compiled from its own sources, or None when absent."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        _ref = _Lib(REF_SO, lambda k: _REF_NAMES[k])
    return _ref


def binned_zeros(fold, kind="d", n=1):
    per = {"d": 2 * fold, "z": 4 * fold, "s": 2 * fold, "c": 4 * fold}[kind]
    dt = np.float64 if kind in "dz" else np.float32
    return np.zeros(per * n, dtype=dt)
