"""reproblas_b200 -- reproducible binned BLAS on NVIDIA B200 (sm_100a).

The product is the shared library ``libreproblas_b200.so`` built from ``csrc/`` and its C ABI
(``include/reproblas_b200.h``), a drop-in for ReproBLAS's ``reproBLAS_*`` / ``binnedBLAS_*``
entry points. This module loads that library with ctypes and exposes the same functions
under the reference's names (``lib.reproBLAS_rddot(fold, N, X, incX, Y, incY)``), plus
``call`` helpers that accept torch tensors (device or host) and numpy arrays.

There is no Python or CPU implementation of any routine: if the library cannot be loaded,
importing this package raises ImportError.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libreproblas_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "reproblas_b200.h")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        "reproblas_b200: %s is missing; build it with `python reproblas_b200/build.py` "
        "(or __graft_entry__.build())" % LIB_PATH)

_c_int, _c_ll, _c_double, _c_float, _c_char, _c_vp = (
    ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_float, ctypes.c_char,
    ctypes.c_void_p)

# name -> (restype, argtypes); mirrors include/reproblas_b200.h
SIGNATURES = {
    "reproBLAS_rdsum": (_c_double, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_dsum": (_c_double, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rddot": (_c_double, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int]),
    "reproBLAS_ddot": (_c_double, [_c_int, _c_vp, _c_int, _c_vp, _c_int]),
    "reproBLAS_rdnrm2": (_c_double, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_dnrm2": (_c_double, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rssum": (_c_float, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_ssum": (_c_float, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rsdot": (_c_float, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int]),
    "reproBLAS_sdot": (_c_float, [_c_int, _c_vp, _c_int, _c_vp, _c_int]),
    "reproBLAS_rzsum_sub": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_zsum_sub": (None, [_c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_rzdotc_sub": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_zdotc_sub": (None, [_c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_rcsum_sub": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_csum_sub": (None, [_c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_dbdsum": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_dbddot": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_dbdssq": (_c_double, [_c_int, _c_int, _c_vp, _c_int, _c_double, _c_vp]),
    "binnedBLAS_sbssum": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_sbsdot": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_zbzsum": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_zbzdotc": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_cbcsum": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_damax": (_c_double, [_c_int, _c_vp, _c_int]),
    "binnedBLAS_samax": (_c_float, [_c_int, _c_vp, _c_int]),
    "binnedBLAS_damaxm": (_c_double, [_c_int, _c_vp, _c_int, _c_vp, _c_int]),
    "binnedBLAS_samaxm": (_c_float, [_c_int, _c_vp, _c_int, _c_vp, _c_int]),
    "binnedBLAS_zamax_sub": (None, [_c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_camax_sub": (None, [_c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_zamaxm_sub": (None, [_c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_camaxm_sub": (None, [_c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_rsnrm2": (_c_float, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_snrm2": (_c_float, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rdznrm2": (_c_double, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_dznrm2": (_c_double, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rscnrm2": (_c_float, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_scnrm2": (_c_float, [_c_int, _c_vp, _c_int]),
    "binnedBLAS_sbsssq": (_c_float, [_c_int, _c_int, _c_vp, _c_int, _c_float, _c_vp]),
    "binnedBLAS_dbzssq": (_c_double, [_c_int, _c_int, _c_vp, _c_int, _c_double, _c_vp]),
    "binnedBLAS_sbcssq": (_c_float, [_c_int, _c_int, _c_vp, _c_int, _c_float, _c_vp]),
    "reproBLAS_rdasum": (_c_double, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_dasum": (_c_double, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rsasum": (_c_float, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_sasum": (_c_float, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rdzasum": (_c_double, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_dzasum": (_c_double, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rscasum": (_c_float, [_c_int, _c_int, _c_vp, _c_int]),
    "reproBLAS_scasum": (_c_float, [_c_int, _c_vp, _c_int]),
    "reproBLAS_rzdotu_sub": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_zdotu_sub": (None, [_c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_rcdotc_sub": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_cdotc_sub": (None, [_c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_rcdotu_sub": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_cdotu_sub": (None, [_c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_dbdasum": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_sbsasum": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_dbzasum": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_sbcasum": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_zbzdotu": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_cbcdotc": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "binnedBLAS_cbcdotu": (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp]),
    "reproBLAS_rdgemv": (None, [_c_int, _c_char, _c_char, _c_int, _c_int, _c_double, _c_vp,
                                _c_int, _c_vp, _c_int, _c_double, _c_vp, _c_int]),
    "reproBLAS_dgemv": (None, [_c_char, _c_char, _c_int, _c_int, _c_double, _c_vp, _c_int,
                               _c_vp, _c_int, _c_double, _c_vp, _c_int]),
    "reproBLAS_rdgemm": (None, [_c_int, _c_char, _c_char, _c_char, _c_int, _c_int, _c_int,
                                _c_double, _c_vp, _c_int, _c_vp, _c_int, _c_double, _c_vp,
                                _c_int]),
    "reproBLAS_dgemm": (None, [_c_char, _c_char, _c_char, _c_int, _c_int, _c_int, _c_double,
                               _c_vp, _c_int, _c_vp, _c_int, _c_double, _c_vp, _c_int]),
    "binnedBLAS_dbdgemv": (None, [_c_int, _c_char, _c_char, _c_int, _c_int, _c_double, _c_vp,
                                  _c_int, _c_vp, _c_int, _c_vp, _c_int]),
    "binnedBLAS_dbdgemm": (None, [_c_int, _c_char, _c_char, _c_char, _c_int, _c_int, _c_int,
                                  _c_double, _c_vp, _c_int, _c_vp, _c_int, _c_vp, _c_int]),
    "rb_dgemm_int8": (_c_int, [_c_int, _c_char, _c_char, _c_char, _c_int, _c_int, _c_int,
                               _c_double, _c_vp, _c_int, _c_vp, _c_int, _c_double, _c_vp,
                               _c_int, _c_int]),
    "rb_dgemm_int8_inspect": (_c_int, [_c_int, _c_int, _c_int, _c_vp, _c_vp, _c_int, _c_vp,
                                       _c_vp, _c_vp, _c_vp, _c_vp]),
    "rb_get_last_error": (_c_int, []),
    "rb_get_last_error_message": (ctypes.c_char_p, []),
    "rb_clear_error": (None, []),
    "rb_set_stream": (None, [_c_vp]),
    "rb_get_stream": (_c_vp, []),
    "rb_set_launch_config": (None, [_c_int, _c_int]),
    "rb_kernel_launch_count": (ctypes.c_ulonglong, []),
    "rb_synchronize": (_c_int, []),
    "rb_probe_launch": (_c_int, [_c_int, _c_ll, _c_int, _c_vp, _c_vp]),
    "rb_probe_occupancy": (_c_int, [_c_int]),
    "rb_debug_fail_allocations": (None, [_c_int]),
    "rb_debug_pipeline_fault": (None, [_c_ll, _c_ll]),
    "rb_version": (ctypes.c_char_p, []),
    "rb_dbdbadd_states": (_c_int, [_c_int, _c_int, _c_vp, _c_vp]),
    "rb_sbsbadd_states": (_c_int, [_c_int, _c_int, _c_vp, _c_vp]),
    "rb_zbzbadd_states": (_c_int, [_c_int, _c_int, _c_vp, _c_vp]),
    "rb_cbcbadd_states": (_c_int, [_c_int, _c_int, _c_vp, _c_vp]),
    "rb_dbdbaddsq_states": (_c_int, [_c_int, _c_int, _c_vp, _c_vp]),
    "rb_sbsbaddsq_states": (_c_int, [_c_int, _c_int, _c_vp, _c_vp]),
    "rb_ddot_noalloc": (_c_int, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp, _c_vp,
                                 _c_vp]),
}

# manual-layout forms: (fold, N, X, incX[, Y, incY][, scale], pri, incpri, car, inccar)
for _n in ("dmdsum", "dmdasum", "zmzsum", "dmzasum", "smssum", "smsasum", "cmcsum", "smcasum"):
    SIGNATURES["binnedBLAS_" + _n] = (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp, _c_int])
for _n in ("dmddot", "zmzdotu", "zmzdotc", "smsdot", "cmcdotu", "cmcdotc"):
    SIGNATURES["binnedBLAS_" + _n] = (None, [_c_int, _c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp, _c_int,
                                             _c_vp, _c_int])
for _n, _r in (("dmdssq", _c_double), ("dmzssq", _c_double), ("smsssq", _c_float), ("smcssq", _c_float)):
    SIGNATURES["binnedBLAS_" + _n] = (_r, [_c_int, _c_int, _c_vp, _c_int, _r, _c_vp, _c_int, _c_vp, _c_int])

# gemv / gemm of FP32 real (scalars by value) and FP64 / FP32 complex elements (scalars by
# pointer to two reals), same argument lists as the FP64 forms above
for _t, _b, _sc in (("s", "sbs", _c_float), ("z", "zbz", _c_vp), ("c", "cbc", _c_vp)):
    SIGNATURES["reproBLAS_r%sgemv" % _t] = (None, [_c_int, _c_char, _c_char, _c_int, _c_int, _sc, _c_vp,
                                                    _c_int, _c_vp, _c_int, _sc, _c_vp, _c_int])
    SIGNATURES["reproBLAS_%sgemv" % _t] = (None, [_c_char, _c_char, _c_int, _c_int, _sc, _c_vp, _c_int,
                                                   _c_vp, _c_int, _sc, _c_vp, _c_int])
    SIGNATURES["binnedBLAS_%sgemv" % _b] = (None, [_c_int, _c_char, _c_char, _c_int, _c_int, _sc, _c_vp,
                                                    _c_int, _c_vp, _c_int, _c_vp, _c_int])
    SIGNATURES["reproBLAS_r%sgemm" % _t] = (None, [_c_int, _c_char, _c_char, _c_char, _c_int, _c_int,
                                                    _c_int, _sc, _c_vp, _c_int, _c_vp, _c_int, _sc,
                                                    _c_vp, _c_int])
    SIGNATURES["reproBLAS_%sgemm" % _t] = (None, [_c_char, _c_char, _c_char, _c_int, _c_int, _c_int,
                                                   _sc, _c_vp, _c_int, _c_vp, _c_int, _sc, _c_vp,
                                                   _c_int])
    SIGNATURES["binnedBLAS_%sgemm" % _b] = (None, [_c_int, _c_char, _c_char, _c_char, _c_int, _c_int,
                                                    _c_int, _sc, _c_vp, _c_int, _c_vp, _c_int, _c_vp,
                                                    _c_int])

class DgemmInstance(ctypes.Structure):
    """rb_dgemm_instance (include/reproblas_b200.h)"""
    _fields_ = [("order", ctypes.c_char), ("transa", ctypes.c_char), ("transb", ctypes.c_char),
                ("m", ctypes.c_int), ("n", ctypes.c_int), ("k", ctypes.c_int),
                ("alpha", ctypes.c_double), ("A", ctypes.c_void_p), ("lda", ctypes.c_int),
                ("B", ctypes.c_void_p), ("ldb", ctypes.c_int), ("beta", ctypes.c_double),
                ("C", ctypes.c_void_p), ("ldc", ctypes.c_int)]


SIGNATURES.update({
    "rb_batch_plan_create": (_c_vp, [_c_int, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                                     _c_int, _c_vp]),
    "rb_batch_plan_autotune": (_c_int, [_c_vp, _c_int]),
    "rb_batch_plan_set_config": (_c_int, [_c_vp, _c_int, _c_ll, _c_ll, _c_int]),
    "rb_batch_plan_run": (_c_int, [_c_vp, _c_vp]),
    "rb_batch_plan_info": (_c_int, [_c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp]),
    "rb_batch_plan_destroy": (None, [_c_vp]),
})

lib = ctypes.CDLL(LIB_PATH)
for _name, (_res, _args) in SIGNATURES.items():
    if hasattr(lib, _name):
        _fn = getattr(lib, _name)
        _fn.restype = _res
        _fn.argtypes = _args


class ReproBLASError(RuntimeError):
    pass


def check():
    """Raise ReproBLASError if the last call on this thread recorded an error."""
    code = lib.rb_get_last_error()
    if code != 0:
        msg = lib.rb_get_last_error_message().decode(errors="replace")
        lib.rb_clear_error()
        raise ReproBLASError("reproblas_b200 error %d: %s" % (code, msg))


def ptr(a):
    """Address of a torch tensor, numpy array, int or None."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if hasattr(a, "ctypes"):
        return a.ctypes.data
    raise TypeError("cannot take the address of %r" % type(a))


def call(name, *args):
    """Call a C-ABI function by name, converting array arguments to pointers and raising
    on a recorded error."""
    fn = getattr(lib, name)
    conv = []
    for a, t in zip(args, fn.argtypes):
        if t is _c_vp:
            conv.append(ptr(a))
        elif t is _c_char:
            conv.append(a.encode() if isinstance(a, str) else a)
        else:
            conv.append(a)
    out = fn(*conv)
    check()
    return out


def exported_symbols():
    """Function names declared in include/reproblas_b200.h."""
    import re
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)) -
                  {"if", "defined"})


def version():
    return lib.rb_version().decode()
