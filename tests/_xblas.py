"""Uniform calls of the FP32 real ("s"), FP64 complex ("z") and FP32 complex ("c") gemv /
gemm forms on the oracle or the compiled reference (ctypes libraries from _ffi) and on the
product's C ABI (reproblas_b200.call)."""
import numpy as np

from _data import XREAL, xscalar
from _ffi import ptr

BIN = {"s": "sbs", "z": "zbz", "c": "cbc"}


def comps(t):
    return 1 if t == "s" else 2


def state_len(t, fold):
    return 2 * fold * comps(t)


def _scal(t, v):
    """(object to keep alive, ctypes argument) for alpha / beta."""
    x = xscalar(t, v)
    return (x, float(x)) if t == "s" else (x, ptr(x))


def lib_gemv(L, t, fold, order, ta, M, N, alpha, A, lda, x, incx, beta, y, incy, binned=False):
    """Value form r?gemv (binned=False, y values) or binned form ?b?gemv (y states) on an
    oracle / reference library; y updated in place (numpy)."""
    ka, a = _scal(t, alpha)
    kb, b = _scal(t, beta)
    if binned:
        getattr(L, BIN[t] + "gemv")(fold, order.encode(), ta.encode(), M, N, a, ptr(A), lda,
                                    ptr(x), incx, ptr(y), incy)
    else:
        getattr(L, "r%sgemv" % t)(fold, order.encode(), ta.encode(), M, N, a, ptr(A), lda,
                                  ptr(x), incx, b, ptr(y), incy)
    del ka, kb


def lib_gemm(L, t, fold, order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
             binned=False):
    ka, a = _scal(t, alpha)
    kb, b = _scal(t, beta)
    if binned:
        getattr(L, BIN[t] + "gemm")(fold, order.encode(), ta.encode(), tb.encode(), M, N, K, a,
                                    ptr(A), lda, ptr(B), ldb, ptr(C), ldc)
    else:
        getattr(L, "r%sgemm" % t)(fold, order.encode(), ta.encode(), tb.encode(), M, N, K, a,
                                  ptr(A), lda, ptr(B), ldb, b, ptr(C), ldc)
    del ka, kb


def rb_scalar(t, v):
    """alpha / beta for reproblas_b200.call: a float, or a two-real host array."""
    x = xscalar(t, v)
    return float(x) if t == "s" else x


def rb_gemv(rb, t, fold, order, ta, M, N, alpha, A, lda, x, incx, beta, y, incy, binned=False):
    """The product's r?gemv / ?b?gemv through the C ABI; operands are numpy arrays (host
    memory) or torch tensors (device memory)."""
    if binned:
        rb.call("binnedBLAS_%sgemv" % BIN[t], fold, order, ta, M, N, rb_scalar(t, alpha), A, lda,
                x, incx, y, incy)
    else:
        rb.call("reproBLAS_r%sgemv" % t, fold, order, ta, M, N, rb_scalar(t, alpha), A, lda, x,
                incx, rb_scalar(t, beta), y, incy)


def rb_gemm(rb, t, fold, order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
            binned=False):
    if binned:
        rb.call("binnedBLAS_%sgemm" % BIN[t], fold, order, ta, tb, M, N, K, rb_scalar(t, alpha),
                A, lda, B, ldb, C, ldc)
    else:
        rb.call("reproBLAS_r%sgemm" % t, fold, order, ta, tb, M, N, K, rb_scalar(t, alpha), A,
                lda, B, ldb, rb_scalar(t, beta), C, ldc)


def real_view(t, a):
    return np.ascontiguousarray(a).view(XREAL[t])


def reference_alpha_a(t, A, alpha, ta):
    """The reference's column-major transposed complex gemm with alpha != 1 multiplies A by
    alpha with alpha's imaginary part in place of its real part in the second product of the
    imaginary part (zbzgemm.ccog:655 for 'T'; 754, 799, 850 for 'C', after conjugation).
    Returns A' such that op(A') with alpha 1 gives those operands (for 'C' the conjugate of
    the reference's product, which op() conjugates back), so that the oracle can reproduce
    the reference's bits there."""
    rt = XREAL[t]
    a0, a1 = rt(complex(alpha).real), rt(complex(alpha).imag)
    ar, ai = A.real.astype(rt), A.imag.astype(rt)
    out = np.empty_like(A)
    if ta in "tT":
        out.real = ar * a0 - ai * a1
        out.imag = ar * a1 + ai * a1
    else:
        out.real = ar * a0 + ai * a1
        out.imag = -(ar * a1 - ai * a1)
    return out
