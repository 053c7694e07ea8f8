"""The int8-sliced tensor-core reproducible dgemm (rb_dgemm_int8).

* the tcgen05 accumulators are exact: raw[t] == sum_{p+q=t} As[p] @ Bs[q]^T in int64;
* the digit slices reconstruct the operands to within 2^(e - 7 S);
* C is within (S + 3) K 2^(e_i + f_j - 7 S) + 2 ulp of the exact beta*C + alpha*A*B
  (exact host oracle: TwoProduct into a wide fixed-point accumulator, rounded once);
* C is bit-identical across decompositions (column blocks, row-major vs transposed
  column-major formulations)."""
import numpy as np
import pytest

from _ffi import ptr

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def baseline_operands(rng, m, n):
    """mantissas uniform in [1, 2), exponents uniform in [-20, 20], random signs"""
    mant = rng.uniform(1.0, 2.0, (m, n))
    ex = rng.integers(-20, 21, (m, n))
    return np.ldexp(mant, ex) * rng.choice([-1.0, 1.0], (m, n))


def rup(x, m):
    return (x + m - 1) // m * m


@pytest.mark.parametrize("S", [2, 3, 4, 7, 8, 9, 12])
def test_raw_accumulators_exact(cuda, rb, S):
    rng = np.random.default_rng(S)
    M, N, K = 200, 100, 300
    A = baseline_operands(rng, M, K)
    B = baseline_operands(rng, K, N)
    # B's rows are padded to the kernel's tile width: 64 columns up to 4 slices, else 32
    # (tile_bn in rb_int8gemm_impl.cuh)
    Mp, Np, Kp = rup(M, 128), rup(N, 64 if S <= 4 else 32), rup(K, 32)
    raw = cuda.zeros(S * Mp * Np, dtype=cuda.int32, device="cuda")
    As = cuda.zeros(S * Mp * Kp, dtype=cuda.int8, device="cuda")
    Bs = cuda.zeros(S * Np * Kp, dtype=cuda.int8, device="cuda")
    ea = cuda.zeros(M, dtype=cuda.int32, device="cuda")
    fb = cuda.zeros(N, dtype=cuda.int32, device="cuda")
    code = rb.call("rb_dgemm_int8_inspect", M, N, K, dev(cuda, A), dev(cuda, B), S, raw, As, Bs, ea, fb)
    assert code == 0
    # pre-tiled layout [Kp/16][S][rows/8][8][16] -> [S][rows][Kp]
    As = As.cpu().numpy().reshape(Kp // 16, S, Mp // 8, 8, 16).transpose(1, 2, 3, 0, 4)
    As = As.reshape(S, Mp, Kp).astype(np.int64)
    Bs = Bs.cpu().numpy().reshape(Kp // 16, S, Np // 8, 8, 16).transpose(1, 2, 3, 0, 4)
    Bs = Bs.reshape(S, Np, Kp).astype(np.int64)
    ea = ea.cpu().numpy()
    fb = fb.cpu().numpy()
    # digits reconstruct the operands
    Ahat = sum(np.ldexp(As[p, :M, :K].astype(np.float64), (ea[:, None] - 7 * (p + 1))) for p in range(S))
    assert np.all(np.abs(A - Ahat) < np.ldexp(1.0, ea[:, None] - 7 * S))
    Bhat = sum(np.ldexp(Bs[q, :N, :K].astype(np.float64), (fb[:, None] - 7 * (q + 1))) for q in range(S))
    assert np.all(np.abs(B.T - Bhat) < np.ldexp(1.0, fb[:, None] - 7 * S))
    assert np.all(As[:, M:, :] == 0) and np.all(As[:, :, K:] == 0)
    # tensor-core accumulators equal the exact integer sums
    raw = raw.cpu().numpy().reshape(S, Mp, Np).astype(np.int64)
    for t in range(S):
        want = sum(As[p] @ Bs[t - p].T for p in range(t + 1))
        assert np.array_equal(raw[t], want), t


def exact_entries(port, A, B, C, alpha, beta, idx):
    out = []
    for i, j in idx:
        a = A[i, :] * alpha if alpha != 1.0 else A[i, :].copy()
        x = np.concatenate([a, [C[i, j] * beta if beta not in (0.0, 1.0) else (C[i, j] if beta == 1.0 else 0.0)]])
        y = np.concatenate([B[:, j], [1.0]])
        x = np.ascontiguousarray(x); y = np.ascontiguousarray(y)
        out.append(port.exact_dot(len(x), ptr(x), 1, ptr(y), 1))
    return np.array(out)


@pytest.mark.parametrize("S", [6, 7, 8, 10, 12])
def test_error_vs_exact_oracle(cuda, rb, port, S):
    rng = np.random.default_rng(10 + S)
    M, N, K = 384, 320, 1000
    A = baseline_operands(rng, M, K)
    B = baseline_operands(rng, K, N)
    C = rng.uniform(-1, 1, (M, N))
    alpha, beta = 1.5, 0.5
    Cd = dev(cuda, C)
    code = rb.call("rb_dgemm_int8", 3, "r", "n", "n", M, N, K, alpha, dev(cuda, A), K, dev(cuda, B), N,
                   beta, Cd, N, S)
    assert code == 0
    got = Cd.cpu().numpy()
    idx = [(int(rng.integers(0, M)), int(rng.integers(0, N))) for _ in range(400)]
    ex = exact_entries(port, A, B, C, alpha, beta, idx)
    e_i = np.array([np.frexp(np.max(np.abs(A[i, :] * alpha)))[1] for i, _ in idx])
    f_j = np.array([np.frexp(np.max(np.abs(B[:, j])))[1] for _, j in idx])
    bound = (S + 3) * K * np.ldexp(1.0, e_i + f_j - 7 * S) + 2 * np.spacing(np.abs(ex))
    err = np.abs(np.array([got[i, j] for i, j in idx]) - ex)
    assert np.all(err <= bound), np.max(err / bound)


@pytest.mark.parametrize("S", [7, 10])
def test_bit_identical_across_decompositions(cuda, rb, S):
    rng = np.random.default_rng(77)
    M, N, K = 256, 256, 512
    A = baseline_operands(rng, M, K)
    B = baseline_operands(rng, K, N)
    C = rng.uniform(-1, 1, (M, N))
    full = dev(cuda, C)
    assert rb.call("rb_dgemm_int8", 3, "r", "n", "n", M, N, K, 1.5, dev(cuda, A), K, dev(cuda, B), N, 0.5, full, N, S) == 0
    full = full.cpu().numpy()
    # columns in two blocks (different tiles see different data)
    parts = []
    for j0, j1 in [(0, 100), (100, N)]:
        Bp = np.ascontiguousarray(B[:, j0:j1]); Cp = dev(cuda, np.ascontiguousarray(C[:, j0:j1]))
        assert rb.call("rb_dgemm_int8", 3, "r", "n", "n", M, j1 - j0, K, 1.5, dev(cuda, A), K,
                       dev(cuda, Bp), j1 - j0, 0.5, Cp, j1 - j0, S) == 0
        parts.append(Cp.cpu().numpy())
    assert np.concatenate(parts, axis=1).tobytes() == full.tobytes()
    # the transposed column-major formulation of the same product
    Ct = dev(cuda, np.ascontiguousarray(C.T))
    assert rb.call("rb_dgemm_int8", 3, "c", "t", "t", M, N, K, 1.5, dev(cuda, A), K, dev(cuda, B), N,
                   0.5, Ct, M, S) == 0
    assert np.ascontiguousarray(Ct.cpu().numpy().T).tobytes() == full.tobytes()


def test_rejects_non_finite_and_host_pointers(cuda, rb):
    A = np.ones((128, 64)); A[3, 5] = np.inf
    B = np.ones((64, 64)); C = dev(cuda, np.zeros((128, 64)))
    Ad, Bd = dev(cuda, A), dev(cuda, B)   # keep the device copies alive across the call
    code = rb.lib.rb_dgemm_int8(3, b"r", b"n", b"n", 128, 64, 64, 1.0, Ad.data_ptr(), 64,
                                Bd.data_ptr(), 64, 0.0, C.data_ptr(), 64, 6)
    assert code == 4 and float(C.abs().sum()) == 0.0
    rb.lib.rb_clear_error()
    code = rb.lib.rb_dgemm_int8(3, b"r", b"n", b"n", 128, 64, 64, 1.0, A.ctypes.data, 64,
                                B.ctypes.data, 64, 0.0, C.data_ptr(), 64, 6)
    assert code == 1
    rb.lib.rb_clear_error()
