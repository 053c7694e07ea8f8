"""GPU merges of binned states of every kind (rb_dbdbadd_states, rb_sbsbadd_states,
rb_zbzbadd_states, rb_cbcbadd_states, rb_dbdbaddsq_states, rb_sbsbaddsq_states): the states
of uneven shards, computed on the GPU, merged into a non-empty state, equal the state of the
whole vector and the oracle's sequential merge in the reference's arithmetic, bit for bit."""
import numpy as np
import pytest

from _cmp import same_state, same_value
from _data import gen, gen_complex
from _ffi import binned_zeros, ptr

pytestmark = pytest.mark.gpu


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


def as_real(a):
    return a.view(np.float64 if a.dtype == np.complex128 else np.float32)


SUMS = {"d": ("binnedBLAS_dbdsum", np.float64, 1), "s": ("binnedBLAS_sbssum", np.float32, 1),
        "z": ("binnedBLAS_zbzsum", np.complex128, 2), "c": ("binnedBLAS_cbcsum", np.complex64, 2)}
MERGE = {"d": "rb_dbdbadd_states", "s": "rb_sbsbadd_states", "z": "rb_zbzbadd_states",
         "c": "rb_cbcbadd_states"}
PORT_ADD = {"d": "dbdbadd", "s": "sbsbadd", "z": "zbzbadd", "c": "cbcbadd"}


def _cuts(n, parts, rng):
    c = np.sort(rng.integers(0, n + 1, parts - 1))
    return np.concatenate([[0], c, [n]]).astype(int)


@pytest.mark.parametrize("kind", ["d", "s", "z", "c"])
@pytest.mark.parametrize("fold", [2, 3, 5, 8])
def test_state_merge_kinds(cuda, rb, port, kind, fold):
    fn, dt, comps = SUMS[kind]
    rng = np.random.default_rng(ord(kind) * 10 + fold)
    for dist, n, parts in [("loguniform", 40000, 7), ("illcond", 3001, 300), ("normal", 5, 9)]:
        x = gen_complex(dist, n, fold, dt) if comps == 2 else gen(dist, n, fold, dt)
        xr = as_real(x) if comps == 2 else x
        cuts = _cuts(n, parts, rng)
        per = len(binned_zeros(fold, kind))
        states = dev(cuda, binned_zeros(fold, kind, parts))
        for i in range(parts):
            rb.call(fn, fold, int(cuts[i + 1] - cuts[i]), dev(cuda, xr[comps * cuts[i]:]), 1,
                    states[i * per:(i + 1) * per])
        # a non-empty state to merge into
        pre = gen("normal", 4, n, np.float64 if dt in (np.float64, np.complex128) else np.float32)
        pre_c = np.repeat(pre, comps) if comps == 2 else pre
        out = dev(cuda, binned_zeros(fold, kind))
        rb.call(fn, fold, 4 // comps if comps == 2 else 4, dev(cuda, pre_c), 1, out)
        start = out.cpu().numpy()
        rb.call(MERGE[kind], fold, parts, states, out)
        got = out.cpu().numpy()
        # oracle: the same states merged one by one, in reverse order
        want = start.copy()
        hs = states.cpu().numpy()
        for i in reversed(range(parts)):
            getattr(port, PORT_ADD[kind])(fold, ptr(np.ascontiguousarray(hs[i * per:(i + 1) * per])),
                                          ptr(want))
        assert same_state(got, want, fold, comps), (kind, fold, dist)
        # and the whole vector reduced at once into the same starting state
        whole = dev(cuda, start)
        rb.call(fn, fold, n, dev(cuda, xr), 1, whole)
        assert same_state(got, whole.cpu().numpy(), fold, comps), (kind, fold, dist, "whole")


@pytest.mark.parametrize("kind", ["dsq", "ssq"])
@pytest.mark.parametrize("fold", [2, 3, 6])
def test_scaled_state_merge(cuda, rb, port, kind, fold):
    """[scale, state] records of the 2-norms' sums of squares: shard records merged on the GPU
    equal the whole vector's record (scale and state) and the oracle's scaled merges."""
    dt = np.float64 if kind == "dsq" else np.float32
    ssq = "binnedBLAS_dbdssq" if kind == "dsq" else "binnedBLAS_sbsssq"
    rng = np.random.default_rng(fold + (0 if kind == "dsq" else 50))
    big = "huge" if kind == "dsq" else "normal"   # FP32 has no finite "huge" inputs
    for dist, n, parts in [("loguniform", 30000, 5), (big, 2000, 17), ("tiny", 700, 3)]:
        x = gen(dist, n, fold, dt)
        cuts = _cuts(n, parts, rng)
        rec = 1 + 2 * fold
        recs = np.zeros(parts * rec, dt)
        for i in range(parts):
            z = dev(cuda, binned_zeros(fold, kind[0]))
            sc = rb.call(ssq, fold, int(cuts[i + 1] - cuts[i]), dev(cuda, x[cuts[i]:]), 1, 0.0, z)
            recs[i * rec] = sc
            recs[i * rec + 1:(i + 1) * rec] = z.cpu().numpy()
        out = dev(cuda, np.zeros(rec, dt))
        merge = "rb_dbdbaddsq_states" if kind == "dsq" else "rb_sbsbaddsq_states"
        rb.call(merge, fold, parts, dev(cuda, recs), out)
        got = out.cpu().numpy()
        # whole vector
        z = dev(cuda, binned_zeros(fold, kind[0]))
        sc = rb.call(ssq, fold, n, dev(cuda, x), 1, 0.0, z)
        assert same_value(dt(got[0]), dt(sc)), (kind, fold, dist)
        assert same_state(got[1:], z.cpu().numpy(), fold), (kind, fold, dist)
        # oracle scaled merges, in order
        body = np.zeros(2 * fold, dt)
        scale = 0.0
        add = port.dbdbaddsq if kind == "dsq" else port.sbsbaddsq
        for i in range(parts):
            r = np.ascontiguousarray(recs[i * rec + 1:(i + 1) * rec])
            scale = add(fold, float(recs[i * rec]), ptr(r), float(scale), ptr(body))
        assert same_value(dt(got[0]), dt(scale)) and same_state(got[1:], body, fold), (kind, fold, dist)


def test_merge_errors(cuda, rb):
    s = dev(cuda, np.zeros(12, np.float32))
    with pytest.raises(rb.ReproBLASError):
        rb.call("rb_cbcbadd_states", 22, 1, s, s)   # above binned_SBMAXFOLD
    with pytest.raises(rb.ReproBLASError):
        rb.call("rb_sbsbadd_states", 3, 1, np.zeros(6, np.float32), s)
    assert rb.call("rb_zbzbadd_states", 3, 0, None, None) == 0
