"""The method of the BLAS1 sweep parity test, checked on the CPU at small sizes: for every
routine, fold and distribution of the sweep, the reference's accumulating prefix pass gives,
at every prefix, the same state, scale and value as a single call over that prefix, and the
oracle restatement gives the same bits as the reference. (The GPU sweep test relies on the
first property to get the reference's result for every N from one pass.)"""
import pytest

from _cmp import same_state, same_value
from _ffi import ref
from _sweep import DISTS, FOLDS, GROUPS, SSQ, group_inputs, reference_prefixes
from _sweep import comps as sweep_comps

LOGN_SMALL = [10, 12, 14, 16]


@pytest.mark.parametrize("group", list(GROUPS))
@pytest.mark.parametrize("dist", DISTS)
def test_prefix_pass_equals_single_calls(port, dist, group):
    x, y = group_inputs(dist, group, 1 << LOGN_SMALL[-1])
    R = ref()
    libs = [port] + ([R] if R is not None else [])
    for r in GROUPS[group]:
        comps = sweep_comps(r)
        for f in FOLDS:
            passes = []
            for L in libs:
                pre = reference_prefixes(L, r, f, x, y, LOGN_SMALL)
                for lg in LOGN_SMALL:
                    st, scl, val = reference_prefixes(L, r, f, x, y, [lg])[lg]
                    pst, pscl, pval = pre[lg]
                    assert same_state(pst, st, f, comps), (r, f, lg)
                    assert pscl == scl and same_value(pval, val), (r, f, lg)
                passes.append(pre)
            if len(passes) == 2:
                for lg in LOGN_SMALL:
                    a, b = passes[0][lg], passes[1][lg]
                    assert same_state(a[0], b[0], f, comps) and a[1] == b[1], (r, f, lg)
                    assert same_value(a[2], b[2]), (r, f, lg)
