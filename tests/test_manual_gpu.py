"""GPU parity of the manual-layout binnedBLAS forms (binnedBLAS_dmddot, zmzdotc, smsssq, ...):
the state held as a strided primary array and a strided carry array, in host or device memory,
ends with the bits of the corresponding ?b? form on the contiguous state, starting from a
non-empty state."""
import numpy as np
import pytest

from _cmp import same_state, same_value
from _data import gen, gen_complex

pytestmark = pytest.mark.gpu

# manual name -> (binned name, element kind of X, state kind, takes Y, sum of squares)
FORMS = {
    "dmdsum": ("dbdsum", "d", "d", False, False), "dmdasum": ("dbdasum", "d", "d", False, False),
    "dmdssq": ("dbdssq", "d", "d", False, True), "dmddot": ("dbddot", "d", "d", True, False),
    "zmzsum": ("zbzsum", "z", "z", False, False), "dmzasum": ("dbzasum", "z", "d", False, False),
    "dmzssq": ("dbzssq", "z", "d", False, True), "zmzdotu": ("zbzdotu", "z", "z", True, False),
    "zmzdotc": ("zbzdotc", "z", "z", True, False), "smssum": ("sbssum", "s", "s", False, False),
    "smsasum": ("sbsasum", "s", "s", False, False), "smsssq": ("sbsssq", "s", "s", False, True),
    "smsdot": ("sbsdot", "s", "s", True, False), "cmcsum": ("cbcsum", "c", "c", False, False),
    "smcasum": ("sbcasum", "c", "s", False, False), "smcssq": ("sbcssq", "c", "s", False, True),
    "cmcdotu": ("cbcdotu", "c", "c", True, False), "cmcdotc": ("cbcdotc", "c", "c", True, False),
}
REAL = {"d": np.float64, "z": np.float64, "s": np.float32, "c": np.float32}


def _vec(kind, n, seed):
    if kind in "dz":
        v = gen_complex("loguniform", n, seed) if kind == "z" else gen("loguniform", n, seed)
    else:
        v = gen_complex("normal", n, seed, np.complex64) if kind == "c" else gen("normal", n, seed, np.float32)
    return np.ascontiguousarray(v).view(REAL[kind])


@pytest.mark.parametrize("name", sorted(FORMS))
def test_manual_forms(cuda, rb, name):
    bname, xk, sk, has_y, ssq = FORMS[name]
    comps = 2 if sk in "zc" else 1
    rt = REAL[sk]
    for fold, n, (ip, ic), where in [(3, 5000, (2, 3), "host"), (4, 1001, (1, 2), "device"),
                                     (2, 17, (3, 1), "device"), (3, 0, (2, 2), "host")]:
        x = _vec(xk, n + 1, fold)
        y = _vec(xk, n + 1, fold + 1)
        # a non-empty starting state, produced by the binned form itself
        pre = _vec(xk, 9, 99)
        z0 = cuda.zeros(2 * fold * comps, dtype=cuda.float64 if rt == np.float64 else cuda.float32).cuda()
        pargs = [fold, 4, cuda.from_numpy(pre).cuda(), 1] + ([cuda.from_numpy(pre).cuda(), 1] if has_y else [])
        sc0 = rb.call("binnedBLAS_" + bname, *pargs, *([0.0] if ssq else []), z0)
        start = z0.cpu().numpy()
        # expected: the binned form on the contiguous state
        zw = cuda.from_numpy(start.copy()).cuda()
        args = [fold, n, cuda.from_numpy(x).cuda(), 1] + ([cuda.from_numpy(y).cuda(), 1] if has_y else [])
        sw = rb.call("binnedBLAS_" + bname, *args, *([sc0] if ssq else []), zw)
        want = zw.cpu().numpy()
        # the manual layout: primaries every ip-th element, carries every ic-th element
        pri = np.full(2 * fold * comps * ip + 4, 7.0, rt)
        car = np.full(2 * fold * comps * ic + 4, 7.0, rt)
        for i in range(fold):
            for c in range(comps):
                pri[comps * i * ip + c] = start[comps * i + c]
                car[comps * i * ic + c] = start[comps * fold + comps * i + c]
        if where == "device":
            dpri, dcar = cuda.from_numpy(pri).cuda(), cuda.from_numpy(car).cuda()
        else:
            dpri, dcar = pri, car
        sg = rb.call("binnedBLAS_" + name, *args, *([sc0] if ssq else []), dpri, ip, dcar, ic)
        hp = dpri.cpu().numpy() if where == "device" else dpri
        hc = dcar.cpu().numpy() if where == "device" else dcar
        got = np.zeros_like(start)
        for i in range(fold):
            for c in range(comps):
                got[comps * i + c] = hp[comps * i * ip + c]
                got[comps * fold + comps * i + c] = hc[comps * i * ic + c]
        assert same_state(got, want, fold, comps), (name, fold, n, where)
        if ssq:
            assert same_value(rt(sg), rt(sw)), (name, fold, n, where)
        # the elements between the strided entries are untouched
        mask_p = np.ones(len(pri), bool)
        mask_c = np.ones(len(car), bool)
        for i in range(fold):
            for c in range(comps):
                mask_p[comps * i * ip + c] = False
                mask_c[comps * i * ic + c] = False
        assert (hp[mask_p] == 7.0).all() and (hc[mask_c] == 7.0).all(), (name, "gaps")


def test_manual_errors(cuda, rb):
    s = np.zeros(12)
    with pytest.raises(rb.ReproBLASError):
        rb.call("binnedBLAS_dmdsum", 3, 4, np.ones(4), 1, s, 0, s, 1)
    with pytest.raises(rb.ReproBLASError):
        # fold above binned_DBMAXFOLD: rejected before the state is touched
        rb.call("binnedBLAS_zmzdotc", 53, 4, np.ones(8), 1, np.ones(8), 1, s, 1, s, 1)
