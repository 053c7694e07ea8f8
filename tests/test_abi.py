"""The C-ABI library loads, exports every function include/reproblas_b200.h declares, and
reports argument errors through its error channel (no GPU needed for these)."""
import math
import subprocess

import numpy as np


def test_library_exports_header(rb):
    names = rb.exported_symbols()
    assert "reproBLAS_rddot" in names and "binnedBLAS_dbddot" in names
    out = subprocess.run(["nm", "-D", "--defined-only", rb.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    defined = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = [n for n in names if n not in defined]
    assert not missing, missing


def test_python_signatures_cover_header(rb):
    missing = [n for n in rb.exported_symbols() if n not in rb.SIGNATURES]
    assert not missing, missing


def test_invalid_fold_sets_error(rb):
    x = np.ones(4)
    rb.lib.rb_clear_error()
    v = rb.lib.reproBLAS_rddot(1, 4, x.ctypes.data, 1, x.ctypes.data, 1)
    assert math.isnan(v)
    assert rb.lib.rb_get_last_error() == 1
    assert b"fold" in rb.lib.rb_get_last_error_message()
    rb.lib.rb_clear_error()
    # binned_DBMAXFOLD = 52 and binned_SBMAXFOLD = 21 are the largest folds
    v = rb.lib.reproBLAS_rdsum(53, 4, x.ctypes.data, 1)
    assert math.isnan(v) and rb.lib.rb_get_last_error() == 1
    rb.lib.rb_clear_error()
    v = rb.lib.reproBLAS_rssum(22, 4, x.astype(np.float32).ctypes.data, 1)
    assert math.isnan(v) and rb.lib.rb_get_last_error() == 1
    rb.lib.rb_clear_error()


def test_negative_stride_sets_error(rb):
    x = np.ones(4)
    rb.lib.rb_clear_error()
    v = rb.lib.reproBLAS_rdsum(3, 4, x.ctypes.data, -1)
    assert math.isnan(v) and rb.lib.rb_get_last_error() == 1
    rb.lib.rb_clear_error()


def test_launch_config_validation(rb):
    rb.lib.rb_clear_error()
    rb.lib.rb_set_launch_config(2, 100)
    assert rb.lib.rb_get_last_error() == 1
    rb.lib.rb_clear_error()
    rb.lib.rb_set_launch_config(0, 0)
    assert rb.lib.rb_get_last_error() == 0


def test_version(rb):
    assert "sm_100a" in rb.version()


def test_every_reference_blas_entry_point_is_exported(rb):
    """Every function include/reproBLAS.h and include/binnedBLAS.h of the reference declare is
    declared (and, by test_library_exports_header, exported) here under the same name."""
    import os
    import re
    import pytest
    from _ffi import reference_tree
    tree = reference_tree()
    if tree is None:
        pytest.skip("reference source tree not present")
    REF_INCLUDE = os.path.join(tree, "include")
    ref = set()
    for h in ("reproBLAS.h", "binnedBLAS.h"):
        text = open(os.path.join(REF_INCLUDE, h)).read()
        ref |= set(re.findall(r"\b((?:reproBLAS|binnedBLAS)_\w+)\s*\(", text))
    ours = set(rb.exported_symbols())
    missing = sorted(ref - ours)
    assert len(ref) >= 100 and not missing, missing
