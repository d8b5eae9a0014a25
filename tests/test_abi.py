"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares; the ctypes table matches the header."""
import ctypes
import glob
import os
import re

from fmm3dbie_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(re.findall(r"\b(bie_\w+)\s*\(", txt))
    return names


def test_library_exports_header_symbols(built):
    lib = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_table_matches_header(built):
    assert _declared() == set(L.exported_symbols())


def test_version_and_errors(built):
    lib = L.lib()
    assert b"sm_100a" in lib.bie_version()
    npols = L.I64()
    assert lib.bie_get_npols(1, 4, ctypes.byref(npols)) == 0 and npols.value == 15
    assert lib.bie_get_npols(11, 5, ctypes.byref(npols)) == 0 and npols.value == 36
    assert lib.bie_get_npols(7, 5, ctypes.byref(npols)) != 0


def test_bad_arguments_are_reported(built, sphere4, sphere_lap_setup):
    """Host-side validation: a corrupted near list is rejected with a status,
    before anything reaches a device."""
    import numpy as np
    from fmm3dbie_b200 import layer, BieError
    from fmm3dbie_b200.surface import NearField
    st = sphere_lap_setup
    bad = NearField(st.near.row_ptr.copy(), st.near.col_ind.copy(), st.near.iquad.copy(),
                    st.near.wnear)
    bad.col_ind[5] = sphere4.npatches + 7
    try:
        layer.lpcomp_lap_comb_dir_addsub(sphere4, 1e-6, (1.0, 1.0), bad, st.over,
                                         np.zeros(sphere4.npts))
    except BieError as e:
        assert e.status in (1, 2)  # 2 only when no CUDA device is present to query
    else:
        raise AssertionError("corrupted col_ind accepted")
