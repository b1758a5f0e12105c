"""The C ABI library loads without a GPU and exports every entry point that
include/vbd_b200.h declares (no compute calls here)."""
import ctypes
import os
import re

import numpy as np
import pytest

from warpvbd_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "vbd_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(vbd_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_bound_functions():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_library_is_built_for_sm100a():
    # the fatbinary's ELF carries the target name in its note section
    data = open(_lib.LIB_PATH, "rb").read()
    assert b"sm_100a" in data


def test_status_strings_and_no_device_paths():
    L = _lib.load()
    assert L.vbd_version() >= 1
    assert L.vbd_status_string(_lib.ERR_NONFINITE) == b"non-finite value"
    # argument validation happens before any device work
    h = ctypes.c_void_p()
    X = np.zeros((4, 3))
    st = L.vbd_create(_lib.ptr(X, "d"), 0, None, 0, None, None, None, None, 0.0, None, None,
                      0, 0, 0, 0, ctypes.byref(h))
    assert st == _lib.ERR_INVALID_ARG
    tets = np.array([[0, 1, 2, 9]], np.int32)
    one = np.ones(1)
    st = L.vbd_create(_lib.ptr(X, "d"), 4, _lib.ptr(tets, "i"), 1, _lib.ptr(one, "d"),
                      _lib.ptr(one, "d"), _lib.ptr(one * 0.3, "d"), None, 0.0, None, None, 0, 0, 0,
                      0, ctypes.byref(h))
    assert st == _lib.ERR_INVALID_ARG
    assert b"out of range" in L.vbd_last_error_message()


def test_native_coloring_rejects_more_than_256_colours():
    from warpvbd_b200.coloring import color_tets
    import pytest
    # 260 vertices all sharing tets with vertex 0..2 -> a clique through shared tets
    n = 262
    tets = np.array([[i, j, k, l] for i, j, k, l in
                     [(a, a + 1, a + 2, a + 3) for a in range(0, n - 3)]], np.int32)
    color_tets(tets)   # a path of tets needs only 4 colours
    big = []
    for a in range(n):
        for b in range(a + 1, n, 37):
            big.append([a, b, (b + 1) % n, (b + 2) % n])
    big = np.array([t for t in big if len(set(t)) == 4], np.int32)
    col = None
    try:
        col = color_tets(big)
    except AssertionError as e:
        assert "Exceeded maximum number of colors" in str(e)
    if col is not None:
        assert col.max() < 256
    with pytest.raises(Exception):
        color_tets(np.array([[0, 1, 2, -5]], np.int32))


def test_cluster_flags_refuse_out_of_range_sizes():
    """The cluster field is 5 bits wide: 0 (automatic) and 1..16 are shifted
    in, anything else is refused before it can spill into other bits."""
    assert _lib.cluster_flags(0) == 0
    assert _lib.cluster_flags(16) == 16 << _lib.CLUSTER_SHIFT
    for bad in (17, 32, 48, -1, 2.5):
        with pytest.raises(ValueError, match="cluster must be"):
            _lib.cluster_flags(bad)
