"""The C-ABI library loads and exports every entry point declared in include/dwba_b200.h."""
import ctypes
import os
import re

import numpy as np

from dwba_b200 import _lib

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "dwba_b200.h")


def declared_symbols():
    text = open(HDR).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dwba_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), s


def test_abi_version_and_struct_layout():
    lib = _lib.load()
    assert lib.dwba_abi_version() == 1
    sizes = (ctypes.c_int64 * 13)()
    assert lib.dwba_struct_sizes(sizes, 13) == 0
    assert tuple(sizes) == (_lib.NODESET_DTYPE.itemsize, _lib.FOLD_DTYPE.itemsize, _lib.FORM_DTYPE.itemsize,
                            _lib.TAIL_DTYPE.itemsize, _lib.FORM_GRAD_DTYPE.itemsize, _lib.FOLD_ADJ_DTYPE.itemsize,
                            _lib.FOLD_MULTI_DTYPE.itemsize, _lib.POTENTIAL_DTYPE.itemsize, _lib.DOT_DTYPE.itemsize,
                            _lib.CUPY_SET_DTYPE.itemsize, _lib.CUPY_FORM_DTYPE.itemsize,
                            _lib.TC_SEGMENT_DTYPE.itemsize, _lib.TC_TILE_DTYPE.itemsize)


def test_status_strings():
    for s in range(7):
        assert _lib.status_string(s)


def test_invalid_args_rejected_without_gpu_work():
    lib = _lib.load()
    # null descriptors / bad sizes are rejected before any launch
    assert lib.dwba_build_nodesets(None, 1, 10, None, None, 5, None, None) == _lib.DWBA_ERR_INVALID_ARG
    assert lib.dwba_fold(None, 1, 10, None) == _lib.DWBA_ERR_INVALID_ARG
    assert lib.dwba_bilinear_semisep_fp64(None, 1, 4, None, 1e-5, 200.0, None, None) == _lib.DWBA_ERR_INVALID_ARG
    ds = np.ones(70)
    assert lib.dwba_bilinear_dense_fp64(None, 1, 99, ds.ctypes.data, None, 1, None, 0, None, None) \
        == _lib.DWBA_ERR_INVALID_ARG
    m = np.array([1000, 300], dtype=np.int32)
    pre = np.zeros(3, dtype=np.int64)
    assert lib.dwba_dense_chunk_prefix(m.ctypes.data, 2, pre.ctypes.data) == 4 + 2
    assert list(pre) == [0, 4, 6]


def test_tensor_core_backward_host_checks():
    """The split-BF16 backward's workspace query and argument checks run on the host."""
    lib = _lib.load()
    assert lib.dwba_tc_backward_workspace_bytes(10, 1, 4, 2) == -1  # grid too short
    assert lib.dwba_tc_backward_workspace_bytes(10, 100, 4, 4) == -1  # 2 or 3 terms only
    # more forms, more grid points or more multipoles never need less workspace
    base = lib.dwba_tc_backward_workspace_bytes(300, 3001, 6, 2)
    assert base > 0 and base % 256 == 0
    assert lib.dwba_tc_backward_workspace_bytes(600, 3001, 6, 2) > base
    assert lib.dwba_tc_backward_workspace_bytes(300, 6001, 6, 2) > base
    assert lib.dwba_tc_backward_workspace_bytes(300, 3001, 9, 2) > base
    assert lib.dwba_tc_backward_workspace_bytes(300, 3001, 6, 3) > base
    # the gradient partials alone: (L_max+1) x padded forms x padded grid doubles
    assert base >= 7 * 512 * 3008 * 8
    ds = np.ones(7)
    assert lib.dwba_bilinear_tc_bf16_backward(None, 1, None, 3001, 6, 2, ds.ctypes.data, None, None, 0, None,
                                              None) == _lib.DWBA_ERR_INVALID_ARG
    assert lib.dwba_bilinear_tc_bf16_backward(None, 0, None, 3001, 6, 2, ds.ctypes.data, None, None, 0, None,
                                              None) == _lib.DWBA_OK  # nothing to do


def test_ragged_tensor_core_host_checks():
    """Workspace of the ragged split-BF16 launch: the segments' B terms share one matrix as wide as
    the largest grid, then each segment's tables; invalid tiles and sizes are rejected on the host."""
    lib = _lib.load()
    segs = np.zeros(3, dtype=_lib.TC_SEGMENT_DTYPE)
    segs["n_forms"] = [300, 0, 1000]
    segs["n_grid"] = [2000, 5000, 15000]
    tile = np.zeros(1, dtype=_lib.TC_TILE_DTYPE)

    def ws(bn=0, stages=0, order=0, nt=2, L=6, s=segs):
        tile["bn"], tile["stages"], tile["order"] = bn, stages, order
        return lib.dwba_tc_ragged_workspace_bytes(s.ctypes.data, len(s), L, nt, tile.ctypes.data)
    base = ws()
    assert base > 0 and base % 256 == 0
    # the B terms alone: 2 terms x (300 + 1000 forms padded to 256) rows x 15040 columns of bf16
    assert base >= 2 * (512 + 1024) * 15040 * 2
    assert lib.dwba_tc_ragged_workspace_bytes(segs.ctypes.data, 3, 6, 2, None) == base  # NULL tile = default
    assert ws(bn=128) < base  # less padding of the form blocks
    assert ws(bn=128, stages=4) == ws(bn=128, stages=3)  # the depth does not change the workspace
    for bad in (dict(bn=64), dict(bn=256, stages=4), dict(bn=256, stages=2), dict(order=2),
                dict(nt=3, bn=256, stages=3), dict(nt=4)):
        assert ws(**bad) == -1, bad
    assert ws(nt=3, bn=256, stages=2) > 0 and ws(nt=3, bn=128, stages=3) > 0
    short = segs.copy()
    short["n_grid"][0] = 1
    assert ws(s=short) == -1
    ds = np.ones(7)
    assert lib.dwba_bilinear_tc_bf16_ragged(segs.ctypes.data, 3, 6, 2, None, ds.ctypes.data, None, 0, None,
                                            None) == _lib.DWBA_ERR_INVALID_ARG
    assert lib.dwba_bilinear_tc_bf16_ragged(segs.ctypes.data, 0, 6, 2, None, ds.ctypes.data, None, 0, None,
                                            None) == _lib.DWBA_OK  # nothing to do
