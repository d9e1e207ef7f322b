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
    sizes = (ctypes.c_int64 * 11)()
    assert lib.dwba_struct_sizes(sizes, 11) == 0
    assert tuple(sizes) == (_lib.NODESET_DTYPE.itemsize, _lib.FOLD_DTYPE.itemsize, _lib.FORM_DTYPE.itemsize,
                            _lib.TAIL_DTYPE.itemsize, _lib.FORM_GRAD_DTYPE.itemsize, _lib.FOLD_ADJ_DTYPE.itemsize,
                            _lib.FOLD_MULTI_DTYPE.itemsize, _lib.POTENTIAL_DTYPE.itemsize, _lib.DOT_DTYPE.itemsize,
                            _lib.CUPY_SET_DTYPE.itemsize, _lib.CUPY_FORM_DTYPE.itemsize)


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
