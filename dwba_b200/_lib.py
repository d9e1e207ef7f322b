"""ctypes binding of ``libdwba_b200.so`` (the C ABI in ``include/dwba_b200.h``).

The shared library is built in-tree by ``dwba_b200/build.py``. Loading fails
loudly: there is no CPU fallback for the engine.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdwba_b200.so")

DWBA_OK = 0
DWBA_ERR_INVALID_ARG = 1
DWBA_ERR_CUDA = 2
DWBA_ERR_NO_DEVICE = 3
DWBA_ERR_WORKSPACE = 4
DWBA_ERR_UNSUPPORTED = 5
DWBA_ERR_RANGE = 6
DWBA_MAX_L = 63

# Struct layouts (must match include/dwba_b200.h; checked against the library at load).
NODESET_DTYPE = np.dtype([(n, "<u8") for n in ("r", "logr", "breaks", "ta", "bx")]
                         + [(n, "<i4") for n in ("n_grid", "n1", "n_breaks", "log1", "log2", "pad")])
FOLD_DTYPE = np.dtype([(n, "<u8") for n in ("op", "f", "g", "out")]
                      + [(n, "<i4") for n in ("half_band", "n_out", "n_src", "n_clear")])
FORM_DTYPE = np.dtype([("r", "<u8"), ("a", "<u8"), ("b", "<u8"), ("n_rows", "<i4"), ("n_cols", "<i4")])
FORM_GRAD_DTYPE = np.dtype([("r", "<u8"), ("a", "<u8"), ("b", "<u8"), ("ga", "<u8"), ("gb", "<u8"),
                            ("n_rows", "<i4"), ("n_cols", "<i4")])
FOLD_ADJ_DTYPE = np.dtype([("op", "<u8"), ("y", "<u8"), ("z", "<u8"), ("half_band", "<i4"), ("n_out", "<i4"),
                           ("n_src", "<i4"), ("pad", "<i4")])
FOLD_MULTI = 8
FOLD_MULTI_DTYPE = np.dtype([("op", "<u8"), ("g", "<u8"), ("f", "<u8", (FOLD_MULTI,)), ("out", "<u8", (FOLD_MULTI,)),
                             ("n_f", "<i4"), ("half_band", "<i4"), ("n_out", "<i4"), ("n_src", "<i4"),
                             ("n_clear", "<i4"), ("pad", "<i4")])
POTENTIAL_DTYPE = np.dtype([("r", "<u8"), ("b", "<u8"), ("phi", "<u8"), ("n_rows", "<i4"), ("n_cols", "<i4"),
                            ("stride", "<i4"), ("pad", "<i4")])
DOT_DTYPE = np.dtype([("a", "<u8"), ("phi", "<u8"), ("out", "<u8"), ("n_rows", "<i4"), ("stride", "<i4")])
DOT_RUN = 16  # descriptors per run sharing one potential (dwba_dot_forms)
CUPY_SET_DTYPE = np.dtype([("r", "<u8"), ("logr", "<u8"), ("ops", "<u8"), ("n1", "<i4"), ("n_breaks", "<i4"),
                           ("L_max", "<i4"), ("pad", "<i4")])
CUPY_FORM_DTYPE = np.dtype([("r", "<u8"), ("a", "<u8"), ("f", "<u8"), ("g", "<u8"), ("ops", "<u8"), ("out", "<u8"),
                            ("n1", "<i4"), ("L_max", "<i4")])
TC_SEGMENT_DTYPE = np.dtype([("forms", "<u8"), ("r", "<u8"), ("out", "<u8"), ("n_forms", "<i4"), ("n_grid", "<i4")])
TC_TILE_DTYPE = np.dtype([("bn", "<i4"), ("stages", "<i4"), ("order", "<i4"), ("pad", "<i4")])
TAIL_DTYPE = np.dtype([("wave", "<f8", (10,)), ("r_m", "<f8"), ("r_max", "<f8"), ("moments", "<u8"), ("out", "<u8"),
                       ("mode", "<i4"), ("pad", "<i4")])


class DWBAError(RuntimeError):
    """Non-zero status from the C ABI."""

    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {status_string(status)} (status {status})")


_lib = None


def _declare(lib):
    c_int, c_i64, c_dbl, c_vp = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
    sig = {
        "dwba_abi_version": (c_int, []),
        "dwba_status_string": (ctypes.c_char_p, [c_int]),
        "dwba_device_probe": (c_int, [ctypes.POINTER(c_int)] * 3),
        "dwba_struct_sizes": (c_int, [ctypes.POINTER(c_i64), c_int]),
        "dwba_build_nodesets": (c_int, [c_vp, c_int, c_int, c_vp, c_vp, c_int, c_vp, c_vp]),
        "dwba_build_nodesets_folded": (c_int, [c_vp, c_vp, c_int, c_int, c_vp, c_vp, c_int, c_vp, c_vp]),
        "dwba_fold": (c_int, [c_vp, c_int, c_int, c_vp]),
        "dwba_dense_chunk_prefix": (c_i64, [c_vp, c_int, c_vp]),
        "dwba_bilinear_dense_fp64": (c_int, [c_vp, c_int, c_int, c_vp, c_vp, c_i64, c_vp, c_i64, c_vp, c_vp]),
        "dwba_bilinear_semisep_fp64": (c_int, [c_vp, c_int, c_int, c_vp, c_dbl, c_dbl, c_vp, c_vp]),
        "dwba_bilinear_semisep_abs_fp64": (c_int, [c_vp, c_int, c_int, c_vp, c_dbl, c_dbl, c_vp, c_vp]),
        "dwba_bilinear_dense_fp64_noalloc": (c_int, [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp]),
        "dwba_tc_workspace_bytes": (c_i64, [c_int, c_int, c_int, c_int]),
        "dwba_bilinear_tc_bf16": (c_int, [c_vp, c_int, c_vp, c_int, c_int, c_int, c_vp, c_vp, c_i64, c_vp, c_vp,
                                          c_vp]),
        "dwba_phase_breaks_coulomb": (c_int, [c_dbl, c_dbl, c_dbl, c_dbl, c_dbl, c_vp, c_int,
                                              ctypes.POINTER(c_int)]),
        "dwba_outer_tails": (c_int, [c_vp, c_dbl, c_dbl, c_int, c_vp, c_int, c_int, c_dbl, c_vp]),
        "dwba_outer_tails_batch": (c_int, [c_vp, c_int, c_int, c_int, c_dbl, c_vp]),
        "dwba_bilinear_semisep_backward_fp64": (c_int, [c_vp, c_int, c_int, c_vp, c_vp, c_dbl, c_dbl, c_vp]),
        "dwba_fold_adjoint": (c_int, [c_vp, c_int, c_int, c_vp]),
        "dwba_tc_backward_workspace_bytes": (c_i64, [c_int, c_int, c_int, c_int]),
        "dwba_bilinear_tc_bf16_backward": (c_int, [c_vp, c_int, c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_i64,
                                                   c_vp, c_vp]),
        "dwba_fold_multi": (c_int, [c_vp, c_int, c_int, c_vp]),
        "dwba_cross_sections": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_dbl,
                                        c_vp, c_vp, c_vp]),
        "dwba_outer_tail_on_device": (c_int, [c_vp, c_dbl, c_dbl]),
        "dwba_tc_set_wait_cycles": (c_int, [c_i64]),
        "dwba_multipole_potentials": (c_int, [c_vp, c_int, c_int, c_vp, c_dbl, c_dbl, c_vp]),
        "dwba_dot_forms": (c_int, [c_vp, c_int, c_int, c_vp]),
        "dwba_cupy_exchange_ops": (c_int, [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_int, c_vp]),
        "dwba_cupy_exchange_forms": (c_int, [c_vp, c_int, c_int, c_dbl, c_dbl, c_vp]),
        "dwba_tc_ragged_workspace_bytes": (c_i64, [c_vp, c_int, c_int, c_int, c_vp]),
        "dwba_bilinear_tc_bf16_ragged": (c_int, [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp]),
        "dwba_copy_from_host": (c_int, [c_vp, c_vp, c_i64, c_vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def load():
    """Load the library (once). Raises if it is missing or its ABI does not match."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m dwba_b200.build` "
                          "(the engine has no CPU fallback)")
    lib = _declare(ctypes.CDLL(LIB_PATH))
    if lib.dwba_abi_version() != 1:
        raise ImportError("libdwba_b200.so ABI version mismatch")
    sizes = (ctypes.c_int64 * 13)()
    lib.dwba_struct_sizes(sizes, 13)
    want = (NODESET_DTYPE.itemsize, FOLD_DTYPE.itemsize, FORM_DTYPE.itemsize, TAIL_DTYPE.itemsize,
            FORM_GRAD_DTYPE.itemsize, FOLD_ADJ_DTYPE.itemsize, FOLD_MULTI_DTYPE.itemsize,
            POTENTIAL_DTYPE.itemsize, DOT_DTYPE.itemsize, CUPY_SET_DTYPE.itemsize, CUPY_FORM_DTYPE.itemsize,
            TC_SEGMENT_DTYPE.itemsize, TC_TILE_DTYPE.itemsize)
    if tuple(sizes) != want:
        raise ImportError(f"struct layout mismatch: library {tuple(sizes)} vs binding {want}")
    _lib = lib
    return lib


def status_string(status: int) -> str:
    return load().dwba_status_string(int(status)).decode()


def check(status: int, where: str) -> None:
    if status != DWBA_OK:
        if status == DWBA_ERR_INVALID_ARG:
            raise ValueError(f"{where}: {status_string(status)}")
        raise DWBAError(status, where)


def device_ok() -> bool:
    """True when a usable sm_100 device is visible (the check_cupy_runtime analogue)."""
    lib = load()
    n, ma, mi = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    return lib.dwba_device_probe(ctypes.byref(n), ctypes.byref(ma), ctypes.byref(mi)) == DWBA_OK


def phase_breaks_coulomb(r_start, r_end, k_total, dphi, eta_total):
    lib = load()
    cap = 10010
    out = np.empty(cap, dtype=np.float64)
    n = ctypes.c_int(0)
    check(lib.dwba_phase_breaks_coulomb(float(r_start), float(r_end), float(k_total), float(dphi), float(eta_total),
                                        out.ctypes.data, cap, ctypes.byref(n)), "dwba_phase_breaks_coulomb")
    return out[:n.value].copy()


def tail_on_device(wave, r_m, r_max) -> bool:
    w = np.ascontiguousarray(wave, dtype=np.float64)
    return bool(load().dwba_outer_tail_on_device(w.ctypes.data, float(r_m), float(r_max)))


def outer_tails(wave, r_m, r_max, L_max, moments, mode, max_filon_segments, max_effective_dphi):
    lib = load()
    w = np.ascontiguousarray(wave, dtype=np.float64)
    m = np.ascontiguousarray(moments, dtype=np.float64)
    out = np.zeros(L_max + 1, dtype=np.float64)
    check(lib.dwba_outer_tails(w.ctypes.data, float(r_m), float(r_max), int(L_max), m.ctypes.data, int(mode),
                               int(max_filon_segments), float(max_effective_dphi), out.ctypes.data),
          "dwba_outer_tails")
    return out
