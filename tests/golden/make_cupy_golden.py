"""Generate golden I_L of the reference's CuPy path (``radial_ME_all_L_gpu``) on the CPU.

The reference's GPU entry point (``dwba_matrix_elements.py:1563-2549``) evaluates a different
quadrature from its CPU path: phase nodes with the un-adapted step (``:1362``), linear-in-r
interpolation (``cp.interp``, ``:1458``), the CC grid on r[:idx_limit] (``:1740``) and the kernel at
the CC nodes formed from interpolated 1/r_> and log-ratio (``:2072-2091``). To pin that semantics
without CuPy, this script puts a NumPy stand-in for the ``cupy`` module in ``sys.modules`` before
importing the reference (arrays gain ``.get()``; the memory pool and device queries answer
constants), runs ``radial_ME_all_L_gpu`` on the inputs of the CPU golden cases and stores its
outputs in ``cupy_semantics.npz`` beside the fixtures. Runs only where the reference source tree is
available (its directory in the environment variable ``DWBA_REFERENCE_PATH``, which must be set).

Usage:  python tests/golden/make_cupy_golden.py
"""
from __future__ import annotations

import json
import logging
import os
import sys
import types
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("DWBA_REFERENCE_PATH")
if not REF:
    sys.exit("set DWBA_REFERENCE_PATH to the reference source tree (the directory holding dwba_matrix_elements.py)")


class _Array(np.ndarray):
    """NumPy array with CuPy's ``.get()`` (device -> host copy)."""

    def get(self):
        return np.asarray(self)


def _wrap(fn):
    def g(*a, **k):
        out = fn(*a, **k)
        return out.view(_Array) if isinstance(out, np.ndarray) else out
    return g


def _cupy_standin() -> types.ModuleType:
    cp = types.ModuleType("cupy")
    cp.ndarray = _Array
    cp.float64 = np.float64
    cp.float32 = np.float32
    for name in ("asarray", "array", "zeros", "ones", "empty", "zeros_like", "maximum", "minimum", "exp", "log",
                 "power", "dot", "sum", "interp", "searchsorted", "clip", "sqrt", "abs", "where", "arange", "linspace",
                 "concatenate", "stack", "cumsum", "outer", "any", "all", "isfinite", "sin", "cos", "real", "imag"):
        setattr(cp, name, _wrap(getattr(np, name)))
    pool = SimpleNamespace(total_bytes=lambda: 0, used_bytes=lambda: 0, free_all_blocks=lambda: None)
    cp.get_default_memory_pool = lambda: pool
    cp.get_default_pinned_memory_pool = lambda: pool
    device = SimpleNamespace(mem_info=(64 << 30, 80 << 30), synchronize=lambda: None, id=0)
    cp.cuda = SimpleNamespace(Device=lambda *a, **k: device,
                              Stream=SimpleNamespace(null=SimpleNamespace(synchronize=lambda: None)),
                              runtime=SimpleNamespace(getDeviceCount=lambda: 1))
    return cp


sys.modules["cupy"] = _cupy_standin()
import scipy.special as _ss  # noqa: E402

if not hasattr(_ss, "sph_harm"):  # removed in SciPy 1.18; only the import needs it
    _ss.sph_harm = lambda m, n, phi, theta: _ss.sph_harm_y(n, m, theta, phi)
sys.path.insert(0, REF)
sys.path.insert(0, os.path.dirname(HERE))
logging.disable(logging.WARNING)

import dwba_matrix_elements as dme  # noqa: E402
from bound_states import BoundOrbital  # noqa: E402
from continuum import ContinuumWave  # noqa: E402
from grid import RadialGrid  # noqa: E402
import golden_cases as gc  # noqa: E402

assert dme.HAS_CUPY and dme.check_cupy_runtime()


def _ref_objects(common, call):
    g = common["grid"]
    grid = RadialGrid(r=g.r, dr=g.dr, w_trapz=g.w_trapz, w_simpson=g.w_simpson)
    bi = common["bound_i"]
    bound_i = BoundOrbital(l=bi.l, energy_au=bi.energy_au, u_of_r=bi.u_of_r, n_index=bi.n_index)
    bf = common["bound_f"]
    if isinstance(bf, gc.ContinuumWave):
        bound_f = ContinuumWave(l=bf.l, k_au=bf.k_au, chi_of_r=bf.chi_of_r, phase_shift=bf.phase_shift,
                                idx_match=bf.idx_match, eta=bf.eta, sigma_l=bf.sigma_l)
    else:
        bound_f = BoundOrbital(l=bf.l, energy_au=bf.energy_au, u_of_r=bf.u_of_r, n_index=bf.n_index)

    def wave(w):
        return ContinuumWave(l=w.l, k_au=w.k_au, chi_of_r=w.chi_of_r, phase_shift=w.phase_shift,
                             idx_match=w.idx_match, eta=w.eta, sigma_l=w.sigma_l)
    return grid, bound_i, bound_f, wave(call["args"][5]), wave(call["args"][6])


def main():
    out, labels = {}, []
    for name in gc.case_names():
        if name.startswith("large_grid"):
            continue  # the reference's GPU path materialises N x N_cc kernels: small cases only
        common, calls = gc.load_case(name)
        for idx, call in enumerate(calls):
            grid, bi, bf, ci, cf = _ref_objects(common, call)
            kw = {k: v for k, v in call["kwargs"].items() if k != "U_f_array"}
            res = dme.radial_ME_all_L_gpu(grid, common["V_core"], common["U_i"], bi, bf, ci, cf, call["L_max"],
                                          U_f_array=common["U_f"], **kw)
            L = call["L_max"]
            out[f"{name}_{idx}_dir"] = np.array([res.I_L_direct[l] for l in range(L + 1)])
            out[f"{name}_{idx}_exc"] = np.array([res.I_L_exchange[l] for l in range(L + 1)])
            labels.append(f"{name}_{idx}")
            print(f"  {name}[{idx}] done")
    out["labels_json"] = np.frombuffer(json.dumps(labels).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "cupy_semantics.npz"), **out)


if __name__ == "__main__":
    main()
