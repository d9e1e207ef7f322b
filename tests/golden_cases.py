"""Load the golden fixtures written by ``tests/golden/make_golden.py``.

The fixtures store plain arrays; this module rebuilds light stand-ins for the
reference's frozen dataclasses (``RadialGrid``, ``BoundOrbital``,
``ContinuumWave``) with the same attribute names, so a fixture can be passed
to the oracle and to the drop-in module unchanged.
"""
from __future__ import annotations

import glob
import json
import os
from dataclasses import dataclass

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@dataclass(frozen=True)
class Grid:
    r: np.ndarray
    dr: np.ndarray
    w_trapz: np.ndarray
    w_simpson: np.ndarray


@dataclass(frozen=True)
class BoundOrbital:
    l: int
    energy_au: float
    u_of_r: np.ndarray
    n_index: int


@dataclass(frozen=True)
class ContinuumWave:
    l: int
    k_au: float
    chi_of_r: np.ndarray
    phase_shift: float
    r_match: float = 0.0
    idx_match: int = -1
    eta: float = 0.0
    sigma_l: float = 0.0

    @property
    def u_of_r(self):
        return self.chi_of_r


def _wave(meta, chi):
    l, k, d, im, eta, sig = meta
    return ContinuumWave(l=int(l), k_au=float(k), chi_of_r=chi, phase_shift=float(d), idx_match=int(im),
                         eta=float(eta), sigma_l=float(sig))


def case_names():
    return sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "case_*.npz")))


def load_case(name):
    """Returns (common, calls): common holds grid/potential/bound objects; each call is a dict
    with positional args, kwargs and the reference outputs."""
    z = np.load(os.path.join(GOLDEN_DIR, f"case_{name}.npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    grid = Grid(r=z["r"], dr=z["dr"], w_trapz=z["w_trapz"], w_simpson=z["w_simpson"])
    bound_i = BoundOrbital(l=0, energy_au=-0.5, u_of_r=z["u_i"], n_index=1)
    if meta["bound_f_is_continuum"]:
        bound_f = _wave(meta["bound_f_meta"], z["u_f"])
    else:
        bound_f = BoundOrbital(l=1, energy_au=-0.125, u_of_r=z["u_f"], n_index=1)
    wi = {int(k): _wave(v, z[f"chi_i_{k}"]) for k, v in meta["waves_i"].items()}
    wf = {int(k): _wave(v, z[f"chi_f_{k}"]) for k, v in meta["waves_f"].items()}
    common = dict(grid=grid, V_core=z["V_core"], U_i=z["U_i"], U_f=z["U_f"], bound_i=bound_i, bound_f=bound_f,
                  waves_i=wi, waves_f=wf)
    calls = []
    for idx, c in enumerate(meta["calls"]):
        calls.append(dict(args=(grid, z["V_core"], z["U_i"], bound_i, bound_f, wi[c["li"]], wf[c["lf"]], c["L_max"]),
                          kwargs=dict(c["kw"], U_f_array=z["U_f"]), L_max=c["L_max"], li=c["li"], lf=c["lf"],
                          ref_dir=z[f"out_dir_{idx}"], ref_exc=z[f"out_exc_{idx}"], label=f"{name}[{idx}]"))
    return common, calls


def all_calls():
    out = []
    for n in case_names():
        out.extend(load_case(n)[1])
    return out


def rel_err(x, ref):
    x = np.asarray(x, dtype=float)
    ref = np.asarray(ref, dtype=float)
    return np.abs(x - ref) / np.maximum(np.abs(ref), 1e-300)
