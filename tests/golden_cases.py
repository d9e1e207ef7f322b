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


def levin_condition(w, r_m, r_max):
    """Largest condition number of the 8-node Levin collocation systems a record solves (0 when
    both phase branches take Filon). The reference builds them with the differentiation matrix of
    descending Chebyshev points on ascending nodes (oscillatory_integrals.py:970-1095); these
    systems reach condition numbers of 1e10, so two correct LU solves agree only to ~1e-16 cond."""
    ka, la, _, ea, _, kb, lb, _, eb, _ = w
    n = 8
    x = np.cos(np.pi * np.arange(n) / (n - 1))
    c = np.ones(n)
    c[0] = c[-1] = 2.0
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            if i != j:
                D[i, j] = (c[i] / c[j]) * (-1.0) ** (i + j) / (x[i] - x[j])
        D[i, i] = -D[i].sum()
    worst = 0.0
    for sgn in (-1, 1):
        def d1(r):
            v = (ka - kb if sgn < 0 else ka + kb) + ea / r + (-eb / r if sgn < 0 else eb / r)
            v = v + la * (la + 1) / (2 * ka * r * r)
            t = lb * (lb + 1) / (2 * kb * r * r)
            return v - t if sgn < 0 else v + t

        def d2(r):
            v = -ea / r ** 2 + (eb / r ** 2 if sgn < 0 else -eb / r ** 2) - la * (la + 1) / (ka * r ** 3)
            t = lb * (lb + 1) / (kb * r ** 3)
            return v + t if sgn < 0 else v - t
        mid = (r_m + r_max) / 2
        h = np.pi / 4 / abs(d1(mid))
        if abs(d2(mid)) * h * h < 0.1:
            continue
        bnd = np.linspace(r_m, r_max, int(max(1, np.ceil((r_max - r_m) / h))) + 1)
        for a, b in zip(bnd[:-1], bnd[1:]):
            xs = 0.5 * (b - a) * (x[::-1] + 1) + a
            worst = max(worst, np.linalg.cond(D * (2 / (xs[-1] - xs[0])) + np.diag(1j * d1(xs))))
    return worst


def fullsize_batch_inputs():
    """Kernel-batch inputs at full size: N = 15000 on [1e-5, 400], the benchmark's four bound pairs
    and 16 continuum pairs over l = 0..63, k = 0.5..8 (the extremes included), seeded."""
    import bench
    g = bench.make_grid(15000, 1e-5, 400.0)
    r = g.r
    _, zeros, bounds, _ = bench.make_workload(15000, n_cont=1)
    rng = np.random.default_rng(101)
    picks = [((0, 0.5), (63, 8.0)), ((63, 0.5), (0, 8.0)), ((63, 8.0), (63, 8.0)), ((0, 0.5), (0, 0.5)),
             ((1, 8.0), (62, 0.5)), ((31, 4.0), (32, 4.25)), ((0, 8.0), (0, 8.0)), ((63, 0.5), (63, 0.5))]
    while len(picks) < 16:
        picks.append(((int(rng.integers(0, 64)), float(rng.uniform(0.5, 8.0))),
                      (int(rng.integers(0, 64)), float(rng.uniform(0.5, 8.0)))))
    pairs = []
    for pi in picks:
        w = []
        for l, k in pi:
            d = float(rng.uniform(0.0, np.pi))
            chi = np.sin(k * r - 0.5 * l * np.pi + d) * (1.0 - np.exp(-(r / ((l + 1) / k)) ** (l + 1)))
            w.append(bench._Wave(l, k, d, chi))
        pairs.append(tuple(w))
    return g, zeros, bounds, pairs
