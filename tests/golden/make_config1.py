"""Config-1 fixture: H 1s->2p at 50 eV, N = 3000 on r in [1e-5, 200], l_i, l_f = 0..15, L = 0..4.

Runs only where the reference source tree is available (its directory in the environment
variable ``DWBA_REFERENCE_PATH``, which must be set). It builds the inputs with the reference's own solvers (exponential grid,
eigensolver bound states, static distorting potentials, distorted waves), evaluates
``radial_ME_all_L`` for all 128 parity-allowed pairs, and turns the integrals into amplitudes,
the DCS on 181 angles and the TCS with the reference's ``dwba_coupling`` and ``sigma_total``
(exactly as ``driver.py:1036-1052`` and ``:1255-1290`` do). Everything is stored in
``config1.npz``; ``tests/config1_tcs.py`` recomputes DCS/TCS from any set of I_L with the same
recipe.

Usage:  python tests/golden/make_config1.py
"""
from __future__ import annotations

import json
import logging
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("DWBA_REFERENCE_PATH")
if not REF:
    sys.exit("set DWBA_REFERENCE_PATH to the reference source tree (the directory holding dwba_matrix_elements.py)")

import scipy.special as _ss  # noqa: E402

if not hasattr(_ss, "sph_harm"):  # removed in SciPy 1.18; the reference still imports it
    _ss.sph_harm = lambda m, n, phi, theta: _ss.sph_harm_y(n, m, theta, phi)
sys.path.insert(0, REF)
logging.disable(logging.WARNING)

from grid import make_r_grid, k_from_E_eV  # noqa: E402
from potential_core import CorePotentialParams, V_core_on_grid  # noqa: E402
from bound_states import solve_bound_states  # noqa: E402
from distorting_potential import build_distorting_potentials  # noqa: E402
from continuum import solve_continuum_wave  # noqa: E402
import dwba_matrix_elements as dme  # noqa: E402
from dwba_coupling import calculate_amplitude_contribution  # noqa: E402
from sigma_total import dcs_dwba, integrate_dcs_over_angles  # noqa: E402

HARTREE_EV = 27.211386245988
L_MAX, LW = 4, 16


def tcs_from_integrals(theta, pairs, I_dir, I_exc, k_i, k_f, Li=0, Lf=1):
    """Amplitudes -> DCS -> TCS with the reference's coupling (driver.py:1036-1052, :1255-1290)."""
    amps = {(Mi, Mf): [np.zeros_like(theta, dtype=complex), np.zeros_like(theta, dtype=complex)]
            for Mi in range(-Li, Li + 1) for Mf in range(-Lf, Lf + 1)}
    for (li, lf), d, e in zip(pairs, I_dir, I_exc):
        dd = {L: float(d[L]) for L in range(len(d))}
        ee = {L: float(e[L]) for L in range(len(e))}
        for (Mi, Mf), acc in amps.items():
            a = calculate_amplitude_contribution(theta, dd, ee, li, lf, k_i, k_f, Li, Lf, Mi, Mf)
            acc[0] += a.f_theta
            acc[1] += a.g_theta
    dcs = np.zeros_like(theta)
    for (Mi, Mf), (f, g) in amps.items():
        dcs += dcs_dwba(theta, f, g, k_i, k_f, Li, 1)
    return dcs, integrate_dcs_over_angles(theta, dcs)


def main():
    N = 3000
    grid = make_r_grid(1e-5, 200.0, N)
    V = V_core_on_grid(grid, CorePotentialParams(Zc=1.0, a1=0, a2=0, a3=0, a4=0, a5=0, a6=0))
    o1s = solve_bound_states(grid, V, l=0, n_states_max=2)[0]
    o2p = solve_bound_states(grid, V, l=1, n_states_max=2)[0]
    E = 50.0
    Ef = E - (o2p.energy_au - o1s.energy_au) * HARTREE_EV
    k_i, k_f = float(k_from_E_eV(E)), float(k_from_E_eV(Ef))
    Ui, Uf = build_distorting_potentials(grid, V, o1s, o2p, k_i, k_f)
    wi = {l: solve_continuum_wave(grid, Ui, l, E, 0.0) for l in range(LW)}
    wf = {l: solve_continuum_wave(grid, Uf, l, Ef, 0.0) for l in range(LW)}
    pairs = [(li, lf) for li in range(LW) for lf in range(LW) if (li + lf) % 2 == 1]
    only = int(os.environ.get("CONFIG1_PAIRS", "0")) or len(pairs)
    I_dir = np.zeros((len(pairs), L_MAX + 1))
    I_exc = np.zeros((len(pairs), L_MAX + 1))
    t0 = time.perf_counter()
    for n, (li, lf) in enumerate(pairs[:only]):
        res = dme.radial_ME_all_L(grid, V, Ui.U_of_r, o1s, o2p, wi[li], wf[lf], L_MAX, U_f_array=Uf.U_of_r)
        I_dir[n] = [res.I_L_direct[L] for L in range(L_MAX + 1)]
        I_exc[n] = [res.I_L_exchange[L] for L in range(L_MAX + 1)]
        if n % 16 == 0:
            print(f"  pair {n}/{len(pairs)} ({li},{lf}) {time.perf_counter() - t0:.0f}s", flush=True)
    ref_seconds = time.perf_counter() - t0
    theta = np.linspace(0.0, np.pi, 181)
    dcs, tcs = tcs_from_integrals(theta, pairs[:only], I_dir[:only], I_exc[:only], k_i, k_f)
    meta = dict(E=E, Ef=Ef, k_i=k_i, k_f=k_f, pairs=pairs[:only], L_max=L_MAX, ref_seconds=ref_seconds,
                waves_i={l: [w.l, w.k_au, w.phase_shift, w.idx_match, w.eta, w.sigma_l] for l, w in wi.items()},
                waves_f={l: [w.l, w.k_au, w.phase_shift, w.idx_match, w.eta, w.sigma_l] for l, w in wf.items()})
    arrays = dict(r=grid.r, w_simpson=grid.w_simpson, w_trapz=grid.w_trapz, dr=grid.dr, V_core=V, U_i=Ui.U_of_r,
                  U_f=Uf.U_of_r, u_i=o1s.u_of_r, u_f=o2p.u_of_r, I_dir=I_dir[:only], I_exc=I_exc[:only], dcs=dcs,
                  tcs=np.array([tcs]), theta=theta,
                  chi_i=np.stack([wi[l].chi_of_r for l in range(LW)]),
                  chi_f=np.stack([wf[l].chi_of_r for l in range(LW)]))
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "config1.npz"), **arrays)
    print(f"config1: {only} pairs, reference {ref_seconds:.1f}s, TCS {tcs:.6e} a.u.")


if __name__ == "__main__":
    main()
