"""Generate the golden I_L fixtures by running the reference implementation.

This script runs only where the reference source tree is available (it is
imported from the directory named by the environment variable ``DWBA_REFERENCE_PATH``,
which must be set). It writes
small ``.npz`` fixtures next to itself; the tests read those fixtures and never
touch the reference.

Each fixture holds every input that ``dwba_matrix_elements.radial_ME_all_L``
receives (grid arrays, potentials, bound orbitals, continuum waves and their
scalar metadata), the call keyword arguments, and the reference outputs
``I_L_direct`` / ``I_L_exchange``. Unit fixtures pin the quadrature pieces
(Clenshaw-Curtis reference weights, phase nodes, adaptive phase increment,
log-grid interpolation, outer tails).

Usage:  python tests/golden/make_golden.py
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

if not hasattr(_ss, "sph_harm"):  # removed in SciPy 1.18; only the import needs it
    _ss.sph_harm = lambda m, n, phi, theta: _ss.sph_harm_y(n, m, theta, phi)
sys.path.insert(0, REF)
logging.disable(logging.WARNING)

from grid import make_r_grid, k_from_E_eV  # noqa: E402
from potential_core import CorePotentialParams, V_core_on_grid  # noqa: E402
from bound_states import solve_bound_states, BoundOrbital  # noqa: E402
from distorting_potential import build_distorting_potentials  # noqa: E402
from continuum import solve_continuum_wave, ContinuumWave  # noqa: E402
import dwba_matrix_elements as dme  # noqa: E402
import oscillatory_integrals as oi  # noqa: E402

HARTREE_EV = 27.211386245988


def _wave_meta(c: ContinuumWave) -> list:
    return [int(c.l), float(c.k_au), float(c.phase_shift), int(c.idx_match),
            float(c.eta), float(c.sigma_l)]


def _save_case(name, grid, V, Ui, Uf, u_i, u_f, f_is_cont, f_meta, waves_i, waves_f, calls):
    """Store one fixture: inputs, per-call kwargs and reference outputs."""
    arrays = dict(r=grid.r, w_simpson=grid.w_simpson, w_trapz=grid.w_trapz, dr=grid.dr,
                  V_core=V, U_i=Ui, U_f=Uf, u_i=u_i, u_f=u_f)
    meta = {"name": name, "bound_f_is_continuum": bool(f_is_cont), "bound_f_meta": f_meta,
            "waves_i": {}, "waves_f": {}, "calls": []}
    for l, c in waves_i.items():
        arrays[f"chi_i_{l}"] = c.chi_of_r
        meta["waves_i"][str(l)] = _wave_meta(c)
    for l, c in waves_f.items():
        arrays[f"chi_f_{l}"] = c.chi_of_r
        meta["waves_f"][str(l)] = _wave_meta(c)
    for idx, call in enumerate(calls):
        li, lf, L_max, kw = call["li"], call["lf"], call["L_max"], call["kw"]
        bound_i = BoundOrbital(l=0, energy_au=-0.5, u_of_r=u_i, n_index=1)
        if f_is_cont:
            bound_f = ContinuumWave(l=f_meta[0], k_au=f_meta[1], chi_of_r=u_f, phase_shift=f_meta[2],
                                    idx_match=f_meta[3], eta=f_meta[4], sigma_l=f_meta[5])
        else:
            bound_f = BoundOrbital(l=1, energy_au=-0.125, u_of_r=u_f, n_index=1)
        t0 = time.perf_counter()
        res = dme.radial_ME_all_L(grid, V, Ui, bound_i, bound_f, waves_i[li], waves_f[lf], L_max,
                                  U_f_array=Uf, **kw)
        dt = time.perf_counter() - t0
        arrays[f"out_dir_{idx}"] = np.array([res.I_L_direct[L] for L in range(L_max + 1)])
        arrays[f"out_exc_{idx}"] = np.array([res.I_L_exchange[L] for L in range(L_max + 1)])
        meta["calls"].append({"li": li, "lf": lf, "L_max": L_max, "kw": kw, "ref_seconds": dt})
        print(f"  {name} call {idx} (li={li}, lf={lf}, kw={kw}) {dt:.2f}s")
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, f"case_{name}.npz"), **arrays)


def case_h_excitation():
    """H 1s->2p at 50 eV, solver-produced waves (analytic bypass, idx_limit = N)."""
    N = 1001
    grid = make_r_grid(1e-5, 200.0, N)
    V = V_core_on_grid(grid, CorePotentialParams(Zc=1.0, a1=0, a2=0, a3=0, a4=0, a5=0, a6=0))
    o1s = solve_bound_states(grid, V, l=0, n_states_max=2)[0]
    o2p = solve_bound_states(grid, V, l=1, n_states_max=2)[0]
    E = 50.0
    Ef = E - (o2p.energy_au - o1s.energy_au) * HARTREE_EV
    ki, kf = float(k_from_E_eV(E)), float(k_from_E_eV(Ef))
    Ui, Uf = build_distorting_potentials(grid, V, o1s, o2p, ki, kf)
    ls = [0, 1, 2, 5, 6, 8, 9]
    wi = {l: solve_continuum_wave(grid, Ui, l, E, 0.0) for l in ls}
    wf = {l: solve_continuum_wave(grid, Uf, l, Ef, 0.0) for l in ls}
    calls = [dict(li=0, lf=1, L_max=4, kw={}), dict(li=1, lf=2, L_max=4, kw={}),
             dict(li=2, lf=1, L_max=4, kw={}), dict(li=5, lf=6, L_max=4, kw={}),
             dict(li=9, lf=8, L_max=4, kw={}),
             dict(li=6, lf=5, L_max=4, kw={"oscillatory_method": "legacy"}),
             dict(li=0, lf=1, L_max=4, kw={"oscillatory_method": "full_split"}),
             dict(li=1, lf=0, L_max=4, kw={"use_oscillatory_quadrature": False}),
             dict(li=8, lf=9, L_max=6, kw={"CC_nodes": 7, "phase_increment": 1.0})]
    _save_case("h_1s2p_50eV", grid, V, Ui.U_of_r, Uf.U_of_r, o1s.u_of_r, o2p.u_of_r,
               False, None, wi, wf, calls)


def case_heplus_ionic():
    """He+ 1s->2s at 100 eV: Coulomb waves (eta != 0), idx_limit < N, outer tails active."""
    N = 1201
    grid = make_r_grid(1e-5, 120.0, N)
    V = V_core_on_grid(grid, CorePotentialParams(Zc=2.0, a1=0, a2=0, a3=0, a4=0, a5=0, a6=0))
    o1s = solve_bound_states(grid, V, l=0, n_states_max=3)[0]
    o2s = solve_bound_states(grid, V, l=0, n_states_max=3)[1]
    E = 100.0
    Ef = E - (o2s.energy_au - o1s.energy_au) * HARTREE_EV
    ki, kf = float(k_from_E_eV(E)), float(k_from_E_eV(Ef))
    Ui, Uf = build_distorting_potentials(grid, V, o1s, o2s, ki, kf)
    ls = [0, 1, 2, 3, 6]
    wi = {l: solve_continuum_wave(grid, Ui, l, E, 1.0) for l in ls}
    wf = {l: solve_continuum_wave(grid, Uf, l, Ef, 1.0) for l in ls}
    calls = [dict(li=0, lf=0, L_max=6, kw={}), dict(li=1, lf=1, L_max=6, kw={}),
             dict(li=2, lf=0, L_max=6, kw={}), dict(li=3, lf=1, L_max=6, kw={}),
             dict(li=6, lf=6, L_max=6, kw={}),
             dict(li=1, lf=3, L_max=6, kw={"oscillatory_method": "legacy"}),
             dict(li=0, lf=2, L_max=4, kw={"use_oscillatory_quadrature": False})]
    _save_case("heplus_1s2s_100eV", grid, V, Ui.U_of_r, Uf.U_of_r, o1s.u_of_r, o2s.u_of_r,
               False, None, wi, wf, calls)


def case_ionization():
    """H 1s ionization at 100 eV: bound_f is an ejected Coulomb wave (no tails, L=0 correction on)."""
    N = 1001
    grid = make_r_grid(1e-5, 150.0, N)
    V = V_core_on_grid(grid, CorePotentialParams(Zc=1.0, a1=0, a2=0, a3=0, a4=0, a5=0, a6=0))
    o1s = solve_bound_states(grid, V, l=0, n_states_max=2)[0]
    E, E_ej = 100.0, 12.0
    IP = -o1s.energy_au * HARTREE_EV
    Ef = E - IP - E_ej
    # incident wave in the static potential of the neutral target (z_ion = 0); scattered and
    # ejected waves in U = V_core with z_ion = 1 (the reference's ionization convention)
    from distorting_potential import DistortingPotential
    Ucore = DistortingPotential(U_of_r=V, V_hartree_of_r=np.zeros_like(V))
    ki = float(k_from_E_eV(E))
    Uinc, _ = build_distorting_potentials(grid, V, o1s, o1s, ki, ki)
    ej = solve_continuum_wave(grid, Ucore, 1, E_ej, 1.0)
    ls = [0, 1, 2, 4]
    wi = {l: solve_continuum_wave(grid, Uinc, l, E, 0.0) for l in ls}
    wf = {l: solve_continuum_wave(grid, Ucore, l, Ef, 1.0) for l in ls}
    calls = [dict(li=0, lf=0, L_max=6, kw={}), dict(li=1, lf=2, L_max=6, kw={}),
             dict(li=4, lf=2, L_max=6, kw={})]
    _save_case("h_ionization_100eV", grid, V, Uinc.U_of_r, V, o1s.u_of_r, ej.chi_of_r,
               True, _wave_meta(ej), wi, wf, calls)


def _synthetic_wave(r, k, l, delta, r0):
    return np.sin(k * r - 0.5 * l * np.pi + delta) * (1.0 - np.exp(-(r / r0) ** (l + 1)))


def case_synthetic_batch():
    """Synthetic kernel batch on a log grid to r = 400 (idx_match = -1, idx_limit = N)."""
    rng0 = np.random.default_rng(0)
    rng1 = np.random.default_rng(1)
    N = 1501
    grid = make_r_grid(1e-5, 400.0, N)
    r = grid.r
    bounds = []
    for _ in range(2):
        a = int(rng0.integers(1, 3))
        b = float(rng0.uniform(0.5, 2.0))
        c = rng0.uniform(-1, 1, size=3)
        u = r ** a * np.exp(-b * r) * (c[0] + c[1] * r + c[2] * r * r)
        u /= np.sqrt(np.sum(grid.w_trapz * u * u))
        bounds.append(u)
    wi, wf = {}, {}
    for idx in range(4):
        k1, k2 = rng1.uniform(0.5, 8.0, size=2)
        d1, d2 = rng1.uniform(0, np.pi, size=2)
        l1, l2 = (int(x) for x in rng1.integers(0, 64, size=2))
        wi[idx] = ContinuumWave(l=l1, k_au=float(k1), chi_of_r=_synthetic_wave(r, k1, l1, d1, (l1 + 1) / k1),
                                phase_shift=float(d1))
        wf[idx] = ContinuumWave(l=l2, k_au=float(k2), chi_of_r=_synthetic_wave(r, k2, l2, d2, (l2 + 1) / k2),
                                phase_shift=float(d2))
    zeros = np.zeros(N)
    calls = [dict(li=i, lf=i, L_max=8, kw={}) for i in range(4)]
    # The waves are keyed by pair index; l is carried in the metadata.
    _save_case("synthetic_r400", grid, zeros, zeros, zeros, bounds[0], bounds[1], False, None,
               wi, wf, calls)


def case_large_grid():
    """Synthetic waves on N = 5001 points to r = 400 at L = 0..8: the largest grid the reference's
    CPU path evaluates here in reasonable time and memory (its exchange gather holds n1 x N_cc
    temporaries), a high partial wave (l = 63), and a Coulomb-like pair (eta != 0, matching point
    inside the grid) whose outer tails are active."""
    rng = np.random.default_rng(7)
    N = 5001
    grid = make_r_grid(1e-5, 400.0, N)
    r = grid.r
    bounds = []
    for _ in range(2):
        a = int(rng.integers(1, 3))
        b = float(rng.uniform(0.5, 2.0))
        c = rng.uniform(-1, 1, size=3)
        u = r ** a * np.exp(-b * r) * (c[0] + c[1] * r + c[2] * r * r)
        u /= np.sqrt(np.sum(grid.w_trapz * u * u))
        bounds.append(u)
    im = int(np.searchsorted(r, 240.0))
    wi, wf = {}, {}
    for idx, (l1, k1, l2, k2, coul) in enumerate([(0, 0.7, 63, 1.3, False), (5, 2.0, 6, 1.5, False),
                                                  (2, 1.1, 3, 0.9, True)]):
        d1, d2 = rng.uniform(0, np.pi, size=2)
        if coul:
            s1, s2 = rng.uniform(-1, 1, size=2)
            e1, e2 = -1.0 / k1, -1.0 / k2
            c1 = np.sin(k1 * r - 0.5 * l1 * np.pi + e1 * np.log(2 * k1 * r) + s1 + d1) * \
                (1.0 - np.exp(-(r * k1 / (l1 + 1)) ** (l1 + 1)))
            c2 = np.sin(k2 * r - 0.5 * l2 * np.pi + e2 * np.log(2 * k2 * r) + s2 + d2) * \
                (1.0 - np.exp(-(r * k2 / (l2 + 1)) ** (l2 + 1)))
            wi[idx] = ContinuumWave(l=l1, k_au=k1, chi_of_r=c1, phase_shift=float(d1), idx_match=im, eta=e1,
                                    sigma_l=float(s1))
            wf[idx] = ContinuumWave(l=l2, k_au=k2, chi_of_r=c2, phase_shift=float(d2), idx_match=im, eta=e2,
                                    sigma_l=float(s2))
        else:
            wi[idx] = ContinuumWave(l=l1, k_au=k1, chi_of_r=_synthetic_wave(r, k1, l1, d1, (l1 + 1) / k1),
                                    phase_shift=float(d1))
            wf[idx] = ContinuumWave(l=l2, k_au=k2, chi_of_r=_synthetic_wave(r, k2, l2, d2, (l2 + 1) / k2),
                                    phase_shift=float(d2))
    V = -1.0 / r
    calls = [dict(li=i, lf=i, L_max=8, kw={}) for i in range(3)]
    _save_case("large_grid_n5001", grid, V, V, V, bounds[0], bounds[1], False, None, wi, wf, calls)


def case_low_k():
    """k_i + k_f <= k_threshold: standard Simpson path; non-orthogonal u_f makes the L=0 correction live."""
    N = 801
    grid = make_r_grid(1e-4, 100.0, N)
    r = grid.r
    V = -1.0 / r
    U_i = -np.exp(-r) * (1.0 + 1.0 / r)
    U_f = -np.exp(-1.3 * r) * (1.0 + 1.0 / r)
    u_i = 2.0 * r * np.exp(-r)
    u_f = r * r * np.exp(-0.7 * r)
    u_f /= np.sqrt(np.sum(grid.w_trapz * u_f * u_f))
    wi = {0: ContinuumWave(l=0, k_au=0.2, chi_of_r=np.sin(0.2 * r + 0.3), phase_shift=0.3, idx_match=600),
          2: ContinuumWave(l=2, k_au=0.2, chi_of_r=_synthetic_wave(r, 0.2, 2, 0.1, 15.0), phase_shift=0.1)}
    wf = {1: ContinuumWave(l=1, k_au=0.15, chi_of_r=_synthetic_wave(r, 0.15, 1, 0.7, 13.0), phase_shift=0.7,
                           idx_match=500)}
    calls = [dict(li=0, lf=1, L_max=4, kw={}), dict(li=2, lf=1, L_max=4, kw={}),
             dict(li=0, lf=1, L_max=3, kw={"oscillatory_method": "legacy"})]
    _save_case("low_k_standard", grid, V, U_i, U_f, u_i, u_f, False, None, wi, wf, calls)


def unit_fixtures():
    """Pins for the quadrature building blocks."""
    out = {}
    for n in (2, 3, 5, 7, 9):
        x, w = oi._get_cc_ref(n)
        out[f"cc_x_{n}"] = np.asarray(x)
        out[f"cc_w_{n}"] = np.asarray(w)
    grid = make_r_grid(1e-5, 200.0, 1001)
    r = grid.r
    cases = [(r[:1001], 2.3, np.pi / 2, 0.0), (r[:700], 9.0, np.pi / 2, 0.0), (r[:1001], 2.3, np.pi / 2, -0.8),
             (r[:900], 1.1, 1.0, -2.5), (r[:400], 0.9, np.pi / 2, 0.0)]
    for i, (rr, k, dphi, eta) in enumerate(cases):
        d = oi._adaptive_phase_increment_for_grid(rr, k, dphi, eta_total=eta, threshold=np.pi / 4,
                                                  min_increment=np.pi / 16)
        nodes = oi.generate_phase_nodes(rr[0], rr[-1], k, d, eta_total=eta)
        out[f"phase_params_{i}"] = np.array([len(rr), k, dphi, eta, d])
        out[f"phase_nodes_{i}"] = nodes
    xs = np.concatenate([np.geomspace(1e-5, 200.0, 333), [1e-5, 200.0, r[17], r[500]]])
    y = np.sin(r) * np.exp(-0.01 * r)
    out["interp_x"] = xs
    out["interp_y"] = oi._interp_on_radial_grid(xs, r, y)
    # Outer tails (scalar pins)
    tails = []
    for (rm, rmax, ki, kf, li, lf, di, df, ei, ef, si, sf, L, mom) in [
            (30.0, 200.0, 1.9, 1.7, 2, 3, 0.1, 0.4, 0.0, 0.0, 0.0, 0.0, 1, 0.7),
            (30.0, 200.0, 1.9, 1.7, 2, 3, 0.1, 0.4, 0.0, 0.0, 0.0, 0.0, 3, -2.1),
            (12.0, 120.0, 2.7, 2.4, 1, 1, 0.3, -0.2, -0.37, -0.41, 0.2, 0.5, 2, 1.3),
            (12.0, 120.0, 2.7, 0.4, 6, 5, 0.3, -0.2, -0.37, -2.5, 0.2, 0.5, 1, 0.9),
            (50.0, 400.0, 0.6, 0.55, 12, 11, 1.0, 2.0, 0.0, 0.0, 0.0, 0.0, 2, 5.0)]:
        env = (lambda m, LL: (lambda x: m / (x ** (LL + 1)) if x > 1e-6 else 0.0))(mom, L)
        t_out = oi.dwba_outer_integral_1d(env, ki, li, di, ei, si, kf, lf, df, ef, sf, rm, rmax,
                                          delta_phi=np.pi / 4)
        t_inf = oi._analytical_multipole_tail(rmax, ki, kf, di, df, li, lf, L, bound_overlap=mom,
                                              eta_i=ei, eta_f=ef, sigma_i=si, sigma_f=sf)
        t_rm = oi._analytical_multipole_tail(rm, ki, kf, di, df, li, lf, L, mom, ei, ef, si, sf)
        batch = oi.dwba_outer_integral_1d_multipole_batch(np.array([mom]), np.array([L]), ki, li, di, ei, si,
                                                          kf, lf, df, ef, sf, rm, rmax, delta_phi=np.pi / 4)
        tails.append([rm, rmax, ki, kf, li, lf, di, df, ei, ef, si, sf, L, mom, t_out, t_inf, t_rm,
                      batch.get(L, 0.0)])
    out["tails"] = np.array(tails)
    np.savez_compressed(os.path.join(HERE, "unit_quadrature.npz"), **out)
    print("  unit fixtures written")


if __name__ == "__main__":
    CASES = {"unit": unit_fixtures, "low_k": case_low_k, "synthetic_batch": case_synthetic_batch,
             "h_excitation": case_h_excitation, "heplus_ionic": case_heplus_ionic, "ionization": case_ionization,
             "large_grid": case_large_grid}
    # python tests/golden/make_golden.py [case ...]   (all cases without arguments)
    for name in (sys.argv[1:] or list(CASES)):
        CASES[name]()
