"""Benchmark: radial integrals/s of the DWBA radial matrix-element hot path on B200.

Workload (synthetic kernel batch): exponential grid N = 15000 on r in [1e-5, 400] a0;
4 seeded bound products u_i u_f with u = r^a e^{-br} P2(r), a in {1,2}, b in U[0.5,2];
2048 seeded continuum pairs (chi_i, chi_f), chi_l = sin(kr - l pi/2 + d)(1 - e^{-(r/r0)^{l+1}}),
k in U[0.5, 8], d in U[0, pi], l in 0..63, r0 = (l+1)/k; multipoles L = 0..8; direct and
exchange for every (continuum pair, bound pair): 147,456 integrals per step, each with the
reference's phase-split Clenshaw-Curtis quadrature (idx_match = -1, so n1 = N).

A step evaluates all of them. ``value`` times the device work (node-set operators, operand
folds, bilinear forms) with every input resident in HBM; ``e2e`` times the public batched API
(``radial_ME_all_L_batch``) from host NumPy arrays: planning, host->device copies, kernels and
the device->host read of the results. Inputs (~1 GB of operands per step) exceed the 126 MB L2.

--impl reference times the oracle port (a NumPy restatement of the reference's CPU algorithm:
dense N x N multipole matrices, Filon direct and the CC exchange gather) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOAD = ("synthetic kernel batch: N=15000 exp grid r in [1e-5,400], 2048 continuum pairs x 4 bound pairs "
            "per GPU, L=0..8, direct+exchange")
METRIC = "radial integrals/s (split-BF16 vs FP64, 1 B200) at <=1e-6 rel TCS error; ms per energy"
N_GRID, R_MAX, N_CONT, N_BOUND, L_MAX = 15000, 400.0, 2048, 4, 8


# ----------------------------------------------------------------------------- workload
class _Grid:
    def __init__(self, r, dr, w_trapz, w_simpson):
        self.r, self.dr, self.w_trapz, self.w_simpson = r, dr, w_trapz, w_simpson


class _Bound:
    def __init__(self, l, u):
        self.l, self.energy_au, self.u_of_r, self.n_index = l, -0.5, u, 1


class _Wave:
    def __init__(self, l, k, d, chi):
        self.l, self.k_au, self.phase_shift, self.chi_of_r = l, k, d, chi
        self.idx_match, self.eta, self.sigma_l = -1, 0.0, 0.0


def make_grid(N=N_GRID, r_min=1e-5, r_max=R_MAX):
    """Exponential grid with trapezoid and non-uniform Simpson weights (grid.py:419-611 formulas)."""
    idx = np.linspace(0.0, 1.0, N)
    r = r_min * ((r_max / r_min) ** idx)
    dr = np.diff(r)
    wt = np.zeros(N)
    wt[0], wt[-1] = 0.5 * dr[0], 0.5 * dr[-1]
    wt[1:-1] = 0.5 * (r[2:] - r[:-2])
    ws = np.zeros(N)
    h1, h2 = dr[0:N - 2:2], dr[1:N - 1:2]
    c = (h1 + h2) / 6.0
    ws[0:N - 2:2] += c * (2.0 - h2 / h1)
    ws[1:N - 1:2] += c * ((h1 + h2) ** 2 / (h1 * h2))
    ws[2:N:2] += c * (2.0 - h1 / h2)
    if N % 2 == 0:
        ws[-2] += 0.5 * dr[-1]
        ws[-1] += 0.5 * dr[-1]
    return _Grid(r, np.append(dr, dr[-1]), wt, ws)


def make_workload(N=N_GRID, n_cont=N_CONT, n_bound=N_BOUND, seed_shift=0, pinned=False):
    """Seeded workload; the continuum waves are rows of one (2*n_cont, N) host matrix (pinned on request)."""
    g = make_grid(N)
    r = g.r
    if pinned:
        import torch
        chi_block = torch.empty((2 * n_cont, N), dtype=torch.float64, pin_memory=True).numpy()
    else:
        chi_block = np.empty((2 * n_cont, N))
    rng0 = np.random.default_rng(0 + seed_shift)
    bounds = []
    for _ in range(n_bound):
        us = []
        for _ in range(2):
            a = int(rng0.integers(1, 3))
            b = float(rng0.uniform(0.5, 2.0))
            c = rng0.uniform(-1, 1, size=3)
            u = r ** a * np.exp(-b * r) * (c[0] + c[1] * r + c[2] * r * r)
            us.append(u / np.sqrt(np.sum(g.w_trapz * u * u)))
        bounds.append((_Bound(0, us[0]), _Bound(1, us[1])))
    rng1 = np.random.default_rng(1 + seed_shift)
    pairs = []
    for i in range(n_cont):
        w = []
        for j in range(2):
            k = float(rng1.uniform(0.5, 8.0))
            d = float(rng1.uniform(0.0, np.pi))
            l = int(rng1.integers(0, 64))
            r0 = (l + 1) / k
            row = chi_block[2 * i + j]
            row[:] = np.sin(k * r - 0.5 * l * np.pi + d) * (1.0 - np.exp(-(r / r0) ** (l + 1)))
            w.append(_Wave(l, k, d, row))
        pairs.append((w[0], w[1]))
    zeros = np.zeros(N)
    return g, zeros, bounds, pairs


def make_ragged_points(n_energy=64, l_max_wave=40, r_max=200.0, seed=3, select=None):
    """Ragged multi-energy sweep with the shapes of the He+ 1s->2s / 1s->2p study: energies
    geomspace(45, 1000, n_energy) eV, one grid per energy with N_e = round(2000 * 7.5^(e/(n-1))) points,
    l_i, l_f <= l_max_wave (parity-filtered per transition), Coulomb-like waves (z = 1: eta = -1/k,
    matching index inside the grid, so n1 < N and the outer tails take part), hydrogenic Z = 2 bound
    states. Synthetic (seeded) stand-ins for the reference's solver outputs. One point per
    (energy, transition). ``select``: indices of the energies to build (the others only advance the
    random stream, so a selected point equals the same point of the full sweep)."""
    rng = np.random.default_rng(seed)
    Z, hartree = 2.0, 27.211386245988
    dE = {"2s": 0.75 * Z * Z / 2 * hartree, "2p": 0.75 * Z * Z / 2 * hartree}
    points = []
    energies = np.geomspace(45.0, 1000.0, n_energy)
    for e, E in enumerate(energies):
        if select is not None and e not in select:
            rng.uniform(size=2 * 2 * 2 * (l_max_wave + 1))  # the draws of this energy's waves
            continue
        N = int(round(2000 * 7.5 ** (e / max(1, n_energy - 1))))
        g = make_grid(N, 1e-5, r_max)
        r = g.r
        u1s = 2.0 * Z ** 1.5 * r * np.exp(-Z * r)
        bound = {"2s": (Z / 2) ** 1.5 / np.sqrt(2.0) * r * (2.0 - Z * r) * np.exp(-Z * r / 2),
                 "2p": (Z / 2) ** 2.5 / np.sqrt(6.0) * r * r * np.exp(-Z * r / 2)}
        k_i = np.sqrt(2.0 * E / hartree)
        im = int(np.searchsorted(r, 0.6 * r_max))
        for name, lf_par in (("2s", 0), ("2p", 1)):
            k_f = np.sqrt(2.0 * (E - dE[name]) / hartree)

            def wave(l, k):
                eta = -1.0 / k
                d, sig = float(rng.uniform(0, np.pi)), float(rng.uniform(-1, 1))
                r0 = (l + 1) / k
                chi = np.sin(k * r - 0.5 * l * np.pi + eta * np.log(2 * k * r) + sig + d) * \
                    (1.0 - np.exp(-(r / r0) ** (l + 1)))
                w = _Wave(l, k, d, chi)
                w.eta, w.sigma_l, w.idx_match = eta, sig, im
                return w
            wi = [wave(l, k_i) for l in range(l_max_wave + 1)]
            wf = [wave(l, k_f) for l in range(l_max_wave + 1)]
            pairs = [(wi[a], wf[b]) for a in range(l_max_wave + 1) for b in range(l_max_wave + 1)
                     if (a + b) % 2 == lf_par]
            V = -Z / r
            points.append(dict(grid=g, V_core_array=V, U_i_array=V, bound_i=_Bound(0, u1s),
                               bound_f=_Bound(1 if name == "2p" else 0, bound[name]), pairs=pairs, U_f_array=V))
    return points


def ragged_sweep(engine, L_max=6, replays=5, n_energy=64, points=None, split=True):
    """Device time of the ragged sweep (node sets, folds, forms and tails of all points in shared
    launches, replayed from a CUDA graph). Returns (summary, [(I_dir, I_exc) per point])."""
    import torch
    from dwba_b200.dwba_matrix_elements import GPUCache, _make_job
    from dwba_b200.engine import MultiPrepared, PreparedJob
    if points is None:
        points = make_ragged_points(n_energy)
    kw = dict(use_oscillatory_quadrature=True, oscillatory_method="advanced", CC_nodes=5, phase_increment=1.5708,
              min_grid_fraction=0.10, k_threshold=0.5)
    parts = []
    for pt in points:
        cache = GPUCache(pt["grid"])
        job = _make_job(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"], pt["bound_f"], pt["pairs"],
                        L_max, pt["U_f_array"], kw, cache)
        parts.append(PreparedJob(job, cache.dg, engine, rebuild_nodesets=True))
    mp = MultiPrepared(parts)
    tile = None
    if mp.tc is not None:
        # the ragged tensor-core launch's tile, chosen by the tuner (median of repeated launches)
        from dwba_b200 import tune
        key = tune.TILE_TUNER.key(mp.tc["nt"], mp.max_grid, int(mp.tc["n"]), L_max)
        tile = {"choice": tune._tile_name(tune.TILE_TUNER.select(key, mp)),
                "timings_ms": tune.TILE_TUNER.timings_ms[key]}
    mp.capture()
    mp.replay()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(replays):
        mp.replay()
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / replays
    # per-stage device time of one more (un-captured) launch sequence, with each stage's bytes
    stages, gbs = None, None
    if split:
        marks = []
        mp.launch(marks)
        torch.cuda.synchronize()
        stages = {f"{b[0]}_ms": a[1].elapsed_time(b[1]) for a, b in zip(marks[:-1], marks[1:])}
        stage_bytes = {"nodesets_ms": sum(p.nodesets.algorithmic_bytes() for p in parts if p.nodesets.n),
                       "folds_ms": sum(p.fold_bytes() for p in parts)}
        if engine == "semisep":
            stage_bytes["forms_ms"] = sum(p.algorithmic_bytes() for p in parts)
        gbs = {k.replace("_ms", "_gbs"): stage_bytes[k] / (stages[k] * 1e-3) / 1e9 for k in stage_bytes
               if stages.get(k)}
    outs = mp.collect()
    finite = all(np.isfinite(d).all() and np.isfinite(e).all() for d, e in outs)
    n_int = sum(2 * p.T * p.P * p.nl for p in parts)
    routed = None
    if mp.tc is not None:  # exchange forms the accuracy guard recomputed in FP64 (dominant forms)
        routed = {"forms": int(mp.tc["guard"].n_routed()), "of": int(mp.tc["n"])}
    n_energy = len(points) // 2
    Ns = [len(pt["grid"].r) for pt in points]
    n_tail = int(sum(p.n_tail for p in parts))
    mp.graph = None
    del mp, parts
    torch.cuda.empty_cache()
    return {"workload": f"ragged sweep: {n_energy} energies geomspace(45, 1000) eV, N_e = 2000..15000 "
                        f"(own grid per energy), He+-like 1s->2s and 1s->2p, l <= 40 parity-filtered, L=0..{L_max}, "
                        "Coulomb-like waves (eta = -1/k, n1 < N, outer tails on the device), synthetic",
            "engine": engine, "energies": n_energy, "points": len(points), "N_min": min(Ns), "N_max": max(Ns),
            "integrals": n_int, "ms_per_sweep": ms, "ms_per_energy": ms / n_energy,
            "integrals_per_s": n_int / (ms * 1e-3), "graph": True, "replays": replays,
            "split_ms": stages, "split_algorithmic_gbs": gbs, "tail_records": n_tail,
            "tc_guard_routed": routed, "tc_tile": tile, "results_finite": bool(finite)}, outs


def sweep_tcs_errors(points, ref, test, L_max=6):
    """Max and median relative TCS difference over the sweep's points between two engines' integrals
    (the DCS is a quadratic form in the integrals; its prefactor and the 2/(pi k_i k_f) scale cancel
    in the ratio, so one coupling table per transition serves every energy)."""
    from dwba_b200.coupling import CouplingTables
    theta = np.linspace(0.0, np.pi, 181)
    tables = {}
    rel = []
    for pt, (rd, re_), (td, te) in zip(points, ref, test):
        Lf = pt["bound_f"].l
        chans = [(w_i.l, w_f.l) for w_i, w_f in pt["pairs"]]
        key = (Lf, len(chans))
        if key not in tables:
            tables[key] = CouplingTables(theta, chans, L_max, 1.0, 1.0, 0, Lf)
        tab = tables[key]
        t_ref = tab.tcs(rd[0], re_[0])
        rel.append(abs(tab.tcs(td[0], te[0]) - t_ref) / abs(t_ref))
    rel = np.array(rel)
    return float(rel.max()), float(np.median(rel))


# ----------------------------------------------------------------------------- ionization workload
IONIZATION_WORKLOAD = ("ionization SDCS: H 1s, E = 200 eV, 40 ejected energies linspace(0.5, 99) eV, N=8000 exp grid "
                       "r in [1e-5,200], l_i, l_f, l_ej <= 30 parity-filtered, L=0..10, Coulomb-like synthetic waves")


class _Continuum(_Wave):
    """A continuum final state (ejected electron): carries chi_of_r, and u_of_r as the reference's does."""

    @property
    def u_of_r(self):
        return self.chi_of_r


def make_ionization_points(n_ej=40, l_max=30, N=8000, r_max=200.0, seed=5, select=None):
    """H 1s ionization at 200 eV with the shapes of the reference's SDCS loop (ionization.py:526-608):
    per ejected energy, one transition per ejected partial wave l_ej, all (l_i, l_f) pairs with
    l_i + l_f = l_ej (mod 2); the two parity classes are two points on the one grid. Coulomb-like
    synthetic waves (z = 1, matching index inside the grid) stand in for the solver's. ``select``:
    indices of the ejected energies to build (the others only advance the random stream)."""
    rng = np.random.default_rng(seed)
    hartree, E, IP = 27.211386245988, 200.0, 13.605693
    g = make_grid(N, 1e-5, r_max)
    r = g.r
    bound = _Bound(0, 2.0 * r * np.exp(-r))
    V = -1.0 / r
    im = int(np.searchsorted(r, 0.6 * r_max))

    def wave(l, k, cls=_Wave):
        eta = -1.0 / k
        d, sig = float(rng.uniform(0, np.pi)), float(rng.uniform(-1, 1))
        chi = np.sin(k * r - 0.5 * l * np.pi + eta * np.log(2 * k * r) + sig + d) * \
            (1.0 - np.exp(-(r / ((l + 1) / k)) ** (l + 1)))
        w = cls(l, k, d, chi)
        w.eta, w.sigma_l, w.idx_match = eta, sig, im
        return w
    k_i = np.sqrt(2.0 * E / hartree)
    incident = [wave(l, k_i) for l in range(l_max + 1)]
    points = []
    for e, E_ej in enumerate(np.linspace(0.5, 99.0, n_ej)):
        if select is not None and e not in select:
            rng.uniform(size=2 * 2 * (l_max + 1))  # the draws of this energy's scattered and ejected waves
            continue
        k_ej = np.sqrt(2.0 * E_ej / hartree)
        k_s = np.sqrt(2.0 * (E - IP - E_ej) / hartree)
        scat = [wave(l, k_s) for l in range(l_max + 1)]
        ej = [wave(l, k_ej, _Continuum) for l in range(l_max + 1)]
        for par in (0, 1):
            pairs = [(incident[a], scat[b]) for a in range(l_max + 1) for b in range(l_max + 1) if (a + b) % 2 == par]
            lej = [l for l in range(l_max + 1) if l % 2 == par]
            points.append(dict(grid=g, V_core_array=V, U_i_array=V, bound_i=[bound] * len(lej),
                               bound_f=[ej[l] for l in lej], pairs=pairs, U_f_array=V, E_ej=float(E_ej),
                               k=(k_i, k_s, k_ej), l_ej=lej))
    return points


def ionization_sweep(engine, points, L_max=10, chunk=16, replays=2):
    """Device time of all points, in chunks of `chunk` points (one MultiPrepared and one CUDA graph
    each, since every point holds its folded operands). Returns (ms, [(I_dir, I_exc) per point])."""
    import torch
    from dwba_b200.dwba_matrix_elements import GPUCache, _make_job
    from dwba_b200.engine import MultiPrepared, PreparedJob
    kw = dict(use_oscillatory_quadrature=True, oscillatory_method="advanced", CC_nodes=5, phase_increment=1.5708,
              min_grid_fraction=0.10, k_threshold=0.5)
    cache = GPUCache(points[0]["grid"])
    total, outs = 0.0, []
    st = torch.cuda.current_stream()
    for c0 in range(0, len(points), chunk):
        parts = []
        for pt in points[c0:c0 + chunk]:
            job = _make_job(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"], pt["bound_f"],
                            pt["pairs"], L_max, pt["U_f_array"], kw, cache)
            parts.append(PreparedJob(job, cache.dg, engine, rebuild_nodesets=True))
        mp = MultiPrepared(parts)
        mp.capture()
        mp.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(replays):
            mp.replay()
        e1.record(st)
        e1.synchronize()
        total += e0.elapsed_time(e1) / replays
        outs.extend(mp.collect())
        mp.graph = None
        del mp, parts
        torch.cuda.empty_cache()
    return total, outs


class IonizationSDCS:
    """Angle-integrated SDCS per ejected energy from the integrals, with the reference's algebra
    (ionization.py:610-642, dwba_coupling.py:507-620): per (l_ej, l_f, M_f) the direct and exchange
    amplitudes summed coherently over l_i, then 0.25|f+g|^2 + 0.75|f-g|^2, times
    (2 pi)^4 (k_s k_ej / k_i) and the amplitude prefactor (2/pi)/(k_i k_s) sqrt(2/pi)/k_ej squared.
    The channel coefficients depend only on angular momenta and are built once per parity class."""

    def __init__(self, points, L_max=10):
        from dwba_b200.coupling import channel_coefficients
        self.L_max = L_max
        self.tabs = {}
        for pt in points[:2]:
            par = pt["l_ej"][0] % 2
            li = np.array([a.l for a, _ in pt["pairs"]])
            lf = np.array([b.l for _, b in pt["pairs"]])
            per_t = []
            for l_ej in pt["l_ej"]:
                per_m = []
                for Mf in range(-l_ej, l_ej + 1):
                    cf = np.zeros((len(li), L_max + 1), dtype=complex)
                    cg = np.zeros_like(cf)
                    for p in range(len(li)):
                        cf[p], cg[p] = channel_coefficients(int(li[p]), int(lf[p]), L_max, 0, l_ej, 0, Mf)
                    per_m.append((cf, cg))
                per_t.append(per_m)
            self.tabs[par] = (lf, per_t)

    def sdcs(self, pt, I_dir, I_exc):
        lf, per_t = self.tabs[pt["l_ej"][0] % 2]
        k_i, k_s, k_ej = pt["k"]
        amp = (2.0 / np.pi) / (k_i * k_s) * np.sqrt(2.0 / np.pi) / k_ej
        tot = 0.0
        for t, per_m in enumerate(per_t):
            for cf, cg in per_m:
                f = np.einsum("pl,pl->p", cf, I_dir[t]) * amp
                g = np.einsum("pl,pl->p", cg, I_exc[t]) * amp
                F = np.bincount(lf, f.real, minlength=lf.max() + 1) + 1j * np.bincount(lf, f.imag, minlength=lf.max() + 1)
                G = np.bincount(lf, g.real, minlength=lf.max() + 1) + 1j * np.bincount(lf, g.imag, minlength=lf.max() + 1)
                tot += float(np.sum(0.25 * np.abs(F + G) ** 2 + 0.75 * np.abs(F - G) ** 2))
        return (2.0 * np.pi) ** 4 * (k_s * k_ej / k_i) * tot


def ionization_run(compare=True):
    """The ionization workload through the exact FP64 engine and the split-BF16 engine (and the plain
    FP64 kernel on one ejected energy); SDCS per ejected energy and the trapezoid TICS over them."""
    import torch
    points = make_ionization_points()
    n_int = sum(2 * len(pt["l_ej"]) * len(pt["pairs"]) * 11 for pt in points)
    ms_ss, ref = ionization_sweep("semisep", points)
    res = {"workload": IONIZATION_WORKLOAD, "integrals": n_int, "points": len(points),
           "semisep_ms": ms_ss, "semisep_integrals_per_s": n_int / (ms_ss * 1e-3),
           "semisep_ms_per_ejected_energy": ms_ss / (len(points) // 2)}
    if compare:
        ms_tc, tc = ionization_sweep("tc_bf16x3", points)
        ms_dense, _ = ionization_sweep("dense", points[:2], replays=1)
        n_e = len(points) // 2
        sd = IonizationSDCS(points)
        E = np.array([pt["E_ej"] for pt in points[0::2]])
        s_ref = np.array([sd.sdcs(points[2 * e], *ref[2 * e]) + sd.sdcs(points[2 * e + 1], *ref[2 * e + 1])
                          for e in range(n_e)])
        s_tc = np.array([sd.sdcs(points[2 * e], *tc[2 * e]) + sd.sdcs(points[2 * e + 1], *tc[2 * e + 1])
                         for e in range(n_e)])
        rel = np.abs(s_tc - s_ref) / np.abs(s_ref)
        tics_ref, tics_tc = np.trapezoid(s_ref, E), np.trapezoid(s_tc, E)
        # integral-level errors of the split form against the exact FP64 integrals, relative to the
        # largest integral of the same kind (direct / exchange) and transition
        dI = np.concatenate([np.abs(np.stack(a) - np.stack(b)).ravel() for a, b in zip(tc, ref)])
        sc = np.concatenate([np.broadcast_to(np.max(np.abs(np.stack(b)), axis=(2, 3), keepdims=True),
                                             np.stack(b).shape).ravel() for b in ref])
        res.update({"tc_bf16x3_ms": ms_tc, "tc_bf16x3_integrals_per_s": n_int / (ms_tc * 1e-3),
                    "dense_fp64_ms_one_ejected_energy": ms_dense, "dense_fp64_ms_scaled": ms_dense * n_e,
                    "split_bf16_vs_plain_fp64_speedup": ms_dense * n_e / ms_tc,
                    "semisep_vs_plain_fp64_speedup": ms_dense * n_e / ms_ss,
                    "tc_bf16x3_sdcs_rel_err_max": float(rel.max()), "tc_bf16x3_sdcs_rel_err_median": float(np.median(rel)),
                    "tc_bf16x3_tics_rel_err": float(abs(tics_tc - tics_ref) / abs(tics_ref)),
                    "tc_bf16x3_max_abs_err_over_transition_max": float(np.max(dI / np.maximum(sc, 1e-300))),
                    "note": "SDCS per ejected energy from each engine's integrals (reference algebra, angle-integrated), "
                            "TICS by the trapezoid rule over the 40 ejected energies; the plain FP64 kernel is timed "
                            "on the first ejected energy and scaled by 40"})
    return res


# ----------------------------------------------------------------------------- gradients
def make_gradient_inputs(seed=9):
    """Inputs at the differentiation config's sizes: N = 6000 on [1e-5, 200], an s->p transition with
    l_i, l_f <= 25, l_i + l_f odd (338 pairs), a parametric SAE-like V_core and U_i = V_core + 0.3 e^-r
    (live L=0 correction), synthetic waves. Returns (grid, V, U, bound_i, bound_f, pairs, rng)."""
    rng = np.random.default_rng(seed)
    g = make_grid(6000, 1e-5, 200.0)
    r = g.r
    V = -(1.0 + 10.0 * np.exp(-3.0 * r) + 2.0 * r * np.exp(-1.5 * r) + np.exp(-0.8 * r)) / r
    U = V + 0.3 * np.exp(-r)
    u_s = r * np.exp(-r) * (1.0 - 0.4 * r + 0.03 * r * r)
    u_p = r * r * np.exp(-0.7 * r) * (1.0 - 0.1 * r)
    bi, bf = _Bound(0, u_s / np.sqrt(np.sum(g.w_trapz * u_s ** 2))), _Bound(1, u_p / np.sqrt(np.sum(g.w_trapz * u_p ** 2)))
    k_i, k_f = 1.21, 1.02

    def wave(l, k):
        d = float(rng.uniform(0, np.pi))
        return _Wave(l, k, d, np.sin(k * r - 0.5 * l * np.pi + d) * (1.0 - np.exp(-(r / ((l + 1) / k)) ** (l + 1))))
    wi = [wave(l, k_i) for l in range(26)]
    wf = [wave(l, k_f) for l in range(26)]
    pairs = [(wi[a], wf[b]) for a in range(26) for b in range(26) if (a + b) % 2 == 1]
    return g, V, U, bi, bf, pairs, rng


def gradient_run(reps=3):
    """The differentiation config end to end: Na-like 3s -> 3p in the parametric SAE core potential
    V = -[1 + 10 e^{-a1 r} + a2 r e^{-a3 r} + a4 e^{-a5 r}]/r (a seeded within +-10 % of
    (3.0, 2.0, 1.5, 1.0, 0.8)), N = 6000 on [1e-5, 200], E = 20 eV, l_i, l_f <= 25 (338 pairs), L = 0..4.
    The inputs come from dwba_b200/sae.py's solvers; dTCS/d(a1..a5) is the CUDA backward (FP64, and the
    split-BF16 tensor-core backward with FP32 accumulation) contracted with the solvers' central-
    difference tangents, against central differences of the TCS (h = 1e-6 relative). Times: the
    integrals' forward and forward+backward from CUDA tensors (host planning included), and one whole
    parameter gradient (11 solver runs, forward, backward, contraction)."""
    import torch
    from dwba_b200 import sae
    from dwba_b200.autograd import RadialIntegrals
    from dwba_b200.coupling import CouplingTables
    from dwba_b200.fit import CouplingCrossSection
    g = make_grid(6000, 1e-5, 200.0)
    p = np.random.default_rng(2).uniform(0.9, 1.1, 5) * np.array([3.0, 2.0, 1.5, 1.0, 0.8])
    prob = sae.SAEProblem(g, sae.Transition(E_eV=20.0, l_max=25, L_max=4), p,
                          full_params=lambda q: np.concatenate([[10.0], q]))
    x0 = prob.inputs(p)
    bi, bf, pairs = prob.wave_objects(x0)
    model = RadialIntegrals(g, bi, bf, pairs, 4, U_f_array=x0.U_f, engine="semisep")
    model_tc = RadialIntegrals(g, bi, bf, pairs, 4, U_f_array=x0.U_f, engine="semisep", backward="tc_bf16x3",
                               gpu_cache=model.cache)
    xs = CouplingCrossSection(CouplingTables(np.linspace(0.0, np.pi, 181), prob.pairs_l, 4, prob.k_i, prob.k_f, 0, 1))
    x = prob.torch_inputs(x0)

    def fwd():
        with torch.no_grad():
            return float(xs.tcs(model(**x)))

    def fwd_bwd(m=model):
        xg = {k: v.clone().requires_grad_(True) for k, v in x.items()}
        loss = xs.tcs(m(**xg))
        loss.backward()
        return {k: v.grad for k, v in xg.items()}
    g64 = fwd_bwd()
    gtc = fwd_bwd(model_tc)
    rel_in = {k: float(torch.linalg.norm(gtc[k] - g64[k]) / torch.linalg.norm(g64[k])) for k in g64}
    tcs, grad, fd = sae.value_and_grad(prob, model, xs.tcs, p, with_fd=True)
    _, grad_tc = sae.value_and_grad(prob, model_tc, xs.tcs, p)
    fwd()
    torch.cuda.synchronize()
    out = {}
    for name, fn in (("forward_ms", fwd), ("forward_backward_ms", fwd_bwd),
                     ("forward_backward_tc_bf16x3_ms", lambda: fwd_bwd(model_tc)),
                     ("parameter_gradient_ms", lambda: sae.value_and_grad(prob, model, xs.tcs, p))):
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        out[name] = (time.perf_counter() - t0) * 1e3 / reps
    return {"workload": "differentiation config: Na-like 3s->3p, parametric SAE potential, N=6000 exp grid r in "
                        "[1e-5,200], E=20 eV, 338 (l_i, l_f <= 25) pairs, L=0..4, inputs from the parameters by "
                        "dwba_b200/sae.py's solvers",
            "integrals": len(pairs) * 2 * 5, "parameters": [float(v) for v in p], "tcs_au": tcs,
            "dtcs_dparams": [float(v) for v in grad], "dtcs_dparams_central_fd": [float(v) for v in fd],
            "dtcs_dparams_rel_err_vs_fd_max": float(np.max(np.abs(grad - fd) / np.abs(fd))),
            "dtcs_dparams_tc_bf16x3_rel_err_max": float(np.max(np.abs(grad_tc - grad) / np.abs(grad))),
            **out, "tc_bf16x3_vs_fp64_input_gradient_rel_err": rel_in,
            "note": "forward/backward wall time per call through RadialIntegrals + the torch TCS (host planning, "
                    "FP64 forward, exact FP64 backward kernels, or the split-BF16 tensor-core backward with FP32 "
                    "accumulation); dTCS/da by the backward chained with central-difference solver tangents, "
                    "against central differences of the TCS (h = 1e-6 relative); input gradient rel err = "
                    "|g_tc - g_fp64| / |g_fp64| per input function"}


# ----------------------------------------------------------------------------- drop-in calls
def dropin_run():
    """H 1s->2p at 50 eV (N = 3000, 128 (l_i, l_f) pairs, L = 0..4; the reference's own solver outputs
    stored in tests/golden/config1.npz): the reference driver's loop of one radial_ME_all_L_gpu call per
    pair, timed per call, and the same pairs in one radial_ME_all_L_batch call."""
    import torch
    from dataclasses import dataclass
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch, radial_ME_all_L_gpu, GPUCache

    @dataclass(frozen=True)
    class Wave:
        l: int
        k_au: float
        chi_of_r: np.ndarray
        phase_shift: float
        idx_match: int = -1
        eta: float = 0.0
        sigma_l: float = 0.0
    z = np.load(os.path.join(ROOT, "tests", "golden", "config1.npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    g = _Grid(z["r"], z["dr"], z["w_trapz"], z["w_simpson"])
    bi, bf = _Bound(0, z["u_i"]), _Bound(1, z["u_f"])

    def wave(m, chi):
        l, k, d, im, eta, sig = m
        return Wave(int(l), float(k), chi, float(d), int(im), float(eta), float(sig))
    wi = {int(l): wave(v, z["chi_i"][int(l)]) for l, v in meta["waves_i"].items()}
    wf = {int(l): wave(v, z["chi_f"][int(l)]) for l, v in meta["waves_f"].items()}
    pairs = [(wi[a], wf[b]) for a, b in meta["pairs"]]
    L = meta["L_max"]
    cache = GPUCache.from_grid(g)
    # the potentials as arrays in memory, as the driver holds them (indexing the npz archive
    # decompresses the array again at every access)
    V_core, U_i, U_f = z["V_core"], z["U_i"], z["U_f"]

    def loop(engine):
        return [radial_ME_all_L_gpu(g, V_core, U_i, bi, bf, ci, cf, L, U_f_array=U_f, gpu_cache=cache,
                                    engine=engine) for ci, cf in pairs]

    def batch(engine):
        return radial_ME_all_L_batch(g, V_core, U_i, bi, bf, pairs, L, U_f_array=U_f, gpu_cache=cache,
                                     engine=engine)
    out = {}
    for engine in ("dense", "semisep"):
        loop(engine), batch(engine)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loop(engine)
        t1 = time.perf_counter()
        for _ in range(3):
            batch(engine)
        t2 = time.perf_counter()
        out[engine] = {"per_pair_call_ms": (t1 - t0) * 1e3 / len(pairs), "all_pairs_loop_ms": (t1 - t0) * 1e3,
                       "batch_call_ms": (t2 - t1) * 1e3 / 3}
    return {"workload": "H 1s->2p 50 eV, N=3000, 128 pairs, L=0..4 (the reference's solver outputs)",
            **out, "integrals": len(pairs) * 2 * (L + 1),
            "note": "wall time from host NumPy inputs to result dicts (the node sets of the grid cached "
                    "across calls, as GPUCache does for the reference's driver)"}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.rows, self.proc, self.gpu = [], None, gpu_index

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # wait (up to 3 s) for the first sample, so that a short timed region is sampled too
            t0 = time.time()
            while not self.rows and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ----------------------------------------------------------------------------- reference / CPU baseline
def cpu_sample(seconds_hint=20.0, N=N_GRID, block=64):
    """Bounded sample of the reference algorithm (oracle port) on this workload.

    The reference's CPU path (dwba_matrix_elements.py:1057-1116 with oscillatory_integrals.py:2555-2777)
    spends its time in per-row work: build K_L rows (1/r_> exp(L log ratio)), contract them with
    rho2 w over N columns (direct) and gather/interpolate them at the N_cc CC nodes (exchange).
    The sample runs exactly that work, the reference's way, for a block of rows of one
    continuum/bound pair at L = 0..8, and scales by the fraction of rows: integrals/s =
    18 * (rows done / n1) / seconds."""
    import oracle  # noqa: F401  (the oracle is the checker and the CPU baseline, never the product)
    from oracle.quadrature import adaptive_phase_increment, cc_nodes_on_breakpoints, generate_phase_nodes, \
        interp_on_radial_grid
    g, zeros, bounds, pairs = make_workload(N, n_cont=1, n_bound=1)
    (bi, bf), (ci, cf) = bounds[0], pairs[0]
    r, w = g.r, g.w_simpson
    n1 = N
    k_total = ci.k_au + cf.k_au
    d = adaptive_phase_increment(r[:n1], k_total, 1.5708)
    X, W, _ = cc_nodes_on_breakpoints(generate_phase_nodes(r[0], r[n1 - 1], k_total, d), 5)
    rho2_dir = bf.u_of_r * bi.u_of_r * w
    rho2_cc = interp_on_radial_grid(X, r, cf.chi_of_r * bi.u_of_r) * W
    iR = np.clip(np.searchsorted(r, X), 1, N - 1)
    iL = iR - 1
    wR = (X - r[iL]) / (r[iR] - r[iL] + 1e-30)
    wL = 1.0 - wR
    rows = 0
    t0 = time.perf_counter()
    i0 = 0
    while time.perf_counter() - t0 < seconds_hint and i0 < n1:
        ri = r[i0:i0 + block, None]
        rl = np.minimum(ri, r[None, :])
        rg = np.maximum(ri, r[None, :])
        ratio = rl / rg
        inv = 1.0 / rg
        lr = np.log(np.minimum(ratio, 1.0 - 1e-12) + 1e-300)
        for L in range(L_MAX + 1):
            K = inv if L == 0 else inv * np.exp(L * lr)
            _ = K @ rho2_dir
            Kcc = K[:, iL] * wL + K[:, iR] * wR
            _ = Kcc @ rho2_cc
        rows += ri.shape[0]
        i0 += block
    dt = time.perf_counter() - t0
    ips = 2 * (L_MAX + 1) * (rows / n1) / dt
    return ips, dt, rows


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = os.cpu_count()
    vals = []
    # about a minute of CPU work in total, whatever the step count (short steps use 16-row blocks)
    for _ in range(args.warmup):
        cpu_sample(seconds_hint=0.5, block=16)
    for _ in range(args.steps):
        hint = max(0.2, min(20.0, 60.0 / max(1, args.steps)))
        ips, dt, rows = cpu_sample(seconds_hint=hint, block=16 if hint < 2.0 else 64)
        vals.append(ips)
    v = float(np.median(vals))
    line = {"metric": METRIC, "value": v, "unit": "integrals/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * 147456 / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "engine": "reference CPU algorithm (oracle port)",
                       "integrals_per_step_per_gpu": 147456, "parallelism": "host"},
            "cpu_baseline": {"value": v, "unit": "integrals/s", "cores": cores, "kind": "port",
                             "sample": "oracle port of the reference CPU algorithm: row blocks of one pair at "
                                       "N=15000, L=0..8, direct+exchange, scaled by rows/n1"},
            "e2e": {"value": v, "unit": "integrals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------------------- our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=150)  # ~0.9 s timed: several 200 ms clock samples
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default=os.environ.get("DWBA_BENCH_ENGINE", "semisep"),
                    choices=["dense", "semisep", "tc_bf16x3", "tc_bf16x6"])
    ap.add_argument("--n-cont", type=int, default=N_CONT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ragged", action="store_true", help="skip the ragged multi-energy sweep")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip timing the split-BF16 and plain FP64 engines on the same batch")
    ap.add_argument("--workload", default="batch", choices=["batch", "ionization"],
                    help="ionization: the H 1s ionization SDCS workload instead of the kernel batch (one GPU)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ionization":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(ionization_run(compare=not args.no_compare)))
        return 0
    import torch
    import torch.distributed as dist
    from dwba_b200.dwba_matrix_elements import GPUCache, _make_job, radial_ME_all_L_batch
    from dwba_b200.engine import PreparedJob

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)

    # each rank owns its shard of independent continuum pairs (weak scaling: fixed work per GPU)
    g, zeros, bounds, pairs = make_workload(n_cont=args.n_cont, seed_shift=1000 * rank, pinned=True)
    n_int = len(pairs) * len(bounds) * (L_MAX + 1) * 2
    cache = GPUCache.from_grid(g)
    kw = dict(use_oscillatory_quadrature=True, oscillatory_method="advanced", CC_nodes=5, phase_increment=1.5708,
              min_grid_fraction=0.10, k_threshold=0.5)
    b_i = [b[0] for b in bounds]
    b_f = [b[1] for b in bounds]
    # one job: the 4 bound transitions share the continuum waves and the 2048 node sets
    job = _make_job(g, zeros, zeros, b_i, b_f, pairs, L_MAX, zeros, kw, cache)
    preps = [PreparedJob(job, cache.dg, args.engine, rebuild_nodesets=True)]
    st = torch.cuda.current_stream()

    def step():
        for p in preps:
            p.launch()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    # kernel-level split of one step (events on the launching stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record(st)
    for p in preps:
        p.nodesets.launch()
    ev[1].record(st)
    for p in preps:
        p.launch_folds()
    ev[2].record(st)
    tc = args.engine.startswith("tc_")
    if tc:
        ev_tc = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        for p in preps:
            p.launch_forms_direct()
        ev_tc[0].record(st)
        for p in preps:
            p.launch_forms_exchange()
        ev_tc[1].record(st)
    else:
        form_marks = []
        for p in preps:
            if args.engine == "semisep":
                p.form_launch.launch(p.lib, p.job.L_max, p.ds, float(p.job.grid.r[0]), float(p.job.grid.r[-1]),
                                     marks=form_marks)
            else:
                p.launch_forms()
    ev[3].record(st)
    barrier()
    split = {"nodesets_ms": ev[0].elapsed_time(ev[1]), "folds_ms": ev[1].elapsed_time(ev[2]),
             "forms_ms": ev[2].elapsed_time(ev[3])}
    sub_ms = {}
    if not tc and args.engine == "semisep":
        # the forms stage per launch: potentials, dot forms, semiseparable forms (events between them)
        prev = ev[2]
        for name, e in form_marks:
            sub_ms[name] = sub_ms.get(name, 0.0) + prev.elapsed_time(e)
            prev = e
        split.update({f"{k}_ms": v for k, v in sub_ms.items()})
    if tc:
        split["forms_exchange_tensor_ms"] = ev_tc[0].elapsed_time(ev_tc[1])
    # timed region
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        t_start.record(st)
        for _ in range(args.steps):
            step()
        t_end.record(st)
        barrier()
    ms = t_start.elapsed_time(t_end) / args.steps
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * n_int / (ms * 1e-3)
    # results of the last step, checked for finiteness
    outs = [p.collect() for p in preps]
    finite = all(np.isfinite(d).all() and np.isfinite(e).all() for d, e in outs)
    nonzero = all(np.abs(d).max() > 0 and np.abs(e).max() > 0 for d, e in outs)

    # per-kernel rooflines; the one reported as "roofline" is the kernel that takes longest
    forms_ms = split["forms_ms"]
    flops = sum(p.algorithmic_flops() for p in preps)
    fb = sum(p.algorithmic_bytes() for p in preps)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    # DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from one ncu capture of
    # the default workload (profiles/launches_semisep_synthetic_batch_N15000.md); other sizes: null
    default_size = args.n_cont == N_CONT
    traffic = {"nodeset_rows_kernel": 0.497e9 + 2.184e9, "fold_kernel": 1.09e6, "potential_kernel": 0.66e6,
               "dot_kernel": 0.498e9 + 0.004e9, "semisep_kernel": 2.191e9 + 0.004e9} if args.engine == "semisep" else {}

    def hbm_roof(kernel, nbytes, t_ms, note):
        ach = nbytes / (t_ms * 1e-3) / 1e9
        return {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                "traffic": traffic.get(kernel) if default_size else None, "kernel": kernel, "ms": t_ms,
                "algorithmic_bytes": nbytes, "peak_source": peak_src, "note": note}
    kernels = [
        hbm_roof("nodeset_rows_kernel", sum(p.nodesets.algorithmic_bytes() for p in preps), split["nodesets_ms"],
                 "algorithmic bytes = per node set 8*2*N grid doubles read, plus 8*(3*n1 + 5*N) operator "
                 "doubles written when stored, or (sets serving one pair, applied at once to its folds) each "
                 "folded function read once and every fold output written; the kernel is issue/latency bound "
                 "(per-row loops over the CC nodes)"),
        hbm_roof("fold_kernel", sum(p.fold_bytes() for p in preps), split["folds_ms"],
                 "algorithmic bytes = every distinct operand array (band operators, continuum waves, bound "
                 "states) read once over its longest use + every output written"),
    ]
    if tc:
        t_ms = split["forms_exchange_tensor_ms"]
        useful = sum(p.tensor_flops()[0] for p in preps)
        executed = sum(p.tensor_flops()[1] for p in preps)
        bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
        ach = executed / (t_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": bf16_peak, "unit": "TFLOP/s", "frac": ach / bf16_peak,
                "traffic": None, "kernel": "tc_exchange_kernel",
                "useful_tflops": useful / (t_ms * 1e-3) / 1e12,
                "note": "achieved = executed bf16 MMA flops (2*M*N*K per product, 3 or 6 products of the split) / "
                        "kernel time; useful = dense-equivalent 2*n_rows*n_cols per exchange integral"}
    elif args.engine == "semisep":
        sb = {}
        for p in preps:
            for k, v in p.form_launch.stage_bytes().items():
                sb[k] = sb.get(k, 0.0) + v
        kernels.append(hbm_roof("potential_kernel", sb["potentials"], sub_ms["potentials"],
                                "algorithmic bytes = b and r read, (L_max+1) potential rows written, per transition"))
        kernels.append(hbm_roof("dot_kernel", sb["dots"], sub_ms["dots"],
                                "algorithmic bytes = each pair's folded density a read once per transition, each "
                                "potential tile once per run of 16 pairs"))
        roof = hbm_roof("semisep_kernel", sb["semisep"], sub_ms["semisep"],
                        "algorithmic bytes = 8*(n_rows + n_cols + n_grid) per exchange form (a, b, r read once)")
    else:
        ach = flops / (forms_ms * 1e-3) / 1e12
        roof = {"bound": "fp64", "achieved": ach, "peak": None, "unit": "TFLOP/s (dense-equivalent 2 n1 n2 per L)",
                "frac": None, "traffic": None, "kernel": "dense_tri_kernel", "ms": forms_ms}
    if not tc:
        roof.setdefault("ms", forms_ms)
    kernels.append(roof)
    roof = max(kernels, key=lambda k: k.get("ms", 0.0) if k["bound"] != "tensor" else float("inf"))

    # end to end through the public API from host arrays
    e2e = None
    if not args.no_e2e:
        def e2e_step():
            cache.clear()  # every step rebuilds its quadrature operators and re-uploads its inputs
            return radial_ME_all_L_batch(g, zeros, zeros, b_i, b_f, pairs, L_MAX, U_f_array=zeros,
                                         gpu_cache=cache, engine=args.engine)
        e2e_step()
        barrier()
        # median of several steps, each from host inputs to results and closed by a synchronize (the
        # host share of a step varies with the load of the host cores)
        e_steps = max(1, min(args.steps, 7))

        def timed(fn):
            ts = []
            for _ in range(e_steps):
                barrier()
                t0 = time.perf_counter()
                fn()
                barrier()
                ts.append((time.perf_counter() - t0) * 1e3)
            return float(np.median(ts))
        e_ms = timed(e2e_step)
        if world > 1:
            tt = torch.tensor([e_ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e_ms = float(tt.item())
        uniq_waves = len({id(w) for pr in pairs for w in pr})
        h2d = (uniq_waves + 2 * len(bounds)) * N_GRID * 8
        d2h = len(bounds) * len(pairs) * 2 * (L_MAX + 1) * 8
        # the same call returning the two result arrays instead of a result object per pair
        def e2e_arrays():
            cache.clear()
            return radial_ME_all_L_batch(g, zeros, zeros, b_i, b_f, pairs, L_MAX, U_f_array=zeros,
                                         gpu_cache=cache, engine=args.engine, as_arrays=True)
        e2e_arrays()
        barrier()
        a_ms = timed(e2e_arrays)
        if world > 1:
            tt = torch.tensor([a_ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            a_ms = float(tt.item())
        e2e = {"value": world * n_int / (e_ms * 1e-3), "unit": "integrals/s", "ms_per_step": e_ms,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "path": "radial_ME_all_L_batch (4 transitions x 2048 pairs) from pinned host NumPy inputs to one "
                       "RadialDWBAIntegrals per (transition, pair)", "steps": e_steps,
               "timing": "median over the steps of the wall time of one call, synchronized on both sides",
               "as_arrays_ms_per_step": a_ms, "as_arrays_value": world * n_int / (a_ms * 1e-3)}

    # the same batch through the split-BF16 tensor-core form and the plain FP64 kernel (whole step,
    # node sets rebuilt), so the line carries the split-BF16 vs FP64 comparison of the metric
    compare = None
    if rank == 0 and world == 1 and not args.no_compare:
        def time_engine(eng, warm, reps):
            pj = PreparedJob(job, cache.dg, eng, plans=preps[0].plans, rebuild_nodesets=True)
            for _ in range(warm):
                pj.launch()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                pj.launch()
            e1.record(st)
            e1.synchronize()
            out = e0.elapsed_time(e1) / reps
            del pj
            torch.cuda.empty_cache()
            return out
        t_x3 = time_engine("tc_bf16x3", 2, 5)
        t_dense = time_engine("dense", 1, 1)
        compare = {"tc_bf16x3_ms_per_step": t_x3, "dense_fp64_ms_per_step": t_dense,
                   "split_bf16_vs_plain_fp64_speedup": t_dense / t_x3,
                   "semisep_fp64_ms_per_step": ms if args.engine == "semisep" else None,
                   "note": "whole step (node sets, folds, forms) on the same batch; the accuracy of each engine "
                           "against the reference's TCS is checked in tests/test_gpu_config1.py"}

    # the 64-energy ragged sweep: exact FP64 (semiseparable) engine, and unless --no-compare the
    # split-BF16 tensor-core engine and the plain FP64 kernel on the same points, with the TCS of
    # every point from the split-BF16 integrals against the FP64 ones
    ragged = None
    if rank == 0 and world == 1 and not args.no_ragged and args.engine in ("semisep", "dense"):
        points = make_ragged_points()
        ragged, ref_outs = ragged_sweep("semisep", points=points)
        if not args.no_compare:
            r_x3, x3_outs = ragged_sweep("tc_bf16x3", replays=3, points=points, split=False)
            worst, med = sweep_tcs_errors(points, ref_outs, x3_outs)
            del x3_outs
            r_dense, dense_outs = ragged_sweep("dense", replays=1, points=points, split=False)
            worst_d, _ = sweep_tcs_errors(points, ref_outs, dense_outs)
            del dense_outs
            ragged["engines"] = {
                "tc_bf16x3_ms_per_sweep": r_x3["ms_per_sweep"], "dense_fp64_ms_per_sweep": r_dense["ms_per_sweep"],
                "split_bf16_vs_plain_fp64_speedup": r_dense["ms_per_sweep"] / r_x3["ms_per_sweep"],
                "semisep_fp64_vs_plain_fp64_speedup": r_dense["ms_per_sweep"] / ragged["ms_per_sweep"],
                "tc_bf16x3_tcs_rel_err_max": worst, "tc_bf16x3_tcs_rel_err_median": med,
                "tc_bf16x3_guard_routed": r_x3.get("tc_guard_routed"), "tc_bf16x3_tile": r_x3.get("tc_tile"),
                "dense_fp64_tcs_rel_err_max": worst_d,
                "note": "TCS of every (energy, transition) point from each engine's integrals against the exact "
                        "FP64 semiseparable engine's (which agrees with the oracle to 1e-12 per integral)"}

    grad = dropin = None
    if rank == 0 and world == 1 and not args.no_ragged and args.engine in ("semisep", "dense"):
        grad = gradient_run()
        dropin = dropin_run()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ips, dt, rows = cpu_sample(seconds_hint=15.0)
        cpu = {"value": ips, "unit": "integrals/s", "cores": 1, "kind": "port",
               "sample": f"oracle port of the reference CPU algorithm, {rows} of {N_GRID} rows of one pair, "
                         f"L=0..8 direct+exchange, {dt:.1f} s, scaled by rows/n1"}
        try:
            import threadpoolctl
            cpu["cores"] = max(i.get("num_threads", 1) for i in threadpoolctl.threadpool_info()) or 1
        except Exception:
            pass
    if rank == 0:
        per_forms = {"dense": 2, "semisep": 1, "tc_bf16x3": 5, "tc_bf16x6": 5}[args.engine]
        n_launch = sum((1 if p.nodesets.n else 0) + (1 if p.nodesets.n_fused else 0) + (p.n_folds + 65534) // 65535 +
                       (p.n_multi + 65534) // 65535 +
                       per_forms for p in preps)
        line = {"metric": METRIC, "value": value, "unit": "integrals/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16 split (x3/x6) + f64" if tc else "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "engine": args.engine, "integrals_per_step_per_gpu": n_int,
                           "l2": "inputs larger than L2 (operands ~1 GB/step)", "parallelism": f"dp{world}"},
                "split_ms": split, "roofline": roof, "kernels": kernels, "e2e": e2e, "cpu_baseline": cpu,
                "engines": compare, "ragged_sweep": ragged, "gradient": grad, "dropin": dropin,
                "gpu_launches": n_launch * args.steps, "results_finite": bool(finite and nonzero), "clocks": clk.summary()}
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
