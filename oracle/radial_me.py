"""NumPy restatement of the reference ``radial_ME_all_L`` (CPU semantics) -- oracle only.

Follows ``dwba_matrix_elements.py:780-1300`` and the 2-D quadrature of
``oscillatory_integrals.py:2385-2777``. Like the reference it materialises the
dense N x N multipole kernels, so it is meant for grids of a few thousand
points (it is also the CPU baseline the benchmark times).
"""
from __future__ import annotations

import numpy as np

from .quadrature import (adaptive_phase_increment, cc_nodes_on_breakpoints, generate_phase_nodes,
                         interp_on_radial_grid)
from .tails import analytical_multipole_tail, outer_integral_1d


def _is_excitation(bound_f) -> bool:
    # dwba_matrix_elements.py:1124 uses isinstance(bound_f, BoundOrbital); a ContinuumWave has chi_of_r.
    return not hasattr(bound_f, "chi_of_r")


def select_idx_limit(r, w_trapz, U_i, U_f, u_i, u_f, k_i, k_f, l_i, l_f, idx_match_i, idx_match_f,
                     min_grid_fraction=0.10):
    """Integration limit n1 for r1; ``dwba_matrix_elements.py:909-1022``."""
    N = len(r)
    n1 = N
    if 0 < idx_match_i < N:
        n1 = min(n1, idx_match_i + 1)
    if 0 < idx_match_f < N:
        n1 = min(n1, idx_match_f + 1)
    k_eff = min(k_i, k_f) if min(k_i, k_f) > 0.1 else max(k_i, k_f)
    lmax = max(l_i, l_f)
    if k_eff > 1e-3:
        r_turn = (lmax + 0.5) / k_eff
        idx_turn = int(np.searchsorted(r, r_turn))
        idx_turn = min(idx_turn, N - 20)
        min_idx = min(max(idx_turn + 20, int(N * min_grid_fraction)), N)
    else:
        min_idx = max(1, int(N * min_grid_fraction))
    if n1 < min_idx:
        n1 = min_idx
    idx99 = 0
    for u in (u_i, u_f):
        usq = u ** 2
        if np.sum(usq) > 1e-30:
            pc = np.cumsum(usq * w_trapz)
            pc /= (pc[-1] + 1e-300)
            idx99 = max(idx99, int(np.searchsorted(pc, 0.99)))
    if idx99 > n1:
        n1 = idx99 + 1

    def veff(i):
        ui = abs(U_i[i])
        uf = abs(U_f[i]) if U_f is not None else 0.0
        return max(ui, uf) + (lmax * (lmax + 1)) / (2.0 * r[i] ** 2)

    ke = 0.5 * min(k_i, k_f) ** 2
    if ke > 1e-10:
        if veff(max(0, n1 - 1)) / ke > 0.03:
            for t in range(n1, min(n1 + 500, N)):
                if veff(t) / ke < 0.03:
                    n1 = t + 1
                    break
    return n1


def _kernel_integral_2d(rho1, rho2, K, r, k_total, n1, method, w, n_nodes, dphi_req, eta_total):
    """``oscillatory_integrals.py:2385-2777`` for methods standard / filon / filon_exchange
    (with ``idx_limit_r2`` left at its default: the full grid)."""
    N = len(r)
    if n1 < 2:
        return 0.0
    rho1 = np.nan_to_num(rho1[:n1].copy(), nan=0.0, posinf=0.0, neginf=0.0)
    rho2 = np.nan_to_num(rho2[:N].copy(), nan=0.0, posinf=0.0, neginf=0.0)
    Klim = K[:n1, :N]
    r1 = r[:n1]
    w1, w2 = w[:n1], w[:N]
    if method == "filon":
        inner = Klim @ (rho2 * w2)
        inner = np.nan_to_num(inner, nan=0.0, posinf=0.0, neginf=0.0)
        d = adaptive_phase_increment(r1, k_total, dphi_req, eta_total=eta_total)
        if k_total < 1e-6:
            res = float(np.dot(rho1 * w1, inner))
        else:
            br = generate_phase_nodes(r1[0], r1[-1], k_total, d, eta_total=eta_total)
            if len(br) - 1 < 1:
                res = float(np.dot(rho1 * w1, inner))
            else:
                X, W, nv = cc_nodes_on_breakpoints(br, n_nodes)
                if nv == 0:
                    res = float(np.dot(rho1 * w1, inner))
                else:
                    res = float(np.sum(interp_on_radial_grid(X, r1, rho1) * interp_on_radial_grid(X, r1, inner) * W))
    elif method == "filon_exchange":
        d = adaptive_phase_increment(r1, k_total, dphi_req, eta_total=eta_total)
        br = generate_phase_nodes(r1[0], r1[-1], k_total, d, eta_total=eta_total) if k_total >= 1e-6 else None
        if br is None or len(br) - 1 < 1:
            res = float(np.dot(rho1 * w1, Klim @ (rho2 * w2)))
        else:
            X, W, nv = cc_nodes_on_breakpoints(br, n_nodes)
            if nv == 0:
                res = float(np.dot(rho1 * w1, Klim @ (rho2 * w2)))
            else:
                rho2_cc = interp_on_radial_grid(X, r, rho2)
                iR = np.clip(np.searchsorted(r, X), 1, N - 1)
                iL = iR - 1
                wR = (X - r[iL]) / (r[iR] - r[iL] + 1e-30)
                wL = 1.0 - wR
                # kernel columns linearly interpolated at the CC nodes (n1 x N_cc temporaries)
                Kcc = Klim[:, iL] * wL + Klim[:, iR] * wR
                inner = Kcc @ (rho2_cc * W)
                res = float(np.sum(interp_on_radial_grid(X, r1, rho1) * interp_on_radial_grid(X, r1, inner) * W))
    else:
        raise ValueError(method)
    return res if np.isfinite(res) else 0.0


def radial_me_all_L(grid, V_core, U_i, bound_i, bound_f, cont_i, cont_f, L_max,
                    use_oscillatory_quadrature=True, oscillatory_method="advanced", CC_nodes=5,
                    phase_increment=1.5708, min_grid_fraction=0.10, k_threshold=0.5, U_f_array=None):
    """Restatement of ``radial_ME_all_L`` (``dwba_matrix_elements.py:780-1300``).

    Returns ``(I_L_direct, I_L_exchange)`` as dicts ``{L: float}``.
    """
    if L_max < 0:
        raise ValueError("radial_ME_all_L: L_max must be >= 0.")
    r = np.asarray(grid.r, dtype=float)
    w = np.asarray(grid.w_simpson, dtype=float)
    w_trapz = np.asarray(grid.w_trapz, dtype=float)
    N = len(r)
    u_i, u_f = bound_i.u_of_r, bound_f.u_of_r
    chi_i, chi_f = cont_i.chi_of_r, cont_f.chi_of_r
    k_i, k_f, l_i, l_f = cont_i.k_au, cont_f.k_au, cont_i.l, cont_f.l
    n1 = select_idx_limit(r, w_trapz, U_i, U_f_array, u_i, u_f, k_i, k_f, l_i, l_f,
                          getattr(cont_i, "idx_match", -1), getattr(cont_f, "idx_match", -1),
                          min_grid_fraction)
    wl = w.copy()
    wl[n1:] = 0.0
    rho1_dir_w, rho2_dir_w = wl * chi_f * chi_i, wl * u_f * u_i
    rho1_ex_w, rho2_ex_w = wl * u_f * chi_i, wl * chi_f * u_i
    rho1_dir, rho2_dir = chi_f * chi_i, u_f * u_i
    rho1_ex, rho2_ex = u_f * chi_i, chi_f * u_i
    V_diff = V_core - U_i
    # dense base matrices (dwba_matrix_elements.py:1057-1080)
    rl = np.minimum(r[:, None], r[None, :])
    rg = np.maximum(r[:, None], r[None, :])
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = rl / rg
        inv_gtr = 1.0 / rg
    ratio[~np.isfinite(ratio)] = 0.0
    inv_gtr[~np.isfinite(inv_gtr)] = 0.0
    log_ratio = np.log(np.minimum(ratio, 1.0 - 1e-12) + 1e-300)
    del rl, rg, ratio
    d_i = getattr(cont_i, "phase_shift", 0.0)
    d_f = getattr(cont_f, "phase_shift", 0.0)
    e_i = getattr(cont_i, "eta", 0.0)
    e_f = getattr(cont_f, "eta", 0.0)
    s_i = getattr(cont_i, "sigma_l", 0.0)
    s_f = getattr(cont_f, "sigma_l", 0.0)
    eta_total = e_i + e_f
    k_total = k_i + k_f
    r_match = r[n1 - 1] if n1 > 0 else r[-1]
    exc = _is_excitation(bound_f)
    osc = use_oscillatory_quadrature and k_total > k_threshold
    out_d, out_e = {}, {}
    for L in range(L_max + 1):
        K = inv_gtr if L == 0 else inv_gtr * np.exp(L * log_ratio)
        if osc:
            I_d = _kernel_integral_2d(rho1_dir, rho2_dir, K, r, k_total, n1, "filon", w, CC_nodes,
                                      phase_increment, eta_total)
            if oscillatory_method != "legacy" and L >= 1 and n1 < N - 10 and exc:
                mom = np.sum(w * (r ** L) * u_f * u_i)
                if abs(mom) > 1e-12:
                    env = (lambda m, LL: (lambda x: m / (x ** (LL + 1)) if x > 1e-6 else 0.0))(mom, L)
                    t = outer_integral_1d(env, k_i, l_i, d_i, e_i, s_i, k_f, l_f, d_f, e_f, s_f,
                                          r_match, r[-1], delta_phi=np.pi / 4)
                    t += analytical_multipole_tail(r[-1], k_i, k_f, d_i, d_f, l_i, l_f, L, mom,
                                                   e_i, e_f, s_i, s_f)
                    I_d += t
        else:
            I_d = np.dot(rho1_dir_w, K @ rho2_dir_w)
        if L == 0:
            s2 = np.sum(rho2_dir_w)
            if abs(s2) > 1e-12:
                I_d += np.dot(rho1_dir_w, V_diff) * s2
        if oscillatory_method == "legacy" and L >= 1 and use_oscillatory_quadrature and n1 < N - 10 and exc:
            mom = np.sum(w * (r ** L) * u_f * u_i)
            if abs(mom) > 1e-12:
                I_d += analytical_multipole_tail(r_match, k_i, k_f, d_i, d_f, l_i, l_f, L, mom,
                                                 e_i, e_f, s_i, s_f)
        out_d[L] = float(I_d)
        if osc:
            I_e = _kernel_integral_2d(rho1_ex, rho2_ex, K, r, k_total, n1, "filon_exchange", w, CC_nodes,
                                      phase_increment, eta_total)
        else:
            I_e = np.dot(rho1_ex_w, K @ rho2_ex_w)
        if L == 0:
            s2e = np.sum(rho2_ex_w)
            if abs(s2e) > 1e-12:
                I_e += np.dot(rho1_ex_w, V_diff) * s2e
        out_e[L] = float(I_e)
    return out_d, out_e
