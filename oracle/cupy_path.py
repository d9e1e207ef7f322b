"""NumPy restatement of the reference's CuPy path ``radial_ME_all_L_gpu`` -- oracle only.

Follows ``dwba_matrix_elements.py:1563-2549`` (with ``_generate_gpu_filon_params`` :1350-1414,
``_gpu_filon_direct`` :1416-1465, ``_gpu_filon_exchange`` :1469-1560 and
``_refine_idx_limit_physics`` :688-777). Its quadrature differs from the CPU path's:
* phase intervals: linspace on [r_0, r_{n1-1}] with the raw step phase_increment / k_total
  (no adaptive clamp, no Coulomb phase), at least two intervals, else the standard form;
* every interpolation is linear in r on r[:n1] (``cp.interp``);
* the exchange inner sum runs over the CC nodes of r[:n1] with the kernel at each node formed from
  the linearly interpolated 1/r_> and log-ratio of its bracketing grid columns (``:2072-2091``);
* the L=0 corrections are added without the overlap gate; the legacy tail uses the moments of
  r[:n1]; the final state's extent counts only for a bound final state.
Like the reference it materialises the n1 x N_cc kernel at the CC nodes: small grids only.
"""
from __future__ import annotations

import numpy as np

from .quadrature import cc_table_rule
from .radial_me import _is_excitation
from .tails import analytical_multipole_tail, outer_integral_1d


def select_idx_limit_cupy(r, w_trapz, U_i, U_f, u_i, u_f, k_i, k_f, l_i, l_f, im_i, im_f, min_grid_fraction,
                          final_is_bound):
    """Integration limit of the CuPy path (``dwba_matrix_elements.py:1676-1720`` and ``:688-777``)."""
    N = len(r)
    n1 = N
    if 0 < im_i < N:
        n1 = min(n1, im_i + 1)
    if 0 < im_f < N:
        n1 = min(n1, im_f + 1)
    k_eff = min(k_i, k_f) if min(k_i, k_f) > 0.1 else max(k_i, k_f)
    lmax = max(l_i, l_f)
    if k_eff > 1e-3:
        idx_turn = min(int(np.searchsorted(r, (lmax + 0.5) / k_eff)), N - 20)
        min_idx = min(max(idx_turn + 20, int(N * min_grid_fraction)), N)
    else:
        min_idx = max(1, int(N * min_grid_fraction))
    n1 = max(n1, min_idx)
    n1 = int(max(1, min(n1, N)))
    idx99 = 0
    for u in ([u_i, u_f] if final_is_bound else [u_i]):
        usq = np.asarray(u)[:N] ** 2
        if float(np.sum(usq)) <= 1e-30:
            continue
        pc = np.cumsum(usq * w_trapz[:N])
        tot = float(pc[-1])
        if tot <= 1e-300 or not np.isfinite(tot):
            continue
        pc /= tot + 1e-300
        idx99 = max(idx99, int(np.searchsorted(pc, 0.99)))
    if idx99 > n1:
        n1 = min(N, idx99 + 1)
    ke = 0.5 * min(k_i, k_f) ** 2
    if ke > 1e-10 and n1 > 0:
        def veff(i):
            ri = max(float(r[i]), 1e-12)
            return max(abs(float(U_i[i])), abs(float(U_f[i])) if U_f is not None else 0.0) + lmax * (lmax + 1) / (2 * ri * ri)
        if veff(max(0, min(n1 - 1, N - 1))) / ke > 0.03:
            for t in range(n1, min(n1 + 500, N)):
                if veff(t) / ke < 0.03:
                    n1 = t + 1
                    break
    return int(max(1, min(n1, N)))


def filon_params_cupy(r1, k_total, phase_increment, n_nodes):
    """CC nodes X, weights W and the bracketing columns of the CuPy path (``:1350-1414``); None when it
    falls back to the standard form."""
    if k_total < 1e-6:
        return None
    dr = phase_increment / k_total
    n_int = max(1, int(np.ceil((float(r1[-1]) - float(r1[0])) / dr)))
    br = np.linspace(float(r1[0]), float(r1[-1]), n_int + 1)
    if n_int < 2:
        return None
    a, b = br[:-1], br[1:]
    ok = (b - a) > 1e-12
    a, b = a[ok], b[ok]
    if len(a) == 0:
        return None
    x_ref, w_ref = cc_table_rule(n_nodes)  # the CuPy path's rule for every node count
    hw = 0.5 * (b - a)
    X = (hw[:, None] * (np.asarray(x_ref) + 1) + a[:, None]).ravel()
    W = (np.asarray(w_ref)[None, :] * hw[:, None]).ravel()
    iR = np.clip(np.searchsorted(r1, X), 1, len(r1) - 1)
    iL = iR - 1
    wR = (X - r1[iL]) / (r1[iR] - r1[iL] + 1e-30)
    return dict(X=X, W=W, iL=iL, iR=iR, wL=1.0 - wR, wR=wR)


def radial_me_all_L_cupy(grid, V_core, U_i, bound_i, bound_f, cont_i, cont_f, L_max,
                         use_oscillatory_quadrature=True, oscillatory_method="advanced", CC_nodes=5,
                         phase_increment=1.5708, min_grid_fraction=0.10, k_threshold=0.5, U_f_array=None):
    """Restatement of ``radial_ME_all_L_gpu``; returns ``(I_L_direct, I_L_exchange)`` dicts."""
    r = np.asarray(grid.r, dtype=float)
    w = np.asarray(grid.w_simpson, dtype=float)
    N = len(r)
    exc = _is_excitation(bound_f)
    u_i, u_f = np.asarray(bound_i.u_of_r)[:N], np.asarray(bound_f.u_of_r)[:N]
    k_i, k_f, l_i, l_f = cont_i.k_au, cont_f.k_au, cont_i.l, cont_f.l
    n1 = select_idx_limit_cupy(r, np.asarray(grid.w_trapz, dtype=float), U_i, U_f_array, u_i, u_f, k_i, k_f, l_i, l_f,
                               getattr(cont_i, "idx_match", -1), getattr(cont_f, "idx_match", -1), min_grid_fraction,
                               exc)
    r1, w1 = r[:n1], w[:n1]
    chi_i, chi_f = np.asarray(cont_i.chi_of_r)[:n1], np.asarray(cont_f.chi_of_r)[:n1]
    ui1, uf1 = u_i[:n1], u_f[:n1]
    rho1_dir_uw, rho2_dir_uw = chi_f * chi_i, uf1 * ui1
    rho1_ex_uw, rho2_ex_uw = uf1 * chi_i, chi_f * ui1
    rho1_dir_w, rho2_dir_w = w1 * rho1_dir_uw, w1 * rho2_dir_uw
    rho1_ex_w, rho2_ex_w = w1 * rho1_ex_uw, w1 * rho2_ex_uw
    V_diff = (np.asarray(V_core) - np.asarray(U_i))[:n1]
    k_total = k_i + k_f
    osc = use_oscillatory_quadrature and k_total > k_threshold
    prm = filon_params_cupy(r1, k_total, phase_increment, CC_nodes) if osc else None
    use_filon = osc and prm is not None

    def kernel(rows, cols):
        inv = 1.0 / np.maximum(rows[:, None], cols[None, :] + 1e-30)
        ratio = np.minimum(np.minimum(rows[:, None], cols[None, :]) * inv, 1.0 - 1e-12)
        return inv, np.log(ratio + 1e-30)
    inv_s, lr_s = kernel(r1, r1)
    if use_filon:
        inv_f, lr_f = kernel(r1, r)
        rho2_full = u_f * u_i * w
        X, W, iL, iR, wL, wR = (prm[k] for k in ("X", "W", "iL", "iR", "wL", "wR"))

        def at_cc(c):
            inv_c = 1.0 / np.maximum(r1[:, None], r1[c][None, :] + 1e-30)
            lr_c = np.log(np.minimum(r1[:, None], r1[c][None, :]) * inv_c + 1e-30)
            return inv_c, lr_c
        invL, lrL = at_cc(iL)
        invR, lrR = at_cc(iR)
        inv_cc = invL * wL + invR * wR
        lr_cc = lrL * wL + lrR * wR
        del invL, lrL, invR, lrR
        rho1d_cc = np.interp(X, r1, rho1_dir_uw)
        rho1e_cc = np.interp(X, r1, rho1_ex_uw)
        rho2e_cc = np.interp(X, r1, rho2_ex_uw)
    d_i, d_f = getattr(cont_i, "phase_shift", 0.0), getattr(cont_f, "phase_shift", 0.0)
    e_i, e_f = getattr(cont_i, "eta", 0.0), getattr(cont_f, "eta", 0.0)
    s_i, s_f = getattr(cont_i, "sigma_l", 0.0), getattr(cont_f, "sigma_l", 0.0)
    r_match = r[n1 - 1] if n1 > 0 else r[-1]
    out_d, out_e = {}, {}
    for L in range(L_max + 1):
        K = inv_s if L == 0 else inv_s * np.exp(L * lr_s)
        if use_filon:
            Kf = inv_f if L == 0 else inv_f * np.exp(L * lr_f)
            int_r2 = Kf @ rho2_full
            I_d = float(np.sum(rho1d_cc * np.interp(X, r1, int_r2) * W))
            if L >= 1 and n1 < N - 10 and exc:
                if oscillatory_method == "legacy":
                    mom = float(np.dot(w1 * uf1 * ui1, r1 ** L))
                    if abs(mom) > 1e-12:
                        I_d += analytical_multipole_tail(r_match, k_i, k_f, d_i, d_f, l_i, l_f, L, mom, e_i, e_f,
                                                         s_i, s_f)
                else:
                    mom = float(np.dot(w * u_f * u_i, r ** L))
                    if abs(mom) > 1e-12:
                        env = (lambda m, LL: (lambda x: m / (x ** (LL + 1)) if x > 1e-6 else 0.0))(mom, L)
                        t = outer_integral_1d(env, k_i, l_i, d_i, e_i, s_i, k_f, l_f, d_f, e_f, s_f, r_match, r[-1],
                                              delta_phi=np.pi / 4)
                        t += analytical_multipole_tail(r[-1], k_i, k_f, d_i, d_f, l_i, l_f, L, mom, e_i, e_f,
                                                       s_i, s_f)
                        I_d += t
        else:
            I_d = float(np.dot(rho1_dir_w, K @ rho2_dir_w))
        if L == 0:
            I_d += float(np.dot(rho1_dir_w, V_diff) * np.sum(rho2_dir_w))
        out_d[L] = I_d
        if osc and use_filon:
            Kcc = inv_cc if L == 0 else inv_cc * np.exp(L * lr_cc)
            inner = Kcc @ (rho2e_cc * W)
            I_e = float(np.sum(rho1e_cc * np.interp(X, r1, inner) * W))
        else:
            I_e = float(np.dot(rho1_ex_w, K @ rho2_ex_w))
        if L == 0:
            I_e += float(np.dot(rho1_ex_w, V_diff) * np.sum(rho2_ex_w))
        out_e[L] = I_e
    return out_d, out_e
