"""Folded (bilinear) restatement of the reference quadrature -- oracle only.

For every branch of ``dwba_matrix_elements.radial_ME_all_L`` (CPU semantics)
the result is

    I_L = a^T K_L b + c_L + t_L,    K_L[i, j] = (1/r_>) * exp(L * log(min(r_</r_>, 1-1e-12) + 1e-300))

where the vectors ``a`` and ``b`` absorb the Simpson weights, the CC node
weights and both interpolation operators of ``oscillatory_integrals.py:2555-2777``,
``c_L`` is the L=0 correction (``dwba_matrix_elements.py:1249-1296``) and
``t_L`` the outer tail of the direct term. This module builds ``a``/``b`` with
sparse NumPy scatter-adds (an implementation independent of the CUDA engine's
banded operators) and evaluates ``a^T K_L b`` densely in row blocks, or in
O(N L) with the semiseparable split of K_L (j < i: r_j^L / r_i^(L+1)).
"""
from __future__ import annotations

import numpy as np

from .quadrature import adaptive_phase_increment, cc_nodes_on_breakpoints, generate_phase_nodes, is_log_spaced_grid
from .radial_me import _is_excitation, select_idx_limit
from .tails import analytical_multipole_tail, outer_integral_1d


def _interp_op(X, x):
    """(j, t) of np.interp on the grid ``x`` (log r on log grids), after the
    reference's clipping (``oscillatory_integrals.py:279-302``). Value = (1-t) y[j] + t y[j+1]."""
    n = len(x)
    xc = np.clip(X, x[0], x[-1])
    if is_log_spaced_grid(x):
        q, xp = np.log(np.maximum(xc, max(x[0], 1e-300))), np.log(np.maximum(x, 1e-300))
    else:
        q, xp = xc, x
    j = np.clip(np.searchsorted(xp, q, side="right") - 1, 0, n - 2)
    t = (q - xp[j]) / (xp[j + 1] - xp[j])
    return j, t


def _P(j, t, y):
    return y[j] * (1 - t) + y[j + 1] * t


def _PT(j, t, c, n):
    return np.bincount(j, c * (1 - t), n) + np.bincount(j + 1, c * t, n)


def fold_pair(grid, V_core, U_i, bound_i, bound_f, cont_i, cont_f, L_max, use_oscillatory_quadrature=True,
              oscillatory_method="advanced", CC_nodes=5, phase_increment=1.5708, min_grid_fraction=0.10,
              k_threshold=0.5, U_f_array=None, interp_op=None):
    """Folded operands of one (cont_i, cont_f) pair: returns a dict with n1, a_dir, b_dir,
    a_ex, b_ex (length N), corr_dir, corr_ex (L=0 scalars) and tail[L] (added to direct).
    ``interp_op``: (j, t) of the interpolation onto the CC nodes, by default the reference's
    arithmetic (``_interp_op``); a test passes another tap arithmetic to separate its effect."""
    r = np.asarray(grid.r, dtype=float)
    w = np.asarray(grid.w_simpson, dtype=float)
    N = len(r)
    u_i, u_f = bound_i.u_of_r, bound_f.u_of_r
    chi_i, chi_f = cont_i.chi_of_r, cont_f.chi_of_r
    k_i, k_f, l_i, l_f = cont_i.k_au, cont_f.k_au, cont_i.l, cont_f.l
    n1 = select_idx_limit(r, grid.w_trapz, U_i, U_f_array, u_i, u_f, k_i, k_f, l_i, l_f,
                          getattr(cont_i, "idx_match", -1), getattr(cont_f, "idx_match", -1), min_grid_fraction)
    e_i, e_f = getattr(cont_i, "eta", 0.0), getattr(cont_f, "eta", 0.0)
    k_total, eta_total = k_i + k_f, e_i + e_f
    wl = w.copy()
    wl[n1:] = 0.0
    out = dict(n1=n1)
    osc = use_oscillatory_quadrature and k_total > k_threshold
    nodes = None
    if osc and n1 >= 2:
        d = adaptive_phase_increment(r[:n1], k_total, phase_increment, eta_total=eta_total)
        br = generate_phase_nodes(r[0], r[n1 - 1], k_total, d, eta_total=eta_total)
        if len(br) >= 2:
            X, W, nv = cc_nodes_on_breakpoints(br, CC_nodes)
            if nv > 0:
                nodes = (X, W)
    if osc and n1 >= 2 and nodes is not None:
        X, W = nodes
        iop = interp_op or _interp_op
        j1, t1 = iop(X, r[:n1])
        a_dir = np.zeros(N)
        a_dir[:n1] = _PT(j1, t1, W * _P(j1, t1, (chi_f * chi_i)[:n1]), n1)
        a_ex = np.zeros(N)
        a_ex[:n1] = _PT(j1, t1, W * _P(j1, t1, (u_f * chi_i)[:n1]), n1)
        b_dir = w * u_f * u_i
        j2, t2 = iop(X, r)
        cex = W * _P(j2, t2, chi_f * u_i)
        iR = np.clip(np.searchsorted(r, X), 1, N - 1)
        iL = iR - 1
        wR = (X - r[iL]) / (r[iR] - r[iL] + 1e-30)
        b_ex = np.bincount(iL, (1.0 - wR) * cex, N) + np.bincount(iR, wR * cex, N)
    elif osc and n1 >= 2:
        # no valid phase interval: weighted dot products (oscillatory_integrals.py:2580-2587)
        a_dir, b_dir = np.where(np.arange(N) < n1, w * chi_f * chi_i, 0.0), w * u_f * u_i
        a_ex, b_ex = np.where(np.arange(N) < n1, w * u_f * chi_i, 0.0), w * chi_f * u_i
    elif osc:
        a_dir = b_dir = a_ex = b_ex = np.zeros(N)
    else:
        a_dir, b_dir = wl * chi_f * chi_i, wl * u_f * u_i
        a_ex, b_ex = wl * u_f * chi_i, wl * chi_f * u_i
    out.update(a_dir=a_dir, b_dir=b_dir, a_ex=a_ex, b_ex=b_ex)
    V_diff = V_core - U_i
    s2 = np.sum(wl * u_f * u_i)
    out["corr_dir"] = float(np.dot(wl * chi_f * chi_i, V_diff) * s2) if abs(s2) > 1e-12 else 0.0
    s2e = np.sum(wl * chi_f * u_i)
    out["corr_ex"] = float(np.dot(wl * u_f * chi_i, V_diff) * s2e) if abs(s2e) > 1e-12 else 0.0
    tail = np.zeros(L_max + 1)
    exc = _is_excitation(bound_f)
    d_i, d_f = getattr(cont_i, "phase_shift", 0.0), getattr(cont_f, "phase_shift", 0.0)
    s_i, s_f = getattr(cont_i, "sigma_l", 0.0), getattr(cont_f, "sigma_l", 0.0)
    r_match = r[n1 - 1]
    for L in range(1, L_max + 1):
        if not (n1 < N - 10 and exc):
            break
        mom = np.sum(w * (r ** L) * u_f * u_i)
        if abs(mom) <= 1e-12:
            continue
        if oscillatory_method == "legacy":
            if use_oscillatory_quadrature:
                tail[L] = analytical_multipole_tail(r_match, k_i, k_f, d_i, d_f, l_i, l_f, L, mom, e_i, e_f, s_i, s_f)
        elif osc:
            env = (lambda m, LL: (lambda x: m / (x ** (LL + 1)) if x > 1e-6 else 0.0))(mom, L)
            tail[L] = outer_integral_1d(env, k_i, l_i, d_i, e_i, s_i, k_f, l_f, d_f, e_f, s_f, r_match, r[-1])
            tail[L] += analytical_multipole_tail(r[-1], k_i, k_f, d_i, d_f, l_i, l_f, L, mom, e_i, e_f, s_i, s_f)
    out["tail"] = tail
    return out


def folded_eval(r, a, b, L_max, block=1024):
    """Dense a^T K_L b for L = 0..L_max, K generated block by block (reference formula)."""
    r = np.asarray(r, dtype=float)
    N = len(r)
    nz_a = np.nonzero(a)[0]
    nz_b = np.nonzero(b)[0]
    out = np.zeros(L_max + 1)
    if len(nz_a) == 0 or len(nz_b) == 0:
        return out
    ia0, ia1 = nz_a[0], nz_a[-1] + 1
    jb0, jb1 = nz_b[0], nz_b[-1] + 1
    rc = r[jb0:jb1]
    bb = b[jb0:jb1]
    for s in range(ia0, ia1, block):
        e = min(s + block, ia1)
        ri = r[s:e, None]
        rl = np.minimum(ri, rc[None, :])
        rg = np.maximum(ri, rc[None, :])
        inv = 1.0 / rg
        lr = np.log(np.minimum(rl / rg, 1.0 - 1e-12) + 1e-300)
        for L in range(L_max + 1):
            K = inv if L == 0 else inv * np.exp(L * lr)
            out[L] += np.dot(a[s:e], K @ bb)
    return out


def semiseparable_eval(r, a, b, L_max):
    """O(N L) evaluation of a^T K_L b using K_L[i,j] = r_j^L / r_i^(L+1) for j < i
    (and the transpose above the diagonal); the diagonal carries (1-1e-12)^L / r_i."""
    r = np.asarray(r, dtype=float)
    out = np.zeros(L_max + 1)
    for L in range(L_max + 1):
        p = r ** L
        q = r ** (-(L + 1))
        lower = np.cumsum(p * b) - p * b                 # sum_{j<i} r_j^L b_j
        upper = np.cumsum((q * b)[::-1])[::-1] - q * b   # sum_{j>i} r_j^-(L+1) b_j
        diag = np.exp(L * np.log(1.0 - 1e-12)) / r
        out[L] = np.dot(a, q * lower) + np.dot(a, p * upper) + np.dot(a, diag * b)
    return out
