"""The oracle's O(N L) semiseparable evaluation against its dense restatement of the reference's
kernel (K_L = (1/r_>) exp(L log(min(r_</r_>, 1-1e-12) + 1e-300)), dwba_matrix_elements.py:1057-1116)
at the full sizes of the measured workloads, where (r_max/r_min)^(L+1) reaches 1e68 to 1e80. The
GPU parity tests at those sizes (tests/test_gpu_fullsize.py) use the semiseparable evaluation as
their checker; this pins it to the dense form there."""
import numpy as np

import bench
from oracle.folded import fold_pair, folded_eval, semiseparable_eval


def _pair(r, l1, k1, l2, k2, seed):
    rng = np.random.default_rng(seed)
    out = []
    for l, k in ((l1, k1), (l2, k2)):
        d = float(rng.uniform(0.0, np.pi))
        out.append(bench._Wave(l, k, d, np.sin(k * r - 0.5 * l * np.pi + d) *
                               (1.0 - np.exp(-(r / ((l + 1) / k)) ** (l + 1)))))
    return out


def _agree(r, a, b, L_max, tol):
    s = semiseparable_eval(r, a, b, L_max)
    d = folded_eval(r, a, b, L_max)
    scale = semiseparable_eval(r, np.abs(a), np.abs(b), L_max)
    assert np.all(np.abs(s - d) <= 1e-13 * np.abs(d) + tol * scale), (s, d, np.abs(s - d) / scale)


def test_kernel_batch_size_exchange_form():
    """N = 15000 on [1e-5, 400], L = 0..8, l = 63 against l = 0 (exchange form of the widest node set)."""
    g, zeros, bounds, _ = bench.make_workload(15000, n_cont=1)
    ci, cf = _pair(g.r, 0, 8.0, 63, 7.5, 3)
    fp = fold_pair(g, zeros, zeros, bounds[0][0], bounds[0][1], ci, cf, 8, U_f_array=zeros)
    assert fp["n1"] == 15000
    _agree(g.r, fp["a_ex"], fp["b_ex"], 8, 1e-15)


def test_ionization_size_direct_form():
    """N = 8000 on [1e-5, 200], L = 0..10, an ejected Coulomb wave as the final state (direct form,
    full-grid inner integral)."""
    pts = bench.make_ionization_points(select=(0,))
    pt = pts[0]
    ci, cf = pt["pairs"][-1]
    fp = fold_pair(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"][-1], pt["bound_f"][-1], ci, cf, 10,
                   U_f_array=pt["U_f_array"])
    _agree(pt["grid"].r, fp["a_dir"], fp["b_dir"], 10, 1e-15)


def _tap_rounding_bound(grid, bi, bf, ci, cf, L_max, n1, phase_increment=1.5708, n_cc=5):
    """First-order bound of what the reference's rounding of its interpolation taps does to a direct
    integral I_L = sum_c W_c (P f)_c (P phi_L)_c (f = chi_f chi_i, phi_L = K_L (w u_f u_i)): each tap
    t = (q - q_j)/(q_{j+1} - q_j) (q = log r on log grids) is off by at most
        dt = eps [(|q| + |q_j|) + t (|q_{j+1}| + |q_j|)] / (q_{j+1} - q_j) + eps,
    and dI/dt_c = W_c [(f_{j+1} - f_j)(P phi)_c + (P f)_c (phi_{j+1} - phi_j)]."""
    from oracle.folded import _interp_op
    from oracle.quadrature import adaptive_phase_increment, cc_nodes_on_breakpoints, generate_phase_nodes, \
        is_log_spaced_grid
    eps = np.finfo(float).eps
    r, w = np.asarray(grid.r), np.asarray(grid.w_simpson)
    k_total, eta = ci.k_au + cf.k_au, ci.eta + cf.eta
    d = adaptive_phase_increment(r[:n1], k_total, phase_increment, eta_total=eta)
    X, W, _ = cc_nodes_on_breakpoints(generate_phase_nodes(r[0], r[n1 - 1], k_total, d, eta_total=eta), n_cc)
    x = r[:n1]
    j, t = _interp_op(X, x)
    q, xp = (np.log(np.clip(X, x[0], x[-1])), np.log(x)) if is_log_spaced_grid(x) else (np.clip(X, x[0], x[-1]), x)
    dt = eps * ((np.abs(q) + np.abs(xp[j])) + t * (np.abs(xp[j + 1]) + np.abs(xp[j]))) / (xp[j + 1] - xp[j]) + eps
    f = (cf.chi_of_r * ci.chi_of_r)[:n1]
    b = w * bf.u_of_r * bi.u_of_r
    Pf = f[j] * (1 - t) + f[j + 1] * t
    out = np.zeros(L_max + 1)
    for L in range(L_max + 1):
        p, s = r ** L, r ** (-(L + 1))
        phi = (s * (np.cumsum(p * b) - p * b) + p * (np.cumsum((s * b)[::-1])[::-1] - s * b) + b / r)[:n1]
        Pp = phi[j] * (1 - t) + phi[j + 1] * t
        out[L] = np.sum(W * dt * (np.abs(f[j + 1] - f[j]) * np.abs(Pp) + np.abs(Pf) * np.abs(phi[j + 1] - phi[j])))
    return out


def test_engine_taps_differ_from_the_reference_taps_by_their_rounding_only():
    """At N = 15000 on [1e-5, 400] the kernel's log taps (series of log(1 + u)) and the reference's
    (difference of two rounded logs) give direct integrals that differ by up to ~3e-14 S_L; the
    difference stays inside the first-order bound of the reference's tap rounding, while the
    exchange integrals (whose inner taps are linear in r) agree to round-off."""
    from golden_cases import fullsize_batch_inputs
    from kernel_model import engine_interp_op
    g, zeros, bounds, pairs = fullsize_batch_inputs()
    r = np.asarray(g.r)
    bi, bf = bounds[0]
    seen = 0.0
    for p in (0, 1, 4, 5):
        ci, cf = pairs[p]
        ref = fold_pair(g, zeros, zeros, bi, bf, ci, cf, 8, U_f_array=zeros)
        eng = fold_pair(g, zeros, zeros, bi, bf, ci, cf, 8, U_f_array=zeros, interp_op=engine_interp_op)
        d_ref = semiseparable_eval(r, ref["a_dir"], ref["b_dir"], 8)
        d_eng = semiseparable_eval(r, eng["a_dir"], eng["b_dir"], 8)
        scale = semiseparable_eval(r, np.abs(ref["a_dir"]), np.abs(ref["b_dir"]), 8)
        bound = _tap_rounding_bound(g, bi, bf, ci, cf, 8, ref["n1"])
        assert np.all(np.abs(d_ref - d_eng) <= bound), (p, np.abs(d_ref - d_eng), bound)
        seen = max(seen, float(np.max(np.abs(d_ref - d_eng) / scale)))
        e_ref = semiseparable_eval(r, ref["a_ex"], ref["b_ex"], 8)
        e_eng = semiseparable_eval(r, eng["a_ex"], eng["b_ex"], 8)
        e_scale = semiseparable_eval(r, np.abs(ref["a_ex"]), np.abs(ref["b_ex"]), 8)
        assert np.all(np.abs(e_ref - e_eng) <= 3e-15 * e_scale), (p, np.abs(e_ref - e_eng) / e_scale)
    assert seen > 1e-14  # the deviation is real at this size
