"""Quadrature building blocks of the reference, restated in NumPy (oracle only).

Reference files: ``oscillatory_integrals.py`` (CC weights, phase splitting,
log-grid interpolation).
"""
from __future__ import annotations

import numpy as np


def cc_table_rule(n: int):
    """The module-level table formula (``oscillatory_integrals.py:120-145``, and the CuPy path's
    ``_init_gpu_cc_weights``, ``dwba_matrix_elements.py:1316-1347``, for every n): nodes cos(pi j/(n-1))
    from +1 to -1, weights (2/(n-1)) (1 - 2 sum_j cos(2 j theta)/(4 j^2 - 1)), the last term halved
    for odd n."""
    theta = np.pi * np.arange(n) / (n - 1)
    x = np.cos(theta)
    jm = (n - 1) // 2
    if jm > 0:
        jv = np.arange(1, jm + 1)
        sums = np.sum(np.cos(2 * jv[:, None] * theta[None, :]) / (4 * jv ** 2 - 1)[:, None], axis=0)
        if (n - 1) % 2 == 0:
            sums += 0.5 * np.cos(2 * jm * theta) / (4 * jm ** 2 - 1)
    else:
        sums = np.zeros(n)
    return x, (2.0 / (n - 1)) * (1 - 2 * sums)


def cc_reference(n: int):
    """Clenshaw-Curtis nodes/weights on [-1, 1] as ``_get_cc_ref`` (``:159-171``) returns them.

    n = 5 comes from the module-level table of ``oscillatory_integrals.py:120-145``
    (its weights are [1, 9, 11, 9, 1]/15 and sum to 31/15, not 2 -- the reference's
    default quadrature carries this factor and parity keeps it); other n use
    ``clenshaw_curtis_nodes`` (``:1539-1618``). Nodes run from +1 down to -1.
    """
    if n < 2:
        raise ValueError("Clenshaw-Curtis requires n >= 2.")
    if n == 5:
        return cc_table_rule(n)
    return clenshaw_curtis_nodes(n, -1.0, 1.0)


def clenshaw_curtis_nodes(n: int, a: float, b: float):
    """General CC rule on [a, b]; ``oscillatory_integrals.py:1539-1618``."""
    if n < 2:
        raise ValueError("Clenshaw-Curtis requires n >= 2 nodes")
    if n == 2:
        return np.array([b, a]), np.array([0.5, 0.5]) * (b - a)
    theta = np.pi * np.arange(n) / (n - 1)
    x = np.cos(theta)
    big = n - 1
    jm = big // 2
    w = np.ones(n)
    if jm > 0:
        jv = np.arange(1, jm + 1)
        w += np.sum((2.0 / (1 - 4 * jv ** 2))[:, None] * np.cos(2 * jv[:, None] * theta[None, :]), axis=0)
    if big % 2 == 0:
        w += np.cos(big * theta) / (1 - big ** 2)
    w *= 2.0 / big
    w[0] /= 2
    w[-1] /= 2
    return 0.5 * (b - a) * (x + 1) + a, w * (0.5 * (b - a))


def check_phase_sampling(r, k_total, threshold=np.pi / 4, eta_total=0.0):
    """Max phase step on the grid; ``oscillatory_integrals.py:1456-1509``."""
    if k_total < 1e-10:
        return 0.0, True, -1
    r = np.asarray(r, dtype=float)
    dr = np.diff(r)
    if abs(eta_total) > 1e-10:
        r_mid = np.maximum(0.5 * (r[:-1] + r[1:]), 1e-10)
        step = np.abs((k_total + eta_total / r_mid) * dr)
    else:
        step = np.abs(k_total * dr)
    mx = float(np.max(step))
    bad = step > threshold
    if np.any(bad):
        return mx, False, int(np.argmax(bad))
    return mx, True, -1


def adaptive_phase_increment(r, k_total, requested, eta_total=0.0, threshold=np.pi / 4,
                             min_increment=np.pi / 16):
    """Undersampling-aware phase step in [min_increment, threshold];
    ``oscillatory_integrals.py:1716-1755``."""
    d = float(max(min_increment, requested))
    d = min(d, threshold)
    if k_total < 1e-10 or len(r) < 2:
        return d
    mx, ok, _ = check_phase_sampling(r, float(k_total), threshold=float(threshold), eta_total=float(eta_total))
    if ok:
        return d
    scale = float(threshold) / max(float(mx), 1e-12)
    d_eff = d * max(0.25, min(1.0, scale))
    return float(np.clip(d_eff, min_increment, threshold))


def generate_phase_nodes(r_start, r_end, k_total, dphi, eta_total=0.0):
    """Constant-phase breakpoints; ``oscillatory_integrals.py:1625-1713``."""
    if k_total < 1e-10:
        return np.array([r_start, r_end])
    if abs(eta_total) < 1e-10:
        dr = dphi / k_total
        n = int(np.ceil((r_end - r_start) / dr)) + 1
        return np.linspace(r_start, r_end, n)
    nodes = [r_start]
    r = r_start
    while r < r_end:
        phi_p = k_total + eta_total / max(r, 1e-10)
        dr = dphi / abs(phi_p)
        dr = min(dr, (r_end - r_start) / 10)
        dr = max(dr, 1e-6)
        rn = r + dr
        if rn >= r_end:
            rn = r_end
        nodes.append(rn)
        r = rn
        if len(nodes) > 10000:
            break
    return np.array(nodes)


def is_log_spaced_grid(r, rel_tol=5e-3):
    """``oscillatory_integrals.py:237-251``."""
    r = np.asarray(r, dtype=float)
    if r.ndim != 1 or len(r) < 3:
        return False
    if r[0] <= 0.0 or np.any(np.diff(r) <= 0.0):
        return False
    d = np.diff(np.log(r))
    m = float(np.mean(d))
    if not np.isfinite(m) or m <= 0.0:
        return False
    return float(np.max(np.abs(d - m))) <= rel_tol * m


def interp_on_radial_grid(x_new, x, y):
    """Log-r interpolation on log grids, else linear; ``oscillatory_integrals.py:279-302``."""
    x = np.asarray(x, dtype=float)
    xn = np.clip(np.asarray(x_new, dtype=float), x[0], x[-1])
    if is_log_spaced_grid(x):
        xs = np.maximum(x, 1e-300)
        return np.interp(np.log(np.maximum(xn, xs[0])), np.log(xs), y)
    return np.interp(xn, x, y)


def cc_nodes_on_breakpoints(breaks, n_nodes):
    """All CC nodes and weights on valid phase intervals, in the reference's
    order (interval-major, node +1 -> -1); ``oscillatory_integrals.py:2578-2601``."""
    a = breaks[:-1]
    b = breaks[1:]
    m = (b - a) > 1e-12
    a, b = a[m], b[m]
    xr, wr = cc_reference(n_nodes)
    hw = 0.5 * (b - a)
    X = (hw[:, None] * (xr + 1) + a[:, None]).ravel()
    W = (wr * hw[:, None]).ravel()
    return X, W, len(a)
