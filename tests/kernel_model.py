"""NumPy model of the device kernels' index arithmetic (test infrastructure).

Mirrors ``dwba_b200/csrc/nodes.cu`` (node positions, interpolation taps, banded
operators) and ``fold.cu`` so the host planning plus the kernel design can be
checked against the golden fixtures on a machine without a GPU. The bilinear
forms are evaluated with the oracle's dense evaluator.
"""
from __future__ import annotations

import numpy as np

from dwba_b200.plan import cc_reference


def node_arrays(r, n1, n_breaks, breaks, n_cc):
    """Node positions/weights in ascending order, as nodes.cu:node_geom."""
    x_ref, w_ref = cc_reference(n_cc)
    n_int = n_breaks - 1
    m = np.repeat(np.arange(n_int), n_cc)
    slot = n_cc - 1 - (np.arange(n_int * n_cc) - m * n_cc)
    if breaks is None:
        start, stop = r[0], r[n1 - 1]
        step = (stop - start) / float(n_int)
        a = m * step + start
        b = np.where(m + 1 == n_int, stop, (m + 1) * step + start)
    else:
        a, b = breaks[m], breaks[m + 1]
    hw = 0.5 * (b - a)
    x = np.clip(hw * (x_ref[slot] + 1.0) + a, a, b)
    w = np.where((b - a) > 1e-12, w_ref[slot] * hw, 0.0)
    return x, w


def _log1p_small(u):
    """Taylor series of log(1 + u) as nodes.cu evaluates it (6 terms for u <= 2^-9, else 12)."""
    p6 = np.zeros_like(u)
    for k in range(6, 0, -1):
        p6 = p6 * u + (1.0 if k % 2 else -1.0) / k
    p12 = np.zeros_like(u)
    for k in range(12, 0, -1):
        p12 = p12 * u + (1.0 if k % 2 else -1.0) / k
    return np.where(u <= 2.0 ** -9, p6, p12) * u


def interp_taps(r, n, log_grid, x):
    j = np.clip(np.searchsorted(r[:n], x, side="right") - 1, 0, n - 2)
    lo = x <= r[0]
    hi = x >= r[n - 1]
    if log_grid:
        # log x - log r_j: the series of log(1 + (x - r_j)/r_j) for steps below 1/64, as the kernel
        xx = np.maximum(x, r[0])
        u = (xx - r[j]) / r[j]
        dl = np.where(u <= 1.0 / 64.0, _log1p_small(np.clip(u, 0.0, 1.0 / 64.0)), np.log(xx) - np.log(r[j]))
        t = dl / (np.log(r[j + 1]) - np.log(r[j]))
    else:
        t = (x - r[j]) / (r[j + 1] - r[j])
    j = np.where(hi, n - 2, np.where(lo, 0, j))
    t = np.where(hi, 1.0, np.where(lo, 0.0, t))
    return j, t


def engine_interp_op(X, x):
    """(j, t) of the interpolation onto the nodes ``X`` with the kernel's tap arithmetic, in the
    form of the oracle's ``_interp_op`` (log taps where the grid passes the log-spacing test)."""
    from oracle.quadrature import is_log_spaced_grid
    x = np.asarray(x, dtype=float)
    return interp_taps(x, len(x), is_log_spaced_grid(x), np.asarray(X, dtype=float))


def bands(r, n1, n_breaks, breaks, n_cc, log1, log2):
    """(ta, bx) banded operators of one node set, as nodes.cu:bands_kernel."""
    N = len(r)
    x, w = node_arrays(r, n1, n_breaks, breaks, n_cc)
    j1, t1 = interp_taps(r, n1, log1, x)
    j2, t2 = interp_taps(r, N, log2, x)
    ir = np.clip(np.searchsorted(r, x, side="left"), 1, N - 1)
    il = ir - 1
    wr = (x - r[il]) / (r[ir] - r[il] + 1e-30)
    ta = np.zeros((n1, 3))
    np.add.at(ta[:, 1], j1, w * (1 - t1) ** 2)
    np.add.at(ta[:, 2], j1, w * (1 - t1) * t1)
    np.add.at(ta[:, 1], j1 + 1, w * t1 * t1)
    np.add.at(ta[:, 0], j1 + 1, w * t1 * (1 - t1))
    bx = np.zeros((N, 5))
    for row, q in ((il, 1 - wr), (il + 1, wr)):
        d0 = j2 - row
        assert np.all(d0 >= -2) and np.all(d0 + 1 <= 2)
        np.add.at(bx, (row, d0 + 2), q * w * (1 - t2))
        np.add.at(bx, (row, d0 + 3), q * w * t2)
    return ta.ravel(), bx.ravel()


def fold(op, h, f, g, n_out, n_src, n_clear):
    out = np.zeros(n_clear)
    prod = f * g
    for d in range(-h, h + 1):
        i = np.arange(n_out)
        k = i + d
        ok = (k >= 0) & (k < n_src)
        out[i[ok]] += op[(2 * h + 1) * i[ok] + d + h] * prod[k[ok]]
    return out
