"""Outer-tail integrals of the direct term, restated in NumPy -- oracle only.

Follows ``oscillatory_integrals.py``: phase closures ``:312-456``,
``dwba_outer_integral_1d`` ``:459-535``, ``compute_outer_integral_oscillatory``
``:1361-1451``, Filon ``:1165-1358``, Levin ``:957-1162`` and
``_analytical_multipole_tail`` ``:2064-2184``. Only the scalar (per-L) path the
CPU ``radial_ME_all_L`` uses is restated here.
"""
from __future__ import annotations

import math
import os

import numpy as np
from scipy.integrate import quad, simpson

_MAX_SEG = max(128, int(os.environ.get("DWBA_MAX_FILON_SEGMENTS", "4096") or 4096))
_MAX_DPHI = max(np.pi / 16, float(os.environ.get("DWBA_MAX_EFFECTIVE_DPHI", str(np.pi / 2)) or np.pi / 2))


def _phase_funcs(k_a, l_a, d_a, e_a, s_a, k_b, l_b, d_b, e_b, s_b):
    """Phases of cos(Phi_a -/+ Phi_b) and derivatives; ``oscillatory_integrals.py:312-456``."""
    km, kp = k_a - k_b, k_a + k_b
    ca = -l_a * np.pi / 2 + s_a + d_a
    cb = -l_b * np.pi / 2 + s_b + d_b
    cm, cp = ca - cb, ca + cb

    def phi(r, sgn):
        v = (km if sgn < 0 else kp) * r + (cm if sgn < 0 else cp)
        if abs(e_a) > 1e-15:
            v += e_a * np.log(2 * k_a * r + 1e-30)
        if abs(e_b) > 1e-15:
            v = v + sgn * e_b * np.log(2 * k_b * r + 1e-30)
        if l_a > 0:
            v -= (l_a * (l_a + 1)) / (2.0 * k_a * r)
        if l_b > 0:
            v = v - sgn * (l_b * (l_b + 1)) / (2.0 * k_b * r)
        return v

    def dphi(r, sgn):
        v = km if sgn < 0 else kp
        if abs(e_a) > 1e-15:
            v += e_a / r
        if abs(e_b) > 1e-15:
            v = v + sgn * e_b / r
        if l_a > 0:
            v += (l_a * (l_a + 1)) / (2.0 * k_a * r ** 2)
        if l_b > 0:
            v = v + sgn * (l_b * (l_b + 1)) / (2.0 * k_b * r ** 2)
        return v

    def d2phi(r, sgn):
        v = 0.0
        if abs(e_a) > 1e-15:
            v -= e_a / (r * r)
        if abs(e_b) > 1e-15:
            v = v - sgn * e_b / (r * r)
        if l_a > 0:
            v -= (l_a * (l_a + 1)) / (k_a * r ** 3)
        if l_b > 0:
            v = v - sgn * (l_b * (l_b + 1)) / (k_b * r ** 3)
        return v

    return phi, dphi, d2phi


def _eval(f, x):
    try:
        v = np.asarray(f(x))
        if v.shape == ():
            v = np.full(x.shape, v)
        return v
    except Exception:
        return np.vectorize(f)(x)


def _filon_segment(f, x, omega, off):
    """``oscillatory_integrals.py:1165-1277``."""
    n = len(x)
    a, b = x[0], x[-1]
    h = b - a
    if n < 2 or h < 1e-15:
        return 0j
    if abs(omega * h) < 1e-3:
        return simpson(f, x=x) * np.exp(1j * (omega * (a + b) / 2 + off))
    if n == 3:
        th = omega * h / 2
        if abs(th) < 0.3:
            t2, t3 = th ** 2, th ** 3
            al = 2 * t3 / 45 * (1 - t2 / 7 + t2 ** 2 / 189)
            be = 2 / 3 + 2 * t2 / 15 - 4 * t2 ** 2 / 105 + 2 * t2 ** 3 / 567
            ga = 4 / 3 - 2 * t2 / 15 + t2 ** 2 / 210 - t2 ** 3 / 11340
        else:
            st, ct = np.sin(th), np.cos(th)
            t2 = th ** 2
            al = (t2 + th * np.sin(2 * th) / 2 - 2 * st ** 2) / th ** 3
            be = 2 * (th * (1 + np.cos(2 * th)) - np.sin(2 * th)) / th ** 3
            ga = 4 * (st - th * ct) / th ** 3
        e0, e1, e2 = (np.exp(1j * (omega * xx + off)) for xx in x)
        return (h / 2) * (al * (-1j / omega) * (f[2] * e2 - f[0] * e0) + be * (f[0] * e0 + f[2] * e2) + ga * f[1] * e1)
    res = 0j
    for i in range(0, n - 2, 2):
        res += _filon_segment(f[i:i + 3], x[i:i + 3], omega, off)
    if n > 2 and (n - 1) % 2 == 1:
        ph = omega * x[-2:] + off
        res += 0.5 * (x[-1] - x[-2]) * (f[-2] * np.exp(1j * ph[0]) + f[-1] * np.exp(1j * ph[1]))
    return res


def _filon(f_func, omega, off, r0, r1, dphi, nseg_nodes=5):
    """``oscillatory_integrals.py:1280-1358``."""
    if abs(omega) < 1e-10:
        re, _ = quad(lambda r: f_func(r) * np.cos(off), r0, r1)
        im, _ = quad(lambda r: f_func(r) * np.sin(off), r0, r1)
        return re + 1j * im
    dr = dphi / abs(omega)
    nraw = max(1, int(np.ceil((r1 - r0) / dr)))
    nseg = min(nraw, _MAX_SEG)
    eff = abs(omega) * (r1 - r0) / max(1, nseg)
    nn = int(nseg_nodes)
    if eff > _MAX_DPHI:
        sc = int(np.ceil(eff / _MAX_DPHI))
        nn = min(15, max(nseg_nodes, nseg_nodes + 2 * (sc - 1)))
    bnd = np.linspace(r0, r1, nseg + 1)
    parts = []
    for i in range(nseg):
        x = np.linspace(bnd[i], bnd[i + 1], nn)
        parts.append(_filon_segment(_eval(f_func, x), x, omega, off))
    parts = np.array(parts)
    return complex(math.fsum(parts.real), math.fsum(parts.imag))


def _cheb_D(n):
    """``oscillatory_integrals.py:970-1021``."""
    th = np.pi * np.arange(n) / (n - 1)
    x = np.cos(th)
    c = np.ones(n)
    c[0] = c[-1] = 2.0
    i, j = np.arange(n)[:, None], np.arange(n)[None, :]
    xd = x[:, None] - x[None, :]
    np.fill_diagonal(xd, 1.0)
    D = (c[:, None] / c[None, :]) * ((-1.0) ** (i + j)) / xd
    np.fill_diagonal(D, 0.0)
    D[np.diag_indices(n)] = -np.sum(D, axis=1)
    return D


def _levin(f_func, phi, dphi_f, r0, r1, n_nodes, nseg):
    """``oscillatory_integrals.py:1024-1162``."""
    bnd = np.linspace(r0, r1, max(1, nseg) + 1)
    parts = []
    xr = np.cos(np.pi * np.arange(n_nodes) / (n_nodes - 1))[::-1]
    for i in range(max(1, nseg)):
        a, b = bnd[i], bnd[i + 1]
        x = 0.5 * (b - a) * (xr + 1) + a
        fv, pv, dpv = _eval(f_func, x), _eval(phi, x), _eval(dphi_f, x)
        h = x[-1] - x[0]
        if h < 1e-15:
            parts.append(0j)
            continue
        A = _cheb_D(n_nodes) * (2.0 / h) + 1j * np.diag(dpv)
        try:
            u = np.linalg.solve(A, fv.astype(complex))
        except np.linalg.LinAlgError:
            u = np.linalg.lstsq(A, fv.astype(complex), rcond=None)[0]
        parts.append(u[-1] * np.exp(1j * pv[-1]) - u[0] * np.exp(1j * pv[0]))
    parts = np.array(parts)
    return complex(math.fsum(parts.real), math.fsum(parts.imag))


def _outer_osc(f_func, phi, dphi_f, d2phi_f, r_m, r_max, delta_phi=np.pi / 4, n_nodes=8, thr=0.1):
    """``compute_outer_integral_oscillatory``, ``oscillatory_integrals.py:1361-1451``."""
    if r_max <= r_m + 1e-10:
        return 0j
    om = abs(dphi_f((r_m + r_max) / 2))
    if om < 1e-10:
        re, _ = quad(lambda r: f_func(r) * np.cos(phi(r)), r_m, r_max)
        im, _ = quad(lambda r: f_func(r) * np.sin(phi(r)), r_m, r_max)
        return re + 1j * im
    h = delta_phi / om
    if abs(d2phi_f((r_m + r_max) / 2)) * h * h < thr:
        return _filon(f_func, om, phi(r_m) - om * r_m, r_m, r_max, delta_phi)
    nseg = max(1, int(np.ceil((r_max - r_m) / h)))
    return _levin(f_func, phi, dphi_f, r_m, r_max, n_nodes, nseg)


def outer_integral_1d(env, k_a, l_a, d_a, e_a, s_a, k_b, l_b, d_b, e_b, s_b, r_m, r_max, delta_phi=np.pi / 4):
    """``dwba_outer_integral_1d``, ``oscillatory_integrals.py:459-535``."""
    if r_max <= r_m + 1e-10:
        return 0.0
    phi, dphi_f, d2phi_f = _phase_funcs(k_a, l_a, d_a, e_a, s_a, k_b, l_b, d_b, e_b, s_b)
    im = _outer_osc(env, lambda r: phi(r, -1), lambda r: dphi_f(r, -1), lambda r: d2phi_f(r, -1),
                    r_m, r_max, delta_phi)
    ip = _outer_osc(env, lambda r: phi(r, +1), lambda r: dphi_f(r, +1), lambda r: d2phi_f(r, +1),
                    r_m, r_max, delta_phi)
    return 0.5 * (im.real - ip.real)


def analytical_multipole_tail(r_m, k_i, k_f, d_i, d_f, l_i, l_f, L, bound_overlap=1.0,
                              eta_i=0.0, eta_f=0.0, sigma_i=0.0, sigma_f=0.0):
    """``_analytical_multipole_tail``, ``oscillatory_integrals.py:2064-2184``."""
    if r_m < 1e-3 or abs(bound_overlap) < 1e-12:
        return 0.0
    lti = eta_i * np.log(2 * k_i * r_m + 1e-30) if abs(eta_i) > 1e-10 else 0.0
    ltf = eta_f * np.log(2 * k_f * r_m + 1e-30) if abs(eta_f) > 1e-10 else 0.0
    ci = -l_i * np.pi / 2 + sigma_i + d_i + lti
    cf = -l_f * np.pi / 2 + sigma_f + d_f + ltf
    kd, ks = k_i - k_f, k_i + k_f
    n = L + 1
    t = 0.0
    pd = kd * r_m + ci - cf
    if abs(kd) > 1e-6:
        t += 0.5 * (np.sin(pd) / (kd * r_m ** n) + n * np.cos(pd) / (kd ** 2 * r_m ** (n + 1)))
    elif n > 1:
        t += 0.5 * np.cos(pd) / ((n - 1) * r_m ** (n - 1))
    ps = ks * r_m + ci + cf
    if ks > 1e-6:
        t -= 0.5 * (np.sin(ps) / (ks * r_m ** n) + n * np.cos(ps) / (ks ** 2 * r_m ** (n + 1)))
    if not np.isfinite(t):
        return 0.0
    return t * bound_overlap
