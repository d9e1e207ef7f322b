"""Parametric single-active-electron (SAE) model: the inputs of the radial integrals as smooth
functions of the core-potential parameters, for gradient fits of those parameters to cross sections.

The reference fits its SAE core potential (``potential_core.py:143-200``,
V(r) = -(Zc + a1 e^{-a2 r} + a3 r e^{-a4 r} + a5 e^{-a6 r}) / r) to binding energies without
gradients (``fit_potential.py:128-269``). Here the path from the parameters to a cross section is
differentiable end to end: the hot path (radial integrals, amplitudes, DCS/TCS) has exact CUDA
backward kernels, and the upstream solvers below are differentiated by central differences on
the host (tangents d(input)/d(parameter)), which are contracted with the backward's gradients.

The solvers are this module's own, kept smooth in the parameters (no adaptive steps, fixed grids,
fixed matching radius); they stand in for the reference's ``bound_states.py``, ``distorting_potential.py``
and ``continuum.py`` with the same definitions, not the same numerics:
* bound states: -u''/2 + (V + l(l+1)/2r^2) u = E u in x = ln r (u = e^{x/2} y), second-order finite
  differences on the uniform x grid, a symmetric tridiagonal eigenproblem (``eigh_tridiagonal``);
* static distorting potentials U_j = V_core + V_H[u_j] (``distorting_potential.py:447-530``);
* continuum waves: Numerov in x = ln r, matched at the grid's end to Riccati-Bessel functions,
  normalised to sin(kr - l pi/2 + delta) (neutral asymptotics, z = 0).
The excitation energy (hence k_f) is held at the value of the reference parameters, as when
fitting at a measured threshold.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

HARTREE_EV = 27.211386245988


def core_potential(r: np.ndarray, Zc: float, a: Sequence[float]) -> np.ndarray:
    """V(r) = -(Zc + a1 e^{-a2 r} + a3 r e^{-a4 r} + a5 e^{-a6 r}) / r (``potential_core.py:143-200``)."""
    a1, a2, a3, a4, a5, a6 = (float(v) for v in a)
    return -(Zc + a1 * np.exp(-a2 * r) + a3 * r * np.exp(-a4 * r) + a5 * np.exp(-a6 * r)) / r


def _log_step(r: np.ndarray) -> float:
    x = np.log(r)
    h = (x[-1] - x[0]) / (len(r) - 1)
    if not np.allclose(np.diff(x), h, rtol=1e-6, atol=0.0):
        raise ValueError("the SAE solvers need an exponential grid (uniform in ln r)")
    return float(h)


def bound_state(r: np.ndarray, w_trapz: np.ndarray, V: np.ndarray, l: int, n_index: int) -> Tuple[float, np.ndarray]:
    """Energy and radial function u (sum w u^2 = 1) of the n_index-th lowest state of angular momentum l.
    Sign: the outer part (weight r) positive."""
    from scipy.linalg import eigh_tridiagonal
    h = _log_step(r)
    q = (l + 0.5) ** 2 + 2.0 * r * r * V
    b = 2.0 * r * r
    diag = (2.0 / (h * h) + q) / b
    off = (-1.0 / (h * h)) / np.sqrt(b[:-1] * b[1:])
    k = int(n_index) - 1
    # the matrix is graded (entries ~1/(h r)^2 near the origin): bisection to a tiny absolute tolerance
    # keeps the small eigenvalues to full relative accuracy (the default tolerance scales with its norm)
    E, z = eigh_tridiagonal(diag, off, select="i", select_range=(k, k), tol=1e-300)
    y = z[:, 0] / np.sqrt(b)
    u = np.sqrt(r) * y
    u /= np.sqrt(np.sum(w_trapz * u * u))
    if np.sum(w_trapz * u * r) < 0.0:
        u = -u
    return float(E[0]), u


def hartree_potential(r: np.ndarray, u: np.ndarray) -> np.ndarray:
    """V_H(r) = (1/r) int_0^r u^2 + int_r^inf u^2 / r' (trapezoid cumulative sums)."""
    rho = u * u
    dr = np.diff(r)
    inner = np.concatenate([[0.0], np.cumsum(0.5 * (rho[1:] + rho[:-1]) * dr)])
    f = rho / r
    outer_rev = np.concatenate([[0.0], np.cumsum((0.5 * (f[1:] + f[:-1]) * dr)[::-1])])[::-1]
    return inner / r + outer_rev


def continuum_waves(r: np.ndarray, U: np.ndarray, ls: Sequence[int], k: float) -> Tuple[np.ndarray, np.ndarray]:
    """chi_l (rows, one per l in ``ls``) normalised to sin(kr - l pi/2 + delta_l) and delta_l, by Numerov in
    x = ln r (y'' = [(l+1/2)^2 + 2 r^2 (U - k^2/2)] y, u = e^{x/2} y) from the first grid point outwards,
    matched to Riccati-Bessel functions at the last two points a quarter wavelength apart."""
    from scipy.special import spherical_jn, spherical_yn
    h = _log_step(r)
    ls = np.asarray(ls, dtype=np.int64)
    E = 0.5 * k * k
    g = (ls[:, None] + 0.5) ** 2 + 2.0 * (r * r * (U - E))[None, :]
    c = 1.0 - (h * h / 12.0) * g
    n = len(r)
    y = np.zeros((len(ls), n))
    # start in the centrifugal region: y ~ r^(l+1/2), two points
    y[:, 0] = (r[0] / r[1]) ** (ls + 0.5)
    y[:, 1] = 1.0
    scale = np.zeros(len(ls))
    for i in range(1, n - 1):
        y[:, i + 1] = ((12.0 - 10.0 * c[:, i]) * y[:, i] - c[:, i - 1] * y[:, i - 1]) / c[:, i + 1]
        big = np.abs(y[:, i + 1]) > 1e100  # keep the recurrence in range (a common factor per wave)
        if big.any():
            y[big, : i + 2] *= 1e-100
            scale[big] += 100.0
    u = np.sqrt(r)[None, :] * y
    i2 = n - 1
    i1 = int(np.searchsorted(r, r[-1] - 0.5 * np.pi / k))
    i1 = min(max(i1, 1), n - 2)
    chi = np.empty_like(u)
    delta = np.empty(len(ls))
    for j, l in enumerate(ls):
        x1, x2 = k * r[i1], k * r[i2]
        jh = np.array([x1 * spherical_jn(l, x1), x2 * spherical_jn(l, x2)])
        nh = np.array([x1 * spherical_yn(l, x1), x2 * spherical_yn(l, x2)])
        # u = A cos(delta) jh - A sin(delta) nh at both points
        M = np.array([[jh[0], -nh[0]], [jh[1], -nh[1]]])
        ac, as_ = np.linalg.solve(M, np.array([u[j, i1], u[j, i2]]))
        A = np.hypot(ac, as_)
        chi[j] = u[j] / A
        delta[j] = np.arctan2(as_, ac)
    return chi, delta


@dataclass
class Transition:
    """An excitation (l_i, n_index_i) -> (l_f, n_index_f) at incident energy E (eV) with partial waves
    l <= l_max and (l_i + l_f) of the parity the dipole-like multipoles couple."""
    l_i: int = 0
    n_index_i: int = 3
    l_f: int = 1
    n_index_f: int = 2
    E_eV: float = 20.0
    l_max: int = 25
    L_max: int = 4
    Zc: float = 1.0


@dataclass
class SAEInputs:
    V: np.ndarray
    U_i: np.ndarray
    U_f: np.ndarray
    u_i: np.ndarray
    u_f: np.ndarray
    chi_i: np.ndarray   # (n_waves_i, N), rows for l = 0..l_max
    chi_f: np.ndarray
    delta_i: np.ndarray
    delta_f: np.ndarray
    E_i: float = 0.0
    E_f: float = 0.0


@dataclass
class SAEProblem:
    """The radial-integral inputs of one excitation as functions of the free parameters p of the core
    potential, with ``full_params(p)`` mapping them onto (a1..a6). ``k_i`` follows from E; ``k_f`` is
    fixed at the excitation energy of the reference parameters ``p_ref``."""
    grid: object
    transition: Transition
    p_ref: np.ndarray
    full_params: object = None
    k_i: float = 0.0
    k_f: float = 0.0
    pairs_l: List[Tuple[int, int]] = field(default_factory=list)

    def __post_init__(self):
        self.p_ref = np.asarray(self.p_ref, dtype=np.float64)
        if self.full_params is None:
            self.full_params = lambda p: np.asarray(p, dtype=np.float64)
        t = self.transition
        base = self._bound(self.p_ref)
        dE = (base[2] - base[0]) * HARTREE_EV
        self.k_i = float(np.sqrt(2.0 * t.E_eV / HARTREE_EV))
        self.k_f = float(np.sqrt(2.0 * (t.E_eV - dE) / HARTREE_EV))
        par = (t.l_i + t.l_f) % 2
        self.pairs_l = [(a, b) for a in range(t.l_max + 1) for b in range(t.l_max + 1) if (a + b) % 2 == par]

    def _bound(self, p):
        g, t = self.grid, self.transition
        V = core_potential(g.r, t.Zc, self.full_params(p))
        E_i, u_i = bound_state(g.r, g.w_trapz, V, t.l_i, t.n_index_i)
        E_f, u_f = bound_state(g.r, g.w_trapz, V, t.l_f, t.n_index_f)
        return E_i, u_i, E_f, u_f, V

    def inputs(self, p) -> SAEInputs:
        g, t = self.grid, self.transition
        E_i, u_i, E_f, u_f, V = self._bound(np.asarray(p, dtype=np.float64))
        U_i = V + hartree_potential(g.r, u_i)
        U_f = V + hartree_potential(g.r, u_f)
        ls = np.arange(t.l_max + 1)
        chi_i, d_i = continuum_waves(g.r, U_i, ls, self.k_i)
        chi_f, d_f = continuum_waves(g.r, U_f, ls, self.k_f)
        return SAEInputs(V, U_i, U_f, u_i, u_f, chi_i, chi_f, d_i, d_f, E_i, E_f)

    def tangents(self, p, rel_step: float = 1e-6) -> Tuple[List[SAEInputs], List[SAEInputs], np.ndarray]:
        """Inputs at p + h_k e_k and p - h_k e_k (h_k = rel_step |p_k|), and the steps."""
        p = np.asarray(p, dtype=np.float64)
        hs = rel_step * np.maximum(np.abs(p), 1e-3)
        plus, minus = [], []
        for k in range(len(p)):
            e = np.zeros_like(p)
            e[k] = hs[k]
            plus.append(self.inputs(p + e))
            minus.append(self.inputs(p - e))
        return plus, minus, hs

    def wave_objects(self, x: SAEInputs):
        """Bound-orbital and continuum-wave objects (the reference's attribute names) for the engine."""
        from types import SimpleNamespace as NS
        t = self.transition
        bi = NS(l=t.l_i, energy_au=x.E_i, u_of_r=x.u_i, n_index=t.n_index_i)
        bf = NS(l=t.l_f, energy_au=x.E_f, u_of_r=x.u_f, n_index=t.n_index_f)
        wi = [NS(l=l, k_au=self.k_i, chi_of_r=x.chi_i[l], phase_shift=float(x.delta_i[l]), idx_match=-1, eta=0.0,
                 sigma_l=0.0) for l in range(t.l_max + 1)]
        wf = [NS(l=l, k_au=self.k_f, chi_of_r=x.chi_f[l], phase_shift=float(x.delta_f[l]), idx_match=-1, eta=0.0,
                 sigma_l=0.0) for l in range(t.l_max + 1)]
        return bi, bf, [(wi[a], wf[b]) for a, b in self.pairs_l]

    def torch_inputs(self, x: SAEInputs, device="cuda") -> Dict[str, "object"]:
        """The six arguments of ``RadialIntegrals`` (float64 tensors on ``device``)."""
        import torch
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)  # noqa: E731
        ia = np.array([a for a, _ in self.pairs_l])
        fb = np.array([b for _, b in self.pairs_l])
        return dict(V_core=t(x.V), U_i=t(x.U_i), u_i=t(x.u_i), u_f=t(x.u_f), chi_i=t(x.chi_i[ia]), chi_f=t(x.chi_f[fb]))


# ----------------------------------------------------------------------------- gradients and fits
def value_and_grad(problem: SAEProblem, model, objective, p, rel_step: float = 1e-6, with_fd: bool = False):
    """objective(model(inputs(p))) and its gradient in the parameters p: the CUDA backward gives the
    gradient in the six radial inputs, which is contracted with the central-difference tangents of
    the solvers (h_k = rel_step |p_k|). With ``with_fd`` also the central differences of the objective
    itself from the same perturbed inputs (the check of the chain). Returns (value, grad[, fd])."""
    import torch
    p = np.asarray(p, dtype=np.float64)
    x0 = problem.inputs(p)
    xs = {k: v.requires_grad_(True) for k, v in problem.torch_inputs(x0).items()}
    val = objective(model(**xs))
    val.backward()
    g_in = {k: v.grad.detach() for k, v in xs.items()}
    plus, minus, hs = problem.tangents(p, rel_step)
    grad = np.zeros(len(p))
    fd = np.zeros(len(p))
    for k in range(len(p)):
        tp, tm = problem.torch_inputs(plus[k]), problem.torch_inputs(minus[k])
        grad[k] = float(sum(((tp[n] - tm[n]) * g_in[n]).sum() for n in g_in)) / (2.0 * hs[k])
        if with_fd:
            with torch.no_grad():
                fd[k] = (float(objective(model(**tp))) - float(objective(model(**tm)))) / (2.0 * hs[k])
    return (float(val.detach()), grad, fd) if with_fd else (float(val.detach()), grad)


def fit_parameters(problem: SAEProblem, model, objective, p0, bounds=None, max_iter: int = 60, rel_step: float = 1e-6):
    """Minimise objective(model(inputs(p))) over the core-potential parameters with L-BFGS-B on the
    gradients of ``value_and_grad`` (the reference's potential fit, fit_potential.py:128-269, with a
    cross-section objective and exact gradients through the hot path). Returns (p, history)."""
    from scipy.optimize import minimize
    history: List[float] = []

    def fun(p):
        v, g = value_and_grad(problem, model, objective, p, rel_step)
        history.append(v)
        return v, g
    res = minimize(fun, np.asarray(p0, dtype=np.float64), jac=True, method="L-BFGS-B", bounds=bounds,
                   options=dict(maxiter=max_iter, ftol=1e-15, gtol=1e-14))
    return res.x, history
