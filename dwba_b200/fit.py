"""Gradient-based fit of model parameters to cross sections (new; extends the reference's
gradient-free potential fit, fit_potential.py:128-269, which matches binding energies with
scipy L-BFGS-B on finite differences).

The radial integrals come from ``RadialIntegrals`` (differentiable, CUDA forward and backward).
The caller supplies ``build_inputs(params) -> dict`` that makes the six radial inputs
(V_core, U_i, u_i, u_f, chi_i, chi_f) from the parameters with torch operations (a parametrised
potential, orbital or wave model; or tangents of upstream solvers), and an objective of the
integrals. ``CrossSection`` turns integrals into the reference's DCS and TCS given the amplitude
of every unit integral (the angular coupling is linear in the integrals):

    f_M(theta) = sum_k F[M, k, theta] I_k,   g_M(theta) = sum_k G[M, k, theta] I_k,
    DCS(theta) = (k_f/k_i) (N_eq/(2L_i+1)) (2 pi)^4 sum_M [1/4 |f_M + g_M|^2 + 3/4 |f_M - g_M|^2]
                 (sigma_total.py:147-177, clipped at 0 as there),
    TCS = 2 pi trapz(sin(theta) DCS, theta)                       (sigma_total.py:179-217).
"""
from __future__ import annotations

from typing import Callable, Dict, List, Tuple

import numpy as np
import torch

from .autograd import RadialIntegrals

__all__ = ["CrossSection", "CouplingCrossSection", "fit_to_cross_section"]


class CrossSection:
    """DCS/TCS as torch functions of the integrals I (P, 2, L_max+1).

    ``F``, ``G``: complex arrays (n_M, 2, P, L_max+1, n_theta) -- the f and g amplitudes of a
    unit direct (index 0) or exchange (index 1) integral, e.g. from the reference's
    ``calculate_amplitude_contribution`` (dwba_coupling.py:285-634) evaluated once per unit integral.
    """

    def __init__(self, theta, F, G, k_i: float, k_f: float, L_i: int = 0, N_equiv: int = 1, device="cuda"):
        self.theta = torch.as_tensor(np.asarray(theta, dtype=np.float64), device=device)
        self.F = torch.as_tensor(np.asarray(F, dtype=np.complex128), device=device)
        self.G = torch.as_tensor(np.asarray(G, dtype=np.complex128), device=device)
        ok = k_i > 0 and k_f > 0
        self.pref = (k_f / k_i) * (float(N_equiv) / float(2 * L_i + 1)) * (2.0 * np.pi) ** 4 if ok else 0.0

    def dcs(self, I: torch.Tensor) -> torch.Tensor:
        Ic = I.to(torch.complex128)
        f = torch.einsum("mkplt,pkl->mt", self.F, Ic)
        g = torch.einsum("mkplt,pkl->mt", self.G, Ic)
        d = 0.25 * (f + g).abs() ** 2 + 0.75 * (f - g).abs() ** 2
        return torch.clamp(self.pref * d.sum(0), min=0.0)

    def tcs(self, I: torch.Tensor) -> torch.Tensor:
        return 2.0 * np.pi * torch.trapezoid(torch.sin(self.theta) * self.dcs(I), self.theta)


class CouplingCrossSection:
    """DCS/TCS as torch functions of the integrals I (P, 2, L_max+1) with the angular coupling of
    ``coupling.CouplingTables`` (the reference's ``calculate_amplitude_contribution``,
    dwba_coupling.py:285-634, and ``dcs_dwba`` / ``integrate_dcs_over_angles``, sigma_total.py:147-217):
    the same values as ``CouplingTables.dcs`` / ``.tcs``, differentiable in I."""

    def __init__(self, tables, device="cuda"):
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=device)  # noqa: E731
        self.cf, self.cg, self.yd, self.ye = t(tables.cf), t(tables.cg), t(tables.yd), t(tables.ye)
        self.theta = t(tables.theta)
        self.pref = float(tables.pref)

    def dcs(self, I: torch.Tensor) -> torch.Tensor:
        Ic = I.to(torch.complex128)
        sd = torch.einsum("apl,pl->ap", self.cf, Ic[:, 0])
        se = torch.einsum("apl,pl->ap", self.cg, Ic[:, 1])
        f = torch.einsum("ap,apt->at", sd, self.yd.to(torch.complex128))
        g = torch.einsum("ap,apt->at", se, self.ye.to(torch.complex128))
        d = self.pref * (0.25 * (f + g).abs() ** 2 + 0.75 * (f - g).abs() ** 2)
        return torch.clamp(d.sum(0), min=0.0)

    def tcs(self, I: torch.Tensor) -> torch.Tensor:
        return 2.0 * np.pi * torch.trapezoid(torch.sin(self.theta) * self.dcs(I), self.theta)


def fit_to_cross_section(model: RadialIntegrals, build_inputs: Callable[[torch.Tensor], Dict[str, torch.Tensor]],
                         objective: Callable[[torch.Tensor], torch.Tensor], params0, max_iter: int = 50,
                         tol: float = 1e-12) -> Tuple[torch.Tensor, List[float]]:
    """Minimise ``objective(model(**build_inputs(params)))`` over ``params`` with L-BFGS
    (strong-Wolfe line search); gradients flow through the CUDA backward of the integrals.
    Returns the fitted parameters and the loss history."""
    params = torch.as_tensor(params0, dtype=torch.float64, device="cuda").clone().requires_grad_(True)
    opt = torch.optim.LBFGS([params], lr=1.0, max_iter=max_iter, tolerance_grad=tol, tolerance_change=tol,
                            history_size=20, line_search_fn="strong_wolfe")
    history: List[float] = []

    def closure():
        opt.zero_grad()
        loss = objective(model(**build_inputs(params)))
        loss.backward()
        history.append(float(loss.detach()))
        return loss

    opt.step(closure)
    return params.detach(), history
