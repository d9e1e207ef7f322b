"""Angular coupling of the radial integrals into scattering amplitudes, DCS and TCS.

The reference builds, per (l_i, l_f) partial-wave channel and target sublevels (M_i, M_f), the
direct and exchange amplitudes (``calculate_amplitude_contribution``, dwba_coupling.py:285-505,
the article's Eq. 412 and 448) and turns their sum into the DCS (``dcs_dwba``,
sigma_total.py:147-177) and the TCS (``integrate_dcs_over_angles``, sigma_total.py:179-217).

Both amplitudes are linear in the integrals and their angular dependence is one spherical
harmonic of l_f at phi = 0 (real):

    f_{M}(theta) = Y_{l_f, -mu_d}(theta, 0) * sum_L cf[L] I_L^dir,   mu_d = M_f - M_i,
    g_{M}(theta) = (-1)^mu_e Y_{l_f, -mu_e}(theta, 0) * sum_L cg[L] I_L^exc,   mu_e = M_i - M_f,

so this module computes the complex scalars cf, cg once per (channel, M_i, M_f) on the host
(Wigner 3j/6j by Racah's single-sum formulas over log-factorials; Clebsch-Gordan and Racah W in
the reference's phase conventions, dwba_coupling.py:154-283; the same 1e-9 cut-offs on the
coupling factors) and the Y table once per angle grid; the CUDA kernel ``dwba_cross_sections``
(csrc/dcs.cu) contracts them with the integrals of all channels and forms the DCS and TCS.
"""
from __future__ import annotations

import math
from functools import lru_cache
from typing import Sequence, Tuple

import numpy as np

__all__ = ["clebsch_gordan", "racah_w", "wigner_3j", "wigner_6j", "channel_coefficients", "CouplingTables"]


@lru_cache(maxsize=None)
def _lf(n: int) -> float:
    """log(n!) (n >= 0)."""
    return math.lgamma(n + 1.0)


def _tri(a: int, b: int, c: int) -> float:
    """log of the triangle coefficient Delta(abc) = (a+b-c)!(a-b+c)!(-a+b+c)!/(a+b+c+1)!."""
    return _lf(a + b - c) + _lf(a - b + c) + _lf(-a + b + c) - _lf(a + b + c + 1)


@lru_cache(maxsize=None)
def wigner_3j(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """(j1 j2 j3; m1 m2 m3) for integer arguments (Racah's formula)."""
    if m1 + m2 + m3 != 0 or not (abs(j1 - j2) <= j3 <= j1 + j2):
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    t0 = max(0, j2 - m1 - j3, j1 + m2 - j3)
    t1 = min(j1 + j2 - j3, j1 - m1, j2 + m2)
    if t0 > t1:
        return 0.0
    pref = 0.5 * (_tri(j1, j2, j3) + _lf(j1 + m1) + _lf(j1 - m1) + _lf(j2 + m2) + _lf(j2 - m2) +
                  _lf(j3 + m3) + _lf(j3 - m3))
    s = 0.0
    for t in range(t0, t1 + 1):
        den = (_lf(t) + _lf(t - (j2 - m1 - j3)) + _lf(t - (j1 + m2 - j3)) + _lf(j1 + j2 - j3 - t) +
               _lf(j1 - m1 - t) + _lf(j2 + m2 - t))
        s += (-1.0) ** t * math.exp(pref - den)
    return (-1.0) ** (j1 - j2 - m3) * s


def clebsch_gordan(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """<j1 m1; j2 m2 | j3 m3> = (-1)^(j1-j2+m3) sqrt(2 j3 + 1) (j1 j2 j3; m1 m2 -m3)."""
    return (-1.0) ** (j1 - j2 + m3) * math.sqrt(2 * j3 + 1) * wigner_3j(j1, j2, j3, m1, m2, -m3)


@lru_cache(maxsize=None)
def wigner_6j(j1: int, j2: int, j3: int, j4: int, j5: int, j6: int) -> float:
    """{j1 j2 j3; j4 j5 j6} for integer arguments (Racah's formula)."""
    def ok(a, b, c):
        return abs(a - b) <= c <= a + b
    if not (ok(j1, j2, j3) and ok(j1, j5, j6) and ok(j4, j2, j6) and ok(j4, j5, j3)):
        return 0.0
    a1, a2, a3, a4 = j1 + j2 + j3, j1 + j5 + j6, j4 + j2 + j6, j4 + j5 + j3
    b1, b2, b3 = j1 + j2 + j4 + j5, j2 + j3 + j5 + j6, j3 + j1 + j6 + j4
    t0, t1 = max(a1, a2, a3, a4), min(b1, b2, b3)
    if t0 > t1:
        return 0.0
    tri = _tri(j1, j2, j3) + _tri(j1, j5, j6) + _tri(j4, j2, j6) + _tri(j4, j5, j3)
    s = 0.0
    for t in range(t0, t1 + 1):
        den = _lf(t - a1) + _lf(t - a2) + _lf(t - a3) + _lf(t - a4) + _lf(b1 - t) + _lf(b2 - t) + _lf(b3 - t)
        s += (-1.0) ** t * math.exp(_lf(t + 1) - den)
    return math.exp(0.5 * tri) * s


def racah_w(l1: int, l2: int, l3: int, l4: int, l5: int, l6: int) -> float:
    """W(l1 l2 l3 l4; l5 l6) = (-1)^(l1+l2+l3+l4) {l1 l2 l5; l4 l3 l6}."""
    return (-1.0) ** (l1 + l2 + l3 + l4) * wigner_6j(l1, l2, l5, l4, l3, l6)


@lru_cache(maxsize=None)
def channel_coefficients(l_i: int, l_f: int, L_max: int, Li: int, Lf: int, Mi: int, Mf: int,
                         ) -> Tuple[np.ndarray, np.ndarray]:
    """(cf, cg): complex per-multipole coefficients of the direct and exchange amplitudes of one
    channel and sublevel pair, without the 2/(pi k_i k_f) prefactor and the Y_lf(theta) factor
    (dwba_coupling.py:337-505)."""
    mu_d, mu_e = Mf - Mi, Mi - Mf
    cf = np.zeros(L_max + 1, dtype=complex)
    cg = np.zeros(L_max + 1, dtype=complex)
    if abs(mu_d) > l_f and abs(mu_e) > l_f:
        return cf, cg
    y_li = math.sqrt((2 * l_i + 1) / (4 * math.pi))
    e_li, e_Li, e_lf, e_Lf = (math.sqrt(2 * x + 1) for x in (l_i, Li, l_f, Lf))
    ph_f = 1j ** (l_i + l_f)
    ph_g = 1j ** (l_i - l_f) * (-1.0) ** (Lf + Mf)
    for lT in range(L_max + 1):
        e_lT = math.sqrt(2 * lT + 1)
        # direct (Eq. 412)
        c1 = clebsch_gordan(l_f, l_i, lT, 0, 0, 0)
        c2 = clebsch_gordan(lT, Li, Lf, 0, 0, 0) if abs(c1) >= 1e-9 else 0.0
        if abs(c1) >= 1e-9 and abs(c2) >= 1e-9:
            s = 0.0
            for gg in range(max(abs(l_i - Li), abs(l_f - Lf)), min(l_i + Li, l_f + Lf) + 1):
                w = racah_w(l_f, l_i, Lf, Li, lT, gg)
                if abs(w) < 1e-9:
                    continue
                s += w * clebsch_gordan(l_i, Li, gg, 0, Mi, Mi) * clebsch_gordan(l_f, Lf, gg, mu_d, -Mf, -Mi)
            cf[lT] = ph_f * y_li * (e_lf * e_li * e_Li / e_lT) * c1 * c2 * s
        # exchange (Eq. 448)
        c1 = clebsch_gordan(Lf, l_i, lT, 0, 0, 0)
        c2 = clebsch_gordan(lT, Li, l_f, 0, 0, 0)
        if abs(c1 * c2) >= 1e-9:
            s = 0.0
            for gg in range(max(abs(l_i - Li), abs(Lf - l_f)), min(l_i + Li, Lf + l_f) + 1):
                w = racah_w(Lf, l_i, l_f, Li, lT, gg)
                s += w * clebsch_gordan(l_i, Li, gg, 0, Mi, Mi) * clebsch_gordan(Lf, l_f, gg, -Mf, -mu_e, -Mi)
            cg[lT] = ph_g * y_li * (e_Lf * e_li * e_Li / e_lT) * c1 * c2 * s
    return cf, cg


def _ylm_real(l: int, m: int, theta: np.ndarray) -> np.ndarray:
    """Y_lm(theta, phi = 0) with the Condon-Shortley phase (real at phi = 0)."""
    from scipy.special import sph_harm_y
    if abs(m) > l:
        return np.zeros_like(theta)
    return np.real(sph_harm_y(l, m, theta, 0.0))


class CouplingTables:
    """Host tables for a set of channels (l_i, l_f) of one transition (target L_i -> L_f):

    ``cf``, ``cg``: (n_M, P, L_max+1) complex128, with 2/(pi k_i k_f) folded in;
    ``yd``, ``ye``: (n_M, P, n_theta) float64, Y_{l_f,-mu_d}(theta) and (-1)^mu_e Y_{l_f,-mu_e}(theta);
    ``pref``: the DCS prefactor (k_f/k_i) N_eq/(2 L_i + 1) (2 pi)^4 (0 unless k_i, k_f > 0).
    """

    def __init__(self, theta: Sequence[float], channels: Sequence[Tuple[int, int]], L_max: int, k_i: float,
                 k_f: float, Li: int, Lf: int, N_equiv: int = 1):
        self.theta = np.asarray(theta, dtype=np.float64)
        self.channels = [(int(a), int(b)) for a, b in channels]
        self.L_max = int(L_max)
        Ms = [(Mi, Mf) for Mi in range(-Li, Li + 1) for Mf in range(-Lf, Lf + 1)]
        self.Ms = Ms
        P, nl, nt = len(self.channels), self.L_max + 1, len(self.theta)
        scale = (2.0 / math.pi) / (k_i * k_f)
        self.cf = np.zeros((len(Ms), P, nl), dtype=complex)
        self.cg = np.zeros((len(Ms), P, nl), dtype=complex)
        self.yd = np.zeros((len(Ms), P, nt))
        self.ye = np.zeros((len(Ms), P, nt))
        ycache = {}

        def Y(l, m):
            key = (l, m)
            if key not in ycache:
                ycache[key] = _ylm_real(l, m, self.theta)
            return ycache[key]
        for a, (Mi, Mf) in enumerate(Ms):
            mu_d, mu_e = Mf - Mi, Mi - Mf
            for p, (li, lf) in enumerate(self.channels):
                cf, cg = channel_coefficients(li, lf, self.L_max, Li, Lf, Mi, Mf)
                self.cf[a, p] = scale * cf
                self.cg[a, p] = scale * cg
                self.yd[a, p] = Y(lf, -mu_d)
                self.ye[a, p] = (-1.0) ** mu_e * Y(lf, -mu_e)
        ok = k_i > 0.0 and k_f > 0.0
        self.pref = (k_f / k_i) * (float(N_equiv) / float(2 * Li + 1)) * (2.0 * math.pi) ** 4 if ok else 0.0

    def amplitudes(self, I_dir: np.ndarray, I_exc: np.ndarray):
        """Host evaluation: f, g of shape (n_M, n_theta) from I (P, L_max+1)."""
        sd = np.einsum("apl,pl->ap", self.cf, I_dir)
        se = np.einsum("apl,pl->ap", self.cg, I_exc)
        return np.einsum("ap,apt->at", sd, self.yd), np.einsum("ap,apt->at", se, self.ye)

    def dcs(self, I_dir: np.ndarray, I_exc: np.ndarray) -> np.ndarray:
        f, g = self.amplitudes(I_dir, I_exc)
        d = self.pref * (0.25 * np.abs(f + g) ** 2 + 0.75 * np.abs(f - g) ** 2)
        return np.clip(np.sum(d, axis=0), 0.0, None)

    def tcs(self, I_dir: np.ndarray, I_exc: np.ndarray) -> float:
        d = self.dcs(I_dir, I_exc)
        return float(2.0 * math.pi * np.trapezoid(np.sin(self.theta) * d, self.theta))

    def cross_sections_gpu(self, I_dir, I_exc):
        """DCS (n_theta) and TCS on the device (``dwba_cross_sections``): I_dir, I_exc are (P, L_max+1)
        float64 arrays or CUDA tensors. Returns torch tensors (dcs, tcs[1])."""
        import torch
        from . import _lib
        dev = torch.device("cuda", torch.cuda.current_device())
        if not hasattr(self, "_dev"):
            as_t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)  # noqa: E731
            self._dev = dict(cf=as_t(self.cf.view(np.float64)), cg=as_t(self.cg.view(np.float64)), yd=as_t(self.yd),
                             ye=as_t(self.ye), theta=as_t(self.theta))
        d = self._dev
        Id = torch.as_tensor(I_dir, dtype=torch.float64, device=dev).contiguous()
        Ie = torch.as_tensor(I_exc, dtype=torch.float64, device=dev).contiguous()
        nM, P, nl = self.cf.shape
        if tuple(Id.shape) != (P, nl) or tuple(Ie.shape) != (P, nl):
            raise ValueError(f"integrals must have shape {(P, nl)}")
        dcs = torch.empty(len(self.theta), dtype=torch.float64, device=dev)
        tcs = torch.empty(1, dtype=torch.float64, device=dev)
        _lib.check(_lib.load().dwba_cross_sections(
            d["cf"].data_ptr(), d["cg"].data_ptr(), d["yd"].data_ptr(), d["ye"].data_ptr(), Id.data_ptr(),
            Ie.data_ptr(), d["theta"].data_ptr(), nM, P, nl, len(self.theta), self.pref, dcs.data_ptr(),
            tcs.data_ptr(), torch.cuda.current_stream().cuda_stream), "dwba_cross_sections")
        return dcs, tcs
