"""Host-side planning of the radial matrix elements (scalar, O(N) per pair).

These functions decide, per (cont_i, cont_f) pair, the integration limit, the
quadrature branch and the phase-split node set, exactly as the reference's CPU
path does (``dwba_matrix_elements.py:780-1300``); the device then evaluates the
folded bilinear forms. Nothing here touches the GPU.
"""
from __future__ import annotations

import math
import os
from typing import List, NamedTuple, Optional, Sequence, Tuple

import numpy as np

from . import _lib

OVERLAP_TOL = 1e-12  # dwba_matrix_elements.py:1050
PI_4 = np.pi / 4
PI_16 = np.pi / 16


def env_int(name: str, default: int, min_value: int) -> int:
    raw = os.environ.get(name, "").strip()
    try:
        return max(min_value, int(raw)) if raw else max(min_value, int(default))
    except Exception:
        return max(min_value, int(default))


def env_float(name: str, default: float, min_value: float) -> float:
    raw = os.environ.get(name, "").strip()
    try:
        return max(min_value, float(raw)) if raw else max(min_value, float(default))
    except Exception:
        return max(min_value, float(default))


def tail_limits() -> Tuple[int, float]:
    """Filon segment cap and effective-phase cap of the outer tails
    (``oscillatory_integrals.py:75-80``: DWBA_MAX_FILON_SEGMENTS, DWBA_MAX_EFFECTIVE_DPHI)."""
    return env_int("DWBA_MAX_FILON_SEGMENTS", 4096, 128), env_float("DWBA_MAX_EFFECTIVE_DPHI", np.pi / 2, np.pi / 16)


def is_excitation(bound_f) -> bool:
    """``isinstance(bound_f, BoundOrbital)`` (dwba_matrix_elements.py:1124): a ContinuumWave carries chi_of_r."""
    return not hasattr(bound_f, "chi_of_r")


def is_log_spaced(r: np.ndarray, rel_tol: float = 5e-3) -> bool:
    """Log-spacing test of ``oscillatory_integrals.py:237-251``."""
    if r.ndim != 1 or len(r) < 3 or r[0] <= 0.0 or np.any(np.diff(r) <= 0.0):
        return False
    d = np.diff(np.log(r))
    m = float(np.mean(d))
    if not np.isfinite(m) or m <= 0.0:
        return False
    return float(np.max(np.abs(d - m))) <= rel_tol * m


class GridInfo:
    """Per-grid host data reused by every pair of an energy point."""

    def __init__(self, r, w_simpson, w_trapz):
        self.r = np.ascontiguousarray(r, dtype=np.float64)
        self.w = np.ascontiguousarray(w_simpson, dtype=np.float64)
        self.w_trapz = np.ascontiguousarray(w_trapz, dtype=np.float64)
        self.N = len(self.r)
        self.dr = np.diff(self.r)
        # prefix maxima of the step size, for the phase-sampling test at eta = 0
        self.dr_prefix_max = np.maximum.accumulate(self.dr) if self.N > 1 else self.dr
        self.log_full = is_log_spaced(self.r)
        self._log_prefix = {}
        self._extent = {}

    def log_prefix(self, n: int) -> bool:
        v = self._log_prefix.get(n)
        if v is None:
            v = is_log_spaced(self.r[:n])
            self._log_prefix[n] = v
        return v

    def log_prefixes(self, ns: Sequence[int]) -> List[bool]:
        """log_prefix(n) for every n of a list (cached values looked up in bulk)."""
        out = list(map(self._log_prefix.get, ns))
        if None in out:
            out = [self.log_prefix(n) if v is None else v for n, v in zip(ns, out)]
        return out

    def extent99(self, u: np.ndarray) -> int:
        """Index of 99 % cumulative |u|^2 (dwba_matrix_elements.py:949-960); -1 if u is ~0."""
        key = (u.__array_interface__["data"][0], len(u))
        v = self._extent.get(key)
        if v is None:
            usq = u ** 2
            if np.sum(usq) > 1e-30:
                pc = np.cumsum(usq * self.w_trapz)
                pc /= (pc[-1] + 1e-300)
                v = int(np.searchsorted(pc, 0.99))
            else:
                v = -1
            self._extent[key] = v
        return v


def idx_limit(g: GridInfo, U_i, U_f, u_i, u_f, k_i, k_f, l_i, l_f, im_i, im_f, min_grid_fraction=0.10) -> int:
    """Integration limit n1 (``dwba_matrix_elements.py:909-1022``)."""
    N = g.N
    r = g.r
    n1 = N
    if 0 < im_i < N:
        n1 = min(n1, im_i + 1)
    if 0 < im_f < N:
        n1 = min(n1, im_f + 1)
    k_eff = min(k_i, k_f) if min(k_i, k_f) > 0.1 else max(k_i, k_f)
    lmax = max(l_i, l_f)
    if k_eff > 1e-3:
        idx_turn = int(np.searchsorted(r, (lmax + 0.5) / k_eff))
        idx_turn = min(idx_turn, N - 20)
        min_idx = min(max(idx_turn + 20, int(N * min_grid_fraction)), N)
    else:
        min_idx = max(1, int(N * min_grid_fraction))
    if n1 < min_idx:
        n1 = min_idx
    idx99 = max(0, g.extent99(u_i), g.extent99(u_f))
    if idx99 > n1:
        n1 = idx99 + 1
    ke = 0.5 * min(k_i, k_f) ** 2
    if ke > 1e-10:
        cent = lmax * (lmax + 1)

        def veff(i):
            ui = abs(U_i[i])
            uf = abs(U_f[i]) if U_f is not None else 0.0
            return max(ui, uf) + cent / (2.0 * r[i] ** 2)

        if veff(max(0, n1 - 1)) / ke > 0.03:
            for t in range(n1, min(n1 + 500, N)):
                if veff(t) / ke < 0.03:
                    n1 = t + 1
                    break
    return n1


def adaptive_dphi(g: GridInfo, n1: int, k_total: float, requested: float, eta_total: float) -> float:
    """Phase step of ``_adaptive_phase_increment_for_grid`` (oscillatory_integrals.py:1716-1755)
    with the sampling test of ``check_phase_sampling`` (:1456-1509) on r[:n1]."""
    d = float(max(PI_16, requested))
    d = min(d, PI_4)
    if k_total < 1e-10 or n1 < 2:
        return d
    if abs(eta_total) > 1e-10:
        r = g.r[:n1]
        r_mid = np.maximum(0.5 * (r[:-1] + r[1:]), 1e-10)
        mx = float(np.max(np.abs((k_total + eta_total / r_mid) * g.dr[:n1 - 1])))
    else:
        mx = abs(k_total * float(g.dr_prefix_max[n1 - 2]))  # |k dr| is monotone in dr
    if not (mx > PI_4):
        return d
    scale = PI_4 / max(mx, 1e-12)
    d_eff = d * max(0.25, min(1.0, scale))
    return float(min(max(d_eff, PI_16), PI_4))


class NodeSetKey(NamedTuple):
    """Everything a node set's operators depend on (a tuple: cheap to build and hash per set)."""
    grid_id: int
    n1: int
    k_total: float
    dphi: float
    eta_total: float
    n_cc: int


class NodeSetPlan(NamedTuple):
    key: NodeSetKey
    n_breaks: int
    breaks: Optional[np.ndarray]  # None => linspace on the device
    log1: bool
    log2: bool


def plan_nodeset(g: GridInfo, key: NodeSetKey) -> Optional[NodeSetPlan]:
    """Breakpoints of ``generate_phase_nodes`` on [r0, r[n1-1]] (oscillatory_integrals.py:1625-1713).
    Returns None when the reference falls back to weighted dot products (no valid interval)."""
    r0, r1 = float(g.r[0]), float(g.r[key.n1 - 1])
    if key.k_total < 1e-10:
        return None
    if abs(key.eta_total) < 1e-10:
        dr = key.dphi / key.k_total
        n = int(np.ceil((r1 - r0) / dr)) + 1
        if n < 2:
            return None
        step = (r1 - r0) / (n - 1)
        if not (step > 1e-12):
            return None
        return NodeSetPlan(key, n, None, g.log_prefix(key.n1), g.log_full)
    br = _lib.phase_breaks_coulomb(r0, r1, key.k_total, key.dphi, key.eta_total)
    if len(br) < 2 or not np.any(np.diff(br) > 1e-12):
        return None
    return NodeSetPlan(key, len(br), br, g.log_prefix(key.n1), g.log_full)


def cc_reference(n: int) -> Tuple[np.ndarray, np.ndarray]:
    """Clenshaw-Curtis reference nodes (descending, +1..-1) and weights on [-1, 1]:
    the module-level n=5 table (oscillatory_integrals.py:120-145) and
    clenshaw_curtis_nodes(n, -1, 1) (:1539-1618) for other n, as _get_cc_ref selects."""
    if n < 2:
        raise ValueError("Clenshaw-Curtis requires n_nodes >= 2.")
    theta = np.pi * np.arange(n) / (n - 1)
    x = np.cos(theta)
    if n == 5:
        jm = (n - 1) // 2
        jv = np.arange(1, jm + 1)
        sums = np.sum(np.cos(2 * jv[:, None] * theta[None, :]) / (4 * jv ** 2 - 1)[:, None], axis=0)
        if (n - 1) % 2 == 0:
            sums += 0.5 * np.cos(2 * jm * theta) / (4 * jm ** 2 - 1)
        return x, (2.0 / (n - 1)) * (1 - 2 * sums)
    if n == 2:
        return np.array([1.0, -1.0]), np.array([1.0, 1.0])
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
    # clenshaw_curtis_nodes(n, -1, 1) maps nodes by 0.5*(b-a)*(x+1)+a and weights by 0.5*(b-a) = 1
    return 1.0 * (x + 1) + -1.0, w * 1.0


def diag_scale(L_max: int) -> np.ndarray:
    """Diagonal factor of K_L: exp(L log(min(1, 1-1e-12) + 1e-300)) (dwba_matrix_elements.py:1079-1080, :1113-1116)."""
    lr = np.log(np.minimum(1.0, 1.0 - 1e-12) + 1e-300)
    return np.array([1.0 if L == 0 else float(np.exp(L * lr)) for L in range(L_max + 1)])


def multipole_moments(g: GridInfo, u_i, u_f, L_max: int) -> np.ndarray:
    """M_L = sum w r^L u_f u_i over the full grid (dwba_matrix_elements.py:1216)."""
    m = np.zeros(L_max + 1)
    for L in range(1, L_max + 1):
        m[L] = np.sum(g.w * (g.r ** L) * u_f * u_i)
    return m


def safe_float(x) -> float:
    v = float(x)
    return v if math.isfinite(v) else 0.0
