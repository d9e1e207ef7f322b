"""Sensitivity of the config-1 DCS and TCS to every radial integral (fixture generator).

H 1s->2p at 50 eV (``config1.npz``): the amplitudes f, g of the reference's ``dwba_coupling``
(``calculate_amplitude_contribution``, dwba_coupling.py:285-634) are linear in the radial
integrals, and its DCS (``dcs_dwba``, sigma_total.py:147-177) is the quadratic form
(k_f/k_i) (N_eq/(2L_i+1)) [1/4 |f+g|^2 + 3/4 |f-g|^2] (2 pi)^4, summed over the target M
sublevels. This script evaluates the amplitude of every unit integral once through the
reference, rebuilds the reference DCS from that basis (checked against the stored reference DCS),
and stores the exact gradients dDCS/dI (at 19 angles) and dTCS/dI (TCS through
``integrate_dcs_over_angles``, sigma_total.py:179-217). With them a test on a machine without the
reference turns per-integral errors dI into DCS/TCS errors: dTCS = g . dI + O(|dI|^2).

Runs only where the reference source tree is available (its directory in the environment
variable ``DWBA_REFERENCE_PATH``, which must be set). Usage:  python tests/golden/make_config1_sensitivity.py
"""
from __future__ import annotations

import json
import logging
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("DWBA_REFERENCE_PATH")
if not REF:
    sys.exit("set DWBA_REFERENCE_PATH to the reference source tree (the directory holding dwba_matrix_elements.py)")

import scipy.special as _ss  # noqa: E402

if not hasattr(_ss, "sph_harm"):  # removed in SciPy 1.18; the reference still imports it
    _ss.sph_harm = lambda m, n, phi, theta: _ss.sph_harm_y(n, m, theta, phi)
sys.path.insert(0, REF)
logging.disable(logging.WARNING)

from dwba_coupling import calculate_amplitude_contribution  # noqa: E402
from sigma_total import dcs_dwba, integrate_dcs_over_angles  # noqa: E402

LI, LF = 0, 1  # 1s -> 2p


def basis(theta, pairs, k_i, k_f, nl):
    """F[m, kind, p, L, theta], G[...]: f and g amplitudes of a unit integral (kind 0 direct, 1 exchange)."""
    Ms = [(Mi, Mf) for Mi in range(-LI, LI + 1) for Mf in range(-LF, LF + 1)]
    F = np.zeros((len(Ms), 2, len(pairs), nl, len(theta)), dtype=complex)
    G = np.zeros_like(F)
    zero = {L: 0.0 for L in range(nl)}
    for m, (Mi, Mf) in enumerate(Ms):
        for p, (li, lf) in enumerate(pairs):
            for L in range(nl):
                unit = {l: (1.0 if l == L else 0.0) for l in range(nl)}
                for kind, (dd, ee) in enumerate(((unit, zero), (zero, unit))):
                    a = calculate_amplitude_contribution(theta, dd, ee, li, lf, k_i, k_f, LI, LF, Mi, Mf)
                    F[m, kind, p, L] = a.f_theta
                    G[m, kind, p, L] = a.g_theta
    return F, G


def main():
    z = np.load(os.path.join(HERE, "config1.npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    theta, k_i, k_f = z["theta"], meta["k_i"], meta["k_f"]
    pairs = [tuple(p) for p in meta["pairs"]]
    I = np.stack([z["I_dir"], z["I_exc"]])  # (2, P, nl)
    nl = I.shape[-1]
    F, G = basis(theta, pairs, k_i, k_f, nl)
    f = np.einsum("mkplt,kpl->mt", F, I)
    g = np.einsum("mkplt,kpl->mt", G, I)
    dcs = sum(dcs_dwba(theta, f[m], g[m], k_i, k_f, LI, 1) for m in range(f.shape[0]))
    rel = np.max(np.abs(dcs - z["dcs"]) / np.max(z["dcs"]))
    tcs = integrate_dcs_over_angles(theta, dcs)
    print(f"basis DCS vs reference DCS: max rel {rel:.2e}; TCS {tcs:.12e} vs {float(z['tcs'][0]):.12e}")
    assert rel < 1e-12
    # d/dI of prefac (2pi)^4 [1/4 |f+g|^2 + 3/4 |f-g|^2] summed over m
    pref = (k_f / k_i) * (1.0 / (2 * LI + 1)) * (2.0 * np.pi) ** 4
    s, d = f + g, f - g
    dD = pref * (0.5 * np.real(np.einsum("mt,mkplt->kplt", np.conj(s), F + G)) +
                 1.5 * np.real(np.einsum("mt,mkplt->kplt", np.conj(d), F - G)))
    dT = np.zeros(I.shape)
    for kind in range(2):
        for p in range(len(pairs)):
            for L in range(nl):
                dT[kind, p, L] = integrate_dcs_over_angles(theta, dD[kind, p, L])
    # the quadratic form is exact: a central difference along a random direction reproduces g . v
    rng = np.random.default_rng(5)
    v = rng.normal(size=I.shape) * np.abs(I) * 1e-3
    def tcs_of(Ix):
        fx = np.einsum("mkplt,kpl->mt", F, Ix)
        gx = np.einsum("mkplt,kpl->mt", G, Ix)
        return integrate_dcs_over_angles(theta, sum(dcs_dwba(theta, fx[m], gx[m], k_i, k_f, LI, 1)
                                                    for m in range(fx.shape[0])))
    fd = (tcs_of(I + v) - tcs_of(I - v)) / 2
    print(f"directional check: g.v {np.sum(dT * v):.6e} vs central difference {fd:.6e}")
    assert abs(np.sum(dT * v) - fd) <= 1e-9 * abs(fd)
    sel = np.arange(0, len(theta), 10)  # 0, 10, ..., 180 degrees
    np.savez_compressed(os.path.join(HERE, "config1_sens.npz"), dtcs=dT, ddcs=dD[..., sel].transpose(3, 0, 1, 2),
                        theta_sel=theta[sel], dcs_sel=dcs[sel], tcs=np.array([tcs]))
    print("wrote config1_sens.npz")


if __name__ == "__main__":
    main()
