"""Host angular coupling against the reference: Wigner/Clebsch-Gordan/Racah identities and the
reference's own config-1 DCS (181 angles) and TCS from its own integrals (tests/golden/config1.npz,
made by running the reference's calculate_amplitude_contribution, dcs_dwba and
integrate_dcs_over_angles)."""
import json
import math
import os

import numpy as np

import golden_cases as gc
from dwba_b200.coupling import CouplingTables, clebsch_gordan, racah_w, wigner_3j, wigner_6j


def test_known_values_and_orthogonality():
    assert abs(clebsch_gordan(1, 1, 2, 0, 0, 0) - math.sqrt(2.0 / 3.0)) < 1e-15
    assert abs(clebsch_gordan(1, 1, 0, 1, -1, 0) - math.sqrt(1.0 / 3.0)) < 1e-15
    assert abs(wigner_3j(1, 1, 0, 0, 0, 0) + 1.0 / math.sqrt(3.0)) < 1e-15
    assert abs(wigner_6j(1, 1, 1, 1, 1, 1) - 1.0 / 6.0) < 1e-15
    # sum_{m1,m2} <j1 m1 j2 m2|J M><j1 m1 j2 m2|J' M> = delta_JJ'
    j1, j2 = 3, 2
    for J in range(1, 6):
        for Jp in range(1, 6):
            s = sum(clebsch_gordan(j1, j2, J, m1, 1 - m1, 1) * clebsch_gordan(j1, j2, Jp, m1, 1 - m1, 1)
                    for m1 in range(-j1, j1 + 1) if abs(1 - m1) <= j2)
            assert abs(s - (1.0 if J == Jp else 0.0)) < 1e-13
    # 6j orthogonality: sum_x (2x+1)(2c+1) {a b x; d e c}{a b x; d e c'} = delta_cc'
    a, b, d, e = 2, 3, 2, 3
    for c in range(0, 5):
        for cp in range(0, 5):
            s = sum((2 * x + 1) * (2 * c + 1) * wigner_6j(a, b, x, d, e, c) * wigner_6j(a, b, x, d, e, cp)
                    for x in range(0, 6))
            want = 1.0 if (c == cp and abs(a - e) <= c <= a + e and abs(d - b) <= c <= d + b) else 0.0
            assert abs(s - want) < 1e-12
    assert racah_w(1, 2, 1, 2, 1, 2) == (-1.0) ** 6 * wigner_6j(1, 2, 1, 2, 1, 2)


def test_config1_dcs_and_tcs_match_reference():
    z = np.load(os.path.join(gc.GOLDEN_DIR, "config1.npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    tab = CouplingTables(z["theta"], [tuple(p) for p in meta["pairs"]], meta["L_max"], meta["k_i"], meta["k_f"], 0, 1)
    dcs = tab.dcs(z["I_dir"], z["I_exc"])
    assert np.max(np.abs(dcs - z["dcs"]) / np.max(z["dcs"])) < 1e-12
    assert np.all(np.abs(dcs - z["dcs"]) <= 1e-11 * np.abs(z["dcs"]) + 1e-14 * np.max(z["dcs"]))
    assert abs(tab.tcs(z["I_dir"], z["I_exc"]) - float(z["tcs"][0])) <= 1e-12 * float(z["tcs"][0])
