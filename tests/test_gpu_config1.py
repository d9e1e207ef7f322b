"""Config 1 (H 1s->2p, 50 eV, N = 3000, 128 (l_i, l_f) pairs, L = 0..4) through every engine.

Reference I_L come from ``tests/golden/make_config1.py`` (the reference's ``radial_ME_all_L`` on
its own solver outputs). The DCS/TCS errors use the exact gradients of the reference's DCS and TCS
with respect to each integral (``tests/golden/make_config1_sensitivity.py``): the DCS is a
quadratic form in the integrals, so dTCS = g . dI up to O(|dI|^2) (relative 1e-13 here)."""
import json
import os

import numpy as np
import pytest

import golden_cases as gc

pytestmark = pytest.mark.gpu

Z = np.load(os.path.join(gc.GOLDEN_DIR, "config1.npz"))
SENS = np.load(os.path.join(gc.GOLDEN_DIR, "config1_sens.npz"))
META = json.loads(bytes(Z["meta_json"]).decode())
# TCS and DCS tolerance per engine (relative); the split-BF16 bound is the accuracy target of the
# tensor-core forms, the FP64 engines must agree to round-off
TCS_TOL = {"dense": 1e-12, "semisep": 1e-12, "tc_bf16x3": 1e-6, "tc_bf16x6": 1e-6}


def inputs():
    grid = gc.Grid(r=Z["r"], dr=Z["dr"], w_trapz=Z["w_trapz"], w_simpson=Z["w_simpson"])
    bi = gc.BoundOrbital(l=0, energy_au=-0.5, u_of_r=Z["u_i"], n_index=1)
    bf = gc.BoundOrbital(l=1, energy_au=-0.125, u_of_r=Z["u_f"], n_index=1)
    wi = {int(l): gc._wave(v, Z["chi_i"][int(l)]) for l, v in META["waves_i"].items()}
    wf = {int(l): gc._wave(v, Z["chi_f"][int(l)]) for l, v in META["waves_f"].items()}
    pairs = [(wi[li], wf[lf]) for li, lf in META["pairs"]]
    return grid, bi, bf, pairs


@pytest.fixture(scope="module")
def engine_results():
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch
    grid, bi, bf, pairs = inputs()
    out = {}
    nl = META["L_max"] + 1
    for eng in TCS_TOL:
        res = radial_ME_all_L_batch(grid, Z["V_core"], Z["U_i"], bi, bf, pairs, META["L_max"], U_f_array=Z["U_f"],
                                    engine=eng)
        out[eng] = np.stack([np.array([[r.I_L_direct[L] for L in range(nl)] for r in res]),
                             np.array([[r.I_L_exchange[L] for L in range(nl)] for r in res])])
    return out


@pytest.mark.parametrize("engine", list(TCS_TOL))
def test_config1_tcs_and_dcs_errors(engine_results, engine):
    I_ref = np.stack([Z["I_dir"], Z["I_exc"]])
    dI = engine_results[engine] - I_ref
    tcs = float(SENS["tcs"][0])
    d_tcs = float(np.sum(SENS["dtcs"] * dI))
    d_dcs = np.einsum("akpl,kpl->a", SENS["ddcs"], dI)
    rel_tcs = abs(d_tcs) / tcs
    rel_dcs = np.max(np.abs(d_dcs) / SENS["dcs_sel"])
    print(f"{engine}: TCS rel {rel_tcs:.2e}, max DCS rel (19 angles) {rel_dcs:.2e}, "
          f"max |dI|/|I| {np.max(np.abs(dI) / np.maximum(np.abs(I_ref), 1e-300)):.2e}")
    assert rel_tcs <= TCS_TOL[engine]
    assert rel_dcs <= 10 * TCS_TOL[engine]


@pytest.mark.parametrize("engine", ["dense", "semisep"])
def test_config1_fp64_integrals_match_reference(engine_results, engine):
    """Every integral of the FP64 engines within 1e-12 relative or 1e-13 of the pair's largest multipole."""
    I_ref = np.stack([Z["I_dir"], Z["I_exc"]])
    scale = np.max(np.abs(I_ref), axis=2, keepdims=True)
    ok = np.abs(engine_results[engine] - I_ref) <= 1e-12 * np.abs(I_ref) + 1e-13 * scale
    assert ok.all(), np.argwhere(~ok)[:5]


def test_gpu_cross_sections_match_reference(engine_results):
    """DCS/TCS on the device (dwba_cross_sections with the host coupling tables) from the reference's
    integrals reproduce the reference's DCS and TCS; from each engine's integrals they stay within
    that engine's tolerance (exact evaluation, no linearisation)."""
    from dwba_b200.coupling import CouplingTables
    tab = CouplingTables(Z["theta"], [tuple(p) for p in META["pairs"]], META["L_max"], META["k_i"], META["k_f"], 0, 1)
    dcs, tcs = tab.cross_sections_gpu(Z["I_dir"], Z["I_exc"])
    dcs = dcs.cpu().numpy()
    assert np.all(np.abs(dcs - Z["dcs"]) <= 1e-11 * np.abs(Z["dcs"]) + 1e-14 * np.max(Z["dcs"]))
    assert abs(float(tcs[0]) - float(Z["tcs"][0])) <= 1e-12 * float(Z["tcs"][0])
    for eng, I in engine_results.items():
        _, t = tab.cross_sections_gpu(I[0], I[1])
        rel = abs(float(t[0]) - float(Z["tcs"][0])) / float(Z["tcs"][0])
        print(f"{eng}: TCS through the device coupling, rel {rel:.2e}")
        assert rel <= TCS_TOL[eng]
