"""The oracle (CPU restatement of the reference) against golden vectors produced by the reference."""
import numpy as np
import pytest

import golden_cases as gc
import oracle
from oracle.folded import fold_pair, folded_eval, semiseparable_eval
from oracle.quadrature import cc_reference, clenshaw_curtis_nodes, generate_phase_nodes, adaptive_phase_increment, interp_on_radial_grid
from oracle.tails import analytical_multipole_tail, outer_integral_1d

UNIT = np.load(gc.GOLDEN_DIR + "/unit_quadrature.npz")
# The full restatement materialises N x N_cc exchange temporaries like the reference: keep it to small cases.
FAST = [c for c in gc.all_calls() if not c["label"].startswith(("synthetic", "large_grid"))]


def _gate(x, ref, scale, rel=1e-12, abs_scale=1e-14):
    """Parity gate: |x - ref| <= rel |ref| + abs_scale * S_L (S_L bounds cancellation)."""
    return np.abs(np.asarray(x) - ref) <= rel * np.abs(ref) + abs_scale * scale


def _scales(call, fp):
    r = call["args"][0].r
    L = call["L_max"]
    sd = folded_eval(r, np.abs(fp["a_dir"]), np.abs(fp["b_dir"]), L) + np.abs(fp["tail"])
    se = folded_eval(r, np.abs(fp["a_ex"]), np.abs(fp["b_ex"]), L)
    sd[0] += abs(fp["corr_dir"])
    se[0] += abs(fp["corr_ex"])
    return sd, se


@pytest.mark.parametrize("call", FAST, ids=[c["label"] for c in FAST])
def test_restatement_matches_reference(call):
    d, e = oracle.radial_me_all_L(*call["args"], **call["kwargs"])
    fp = fold_pair(*call["args"], **call["kwargs"])
    sd, se = _scales(call, fp)
    L = call["L_max"]
    assert _gate([d[l] for l in range(L + 1)], call["ref_dir"], sd).all()
    assert _gate([e[l] for l in range(L + 1)], call["ref_exc"], se).all()


@pytest.mark.parametrize("call", gc.all_calls(), ids=[c["label"] for c in gc.all_calls()])
def test_folded_and_semiseparable_match_reference(call):
    fp = fold_pair(*call["args"], **call["kwargs"])
    r = call["args"][0].r
    L = call["L_max"]
    sd, se = _scales(call, fp)
    for ev in (folded_eval, semiseparable_eval):
        d = ev(r, fp["a_dir"], fp["b_dir"], L) + fp["tail"]
        e = ev(r, fp["a_ex"], fp["b_ex"], L)
        d[0] += fp["corr_dir"]
        e[0] += fp["corr_ex"]
        assert _gate(d, call["ref_dir"], sd, abs_scale=2e-14).all(), ev.__name__
        assert _gate(e, call["ref_exc"], se, abs_scale=2e-14).all(), ev.__name__


def test_cc_reference_weights():
    for n in (2, 3, 5, 7, 9):
        x, w = cc_reference(n)
        np.testing.assert_allclose(x, UNIT[f"cc_x_{n}"], rtol=0, atol=1e-15)
        np.testing.assert_allclose(w, UNIT[f"cc_w_{n}"], rtol=0, atol=1e-15)
        # known answer of the reference's debug/diag_oscillatory.py:20-24 (general rule on [0, 1])
        _, w01 = clenshaw_curtis_nodes(n, 0.0, 1.0)
        assert abs(np.sum(w01) - 1.0) < 1e-14
    # the cached n=5 table the quadrature actually uses sums to 31/15 on [-1, 1]
    assert abs(np.sum(cc_reference(5)[1]) - 31.0 / 15.0) < 1e-14


def test_phase_nodes_bit_exact():
    from golden_cases import Grid  # noqa: F401
    r = np.load(gc.GOLDEN_DIR + "/case_h_1s2p_50eV.npz")["r"]
    for i in range(5):
        n, k, dphi, eta, d_ref = UNIT[f"phase_params_{i}"]
        rr = r[: int(n)]
        d = adaptive_phase_increment(rr, k, dphi, eta_total=eta)
        assert d == d_ref
        nodes = generate_phase_nodes(rr[0], rr[-1], k, d, eta_total=eta)
        np.testing.assert_array_equal(nodes, UNIT[f"phase_nodes_{i}"])


def test_log_grid_interpolation():
    r = np.load(gc.GOLDEN_DIR + "/case_h_1s2p_50eV.npz")["r"]
    y = np.sin(r) * np.exp(-0.01 * r)
    np.testing.assert_allclose(interp_on_radial_grid(UNIT["interp_x"], r, y), UNIT["interp_y"], rtol=1e-13, atol=1e-15)


def test_outer_tails_restatement():
    for row in UNIT["tails"]:
        rm, rmax, ki, kf, li, lf, di, df, ei, ef, si, sf, L, mom, t_out, t_inf, t_rm, _ = row
        li, lf, L = int(li), int(lf), int(L)
        env = (lambda m, LL: (lambda x: m / (x ** (LL + 1)) if x > 1e-6 else 0.0))(mom, L)
        v = outer_integral_1d(env, ki, li, di, ei, si, kf, lf, df, ef, sf, rm, rmax)
        assert abs(v - t_out) <= 1e-12 * abs(t_out) + 1e-16
        assert abs(analytical_multipole_tail(rmax, ki, kf, di, df, li, lf, L, mom, ei, ef, si, sf) - t_inf) <= 1e-14 * abs(t_inf) + 1e-18
        assert abs(analytical_multipole_tail(rm, ki, kf, di, df, li, lf, L, mom, ei, ef, si, sf) - t_rm) <= 1e-14 * abs(t_rm) + 1e-18


def test_hydrogen_slater_F0_known_answer():
    """F0(1s,1s) = int int u^2 (1/r>) u^2 = 5/8 Ha for hydrogen (closed form)."""
    from oracle.folded import semiseparable_eval
    r = np.geomspace(1e-5, 60.0, 6001)
    # Simpson-like trapezoid weights on the log grid
    w = np.zeros_like(r)
    w[1:-1] = 0.5 * (r[2:] - r[:-2])
    w[0] = 0.5 * (r[1] - r[0])
    w[-1] = 0.5 * (r[-1] - r[-2])
    u2 = 4.0 * r * r * np.exp(-2 * r)
    a = w * u2
    F0 = semiseparable_eval(r, a, a, 0)[0]
    F0d = folded_eval(r, a, a, 0)[0]
    assert abs(F0 - 0.625) < 2e-6 and abs(F0d - F0) < 1e-13


def test_oracle_config1_sample():
    """The folded oracle against the reference's own I_L for config 1 (H 1s->2p, 50 eV, N = 3000)
    on 16 of its 128 pairs: 1e-12 relative or 1e-13 of the pair's largest multipole."""
    import json
    import os
    z = np.load(os.path.join(gc.GOLDEN_DIR, "config1.npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    grid = gc.Grid(r=z["r"], dr=z["dr"], w_trapz=z["w_trapz"], w_simpson=z["w_simpson"])
    bi = gc.BoundOrbital(l=0, energy_au=-0.5, u_of_r=z["u_i"], n_index=1)
    bf = gc.BoundOrbital(l=1, energy_au=-0.125, u_of_r=z["u_f"], n_index=1)
    L = meta["L_max"]
    for p in range(0, len(meta["pairs"]), 8):
        li, lf = meta["pairs"][p]
        ci = gc._wave(meta["waves_i"][str(li)], z["chi_i"][li])
        cf = gc._wave(meta["waves_f"][str(lf)], z["chi_f"][lf])
        fp = fold_pair(grid, z["V_core"], z["U_i"], bi, bf, ci, cf, L, U_f_array=z["U_f"])
        Id = folded_eval(grid.r, fp["a_dir"], fp["b_dir"], L) + fp["tail"]
        Ie = folded_eval(grid.r, fp["a_ex"], fp["b_ex"], L)
        Id[0] += fp["corr_dir"]
        Ie[0] += fp["corr_ex"]
        for I, R in ((Id, z["I_dir"][p]), (Ie, z["I_exc"][p])):
            assert np.all(np.abs(I - R) <= 1e-12 * np.abs(R) + 1e-13 * np.max(np.abs(R))), (li, lf, I, R)


CUPY = np.load(gc.GOLDEN_DIR + "/cupy_semantics.npz")


@pytest.mark.parametrize("call", [c for c in gc.all_calls() if not c["label"].startswith("large_grid")],
                         ids=[c["label"] for c in gc.all_calls() if not c["label"].startswith("large_grid")])
def test_cupy_path_restatement_matches_reference_gpu_path(call):
    """The oracle's restatement of the reference's CuPy path (oracle/cupy_path.py) against that path's
    own outputs, recorded on the CPU through a NumPy stand-in for CuPy (tests/golden/make_cupy_golden.py)."""
    from oracle.cupy_path import radial_me_all_L_cupy
    name, idx = call["label"].rstrip("]").split("[")
    d, e = radial_me_all_L_cupy(*call["args"], **call["kwargs"])
    L = call["L_max"]
    for got, key in ((d, f"{name}_{idx}_dir"), (e, f"{name}_{idx}_exc")):
        ref = CUPY[key]
        g = np.array([got[l] for l in range(L + 1)])
        assert np.all(np.abs(g - ref) <= 1e-12 * np.abs(ref) + 1e-14 * np.max(np.abs(ref))), (key, g, ref)
