"""The split-BF16 engine with its accuracy guard on the sweep's worst points.

Without the guard, the tensor-core forms of the 64-energy ragged sweep give TCS errors up to
5.8e-6 at the low-energy points (FP32 values of K_L and FP32 accumulation, about 1e-6 of each
form's scale). The guard (engine.py::TCGuard, theta = 0.1 by default) recomputes in FP64 every
exchange form whose |I_L| exceeds theta times the largest |I_L| of its transition. Checked here on
the two worst points of that sweep (45 eV 1s->2s, N = 2347, 841 pairs; and the lowest-energy
point) through the public sweep entry point: TCS of the split-BF16 integrals against the exact
FP64 engine's within 1e-6, with the guard routing only a small share of the forms, and the same
points without the guard outside that bound (the guard is what brings them in).
"""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


def _points():
    pts = bench.make_ragged_points(64, select=(0, 5))
    return [pts[0], pts[2]]  # 45 eV and the sixth energy, 1s->2s: the worst points of the sweep


def _tcs(pt, d, e):
    from dwba_b200.coupling import CouplingTables
    chans = [(w_i.l, w_f.l) for w_i, w_f in pt["pairs"]]
    tab = CouplingTables(np.linspace(0.0, np.pi, 181), chans, 6, 1.0, 1.0, 0, pt["bound_f"].l)
    return tab.tcs(d, e)


def _sweep(points, engine):
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_sweep
    keys = ("grid", "V_core_array", "U_i_array", "bound_i", "bound_f", "pairs", "U_f_array")
    res = radial_ME_all_L_sweep([{k: pt[k] for k in keys} for pt in points], 6, engine=engine)
    out = []
    for rr in res:
        d = np.array([[x.I_L_direct[L] for L in range(7)] for x in rr])
        e = np.array([[x.I_L_exchange[L] for L in range(7)] for x in rr])
        out.append((d, e))
    return out


def test_guarded_split_bf16_tcs_within_1e6_on_the_worst_points(monkeypatch):
    pts = _points()
    ref = _sweep(pts, "semisep")
    monkeypatch.setenv("DWBA_B200_TC_ROUTE", "0.1")
    tc = _sweep(pts, "tc_bf16x3")
    monkeypatch.setenv("DWBA_B200_TC_ROUTE", "0")
    raw = _sweep(pts, "tc_bf16x3")
    worst_raw = 0.0
    for pt, (rd, re_), (td, te), (ud, ue) in zip(pts, ref, tc, raw):
        t_ref = _tcs(pt, rd, re_)
        assert abs(_tcs(pt, td, te) - t_ref) <= 1e-6 * abs(t_ref)
        worst_raw = max(worst_raw, abs(_tcs(pt, ud, ue) - t_ref) / abs(t_ref))
        routed = np.mean(np.all(te == re_, axis=1))
        assert 0.0 < routed < 0.25, routed  # a small share of the forms is recomputed in FP64
        assert np.array_equal(td, rd)  # the direct forms are exact FP64 on every engine
    assert worst_raw > 1e-6  # without the guard these points miss the bound
