"""Outer tails on the GPU (dwba_outer_tails_batch) against the native host path and the
reference's tail values held in the unit fixture (oscillatory_integrals.py:459-535, :2064-2184)."""
import os

import numpy as np
import pytest
import torch

from dwba_b200 import _lib
from golden_cases import levin_condition

pytestmark = pytest.mark.gpu

UNIT = np.load(os.path.join(os.path.dirname(__file__), "golden", "unit_quadrature.npz"))
SEG, DPHI = 4096, np.pi / 2


def _device_tails(waves, r_m, r_max, moments, mode, L_max, seg=SEG, dphi=DPHI):
    n = len(waves)
    nl = L_max + 1
    mom = torch.tensor(np.asarray(moments, dtype=np.float64).reshape(n, nl), device="cuda")
    out = torch.full((n, nl), np.nan, dtype=torch.float64, device="cuda")
    rec = np.zeros(n, dtype=_lib.TAIL_DTYPE)
    rec["wave"] = waves
    rec["r_m"], rec["r_max"], rec["mode"] = r_m, r_max, mode
    rec["moments"] = mom.data_ptr() + 8 * nl * np.arange(n, dtype=np.uint64)
    rec["out"] = out.data_ptr() + 8 * nl * np.arange(n, dtype=np.uint64)
    rec_d = torch.from_numpy(rec.view(np.uint8).copy()).cuda()
    lib = _lib.load()
    _lib.check(lib.dwba_outer_tails_batch(rec_d.data_ptr(), n, L_max, seg, dphi,
                                          torch.cuda.current_stream().cuda_stream), "dwba_outer_tails_batch")
    return out.cpu().numpy()


@pytest.mark.parametrize("mode", [0, 1])
def test_unit_fixture_tails(mode):
    rows = UNIT["tails"]
    L_max = int(rows[:, 12].max())
    waves, rms, rmaxs, moms, want = [], [], [], [], []
    for row in rows:
        rm, rmax, ki, kf, li, lf, di, df, ei, ef, si, sf, L, mom, t_out, t_inf, t_rm, _ = row
        m = np.zeros(L_max + 1)
        m[int(L)] = mom
        waves.append([ki, li, di, ei, si, kf, lf, df, ef, sf])
        rms.append(rm)
        rmaxs.append(rmax)
        moms.append(m)
        want.append((int(L), t_out + t_inf if mode == 0 else t_rm))
    routed = [mode == 1 or _lib.tail_on_device(w, a, b) for w, a, b in zip(waves, rms, rmaxs)]
    assert all(routed)
    got = _device_tails(np.array(waves), np.array(rms), np.array(rmaxs), np.array(moms), mode, L_max)
    for k, (L, ref) in enumerate(want):
        host = _lib.outer_tails(waves[k], rms[k], rmaxs[k], L_max, moms[k], mode, SEG, DPHI)
        assert got[k, 0] == 0.0
        assert abs(got[k, L] - ref) <= 1e-12 * abs(ref) + 1e-16, (k, got[k, L], ref)
        assert abs(got[k, L] - host[L]) <= 1e-13 * abs(host[L]) + 1e-17, (k, got[k, L], host[L])
        others = [l for l in range(1, L_max + 1) if l != L]
        assert np.all(got[k, others] == 0.0)


def test_random_records_match_host():
    """Coulomb and neutral waves, l up to 20, short and long outer intervals, Filon and Levin branches.
    Filon records agree to round-off; Levin records to round-off times the system's condition number."""
    rng = np.random.default_rng(7)
    n, L_max = 96, 6
    ki = rng.uniform(0.3, 3.0, n)
    kf = ki * rng.uniform(0.2, 0.95, n)
    eta = np.where(rng.random(n) < 0.5, 0.0, -rng.uniform(0.1, 2.0, n))
    waves = np.stack([ki, rng.integers(0, 21, n), rng.uniform(-1, 1, n), eta / ki, rng.uniform(-2, 2, n),
                      kf, rng.integers(0, 21, n), rng.uniform(-1, 1, n), eta / kf, rng.uniform(-2, 2, n)], axis=1)
    r_m = rng.uniform(5.0, 60.0, n)
    r_max = r_m + rng.uniform(1.0, 400.0, n)
    # a second population in the Levin regime: high l, near-threshold k_f, short outer intervals
    m2 = 48
    k2 = rng.uniform(0.5, 2.0, m2)
    kf2 = k2 * rng.uniform(0.85, 0.98, m2)
    eta2 = np.where(rng.random(m2) < 0.5, 0.0, -rng.uniform(0.1, 1.0, m2))
    waves = np.concatenate([waves, np.stack([k2, rng.integers(8, 31, m2), rng.uniform(-1, 1, m2), eta2 / k2,
                                             rng.uniform(-2, 2, m2), kf2, rng.integers(8, 31, m2),
                                             rng.uniform(-1, 1, m2), eta2 / kf2, rng.uniform(-2, 2, m2)], axis=1)])
    rm2 = rng.uniform(4.0, 15.0, m2)
    r_m = np.concatenate([r_m, rm2])
    r_max = np.concatenate([r_max, rm2 + rng.uniform(2.0, 30.0, m2)])
    n += m2
    moms = rng.normal(size=(n, L_max + 1)) * 10.0 ** rng.uniform(-3, 1, (n, 1))
    moms[::7, 2] = 0.0  # moments below the cut-off give a zero tail
    keep = np.array([_lib.tail_on_device(w, a, b) for w, a, b in zip(waves, r_m, r_max)])
    assert keep.all()
    cond = np.array([levin_condition(w, a, b) for w, a, b in zip(waves, r_m, r_max)])
    assert (cond == 0).sum() >= 20 and (cond > 0).sum() >= 10  # both branches exercised
    for mode in (0, 1):
        got = _device_tails(waves, r_m, r_max, moms, mode, L_max)
        for k in range(n):
            host = _lib.outer_tails(waves[k], r_m[k], r_max[k], L_max, moms[k], mode, SEG, DPHI)
            scale = np.abs(moms[k]) / r_m[k] ** (np.arange(L_max + 1) + 1) * (r_max[k] - r_m[k])
            rel = 1e-14 + (1e-16 * cond[k] if mode == 0 else 0.0)
            assert np.all(np.abs(got[k] - host) <= 1e-13 * np.abs(host) + rel * scale), (mode, k, got[k], host)


def test_segment_cap_and_dphi_limits():
    """Tighter Filon segment caps and phase steps change the node count per segment identically."""
    w = np.array([[2.0, 1, 0.2, 0.0, 0.0, 1.4, 2, -0.3, 0.0, 0.0]])
    m = np.array([[0.0, 0.7, -0.2, 0.05]])
    for seg, dphi in ((128, np.pi / 16), (300, np.pi / 4), (4096, np.pi / 2)):
        got = _device_tails(w, np.array([12.0]), np.array([900.0]), m, 0, 3, seg, dphi)[0]
        host = _lib.outer_tails(w[0], 12.0, 900.0, 3, m[0], 0, seg, dphi)
        assert np.allclose(got, host, rtol=1e-13, atol=1e-18)


def test_dropin_device_tails_equal_host_tails(monkeypatch):
    """The drop-in call with tails on the device and on the host agrees to FP64 round-off."""
    import golden_cases as gc
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L
    for call in gc.all_calls():
        monkeypatch.setenv("DWBA_B200_TAILS", "device")
        a = radial_ME_all_L(*call["args"], **call["kwargs"])
        monkeypatch.setenv("DWBA_B200_TAILS", "host")
        b = radial_ME_all_L(*call["args"], **call["kwargs"])
        L = call["L_max"]
        da = np.array([a.I_L_direct[l] for l in range(L + 1)])
        db = np.array([b.I_L_direct[l] for l in range(L + 1)])
        assert np.all(np.abs(da - db) <= 1e-13 * np.abs(db) + 1e-18), (call["label"], da, db)
        assert all(a.I_L_exchange[l] == b.I_L_exchange[l] for l in range(L + 1))


def test_many_multipoles_in_several_chunks():
    """L_max = 19: the device kernel takes the multipoles in chunks of eight (1..8, 9..16, 17..19);
    every entry of every chunk equals the host path (Levin records to round-off times the condition
    number of their collocation systems, as in test_random_records_match_host), and zero moments
    give zero tails."""
    rng = np.random.default_rng(21)
    n, L_max = 40, 19
    ki = rng.uniform(0.5, 3.0, n)
    kf = ki * rng.uniform(0.3, 0.9, n)
    eta = np.where(rng.random(n) < 0.5, 0.0, -rng.uniform(0.1, 1.0, n))
    waves = np.stack([ki, rng.integers(0, 15, n), rng.uniform(-1, 1, n), eta / ki, rng.uniform(-2, 2, n),
                      kf, rng.integers(0, 15, n), rng.uniform(-1, 1, n), eta / kf, rng.uniform(-2, 2, n)], axis=1)
    r_m = rng.uniform(10.0, 40.0, n)
    r_max = r_m + rng.uniform(20.0, 200.0, n)
    moms = rng.normal(size=(n, L_max + 1)) * 10.0 ** rng.uniform(-2, 1, (n, 1))
    moms[::5, 9:17] = 0.0  # a whole chunk of zero moments
    assert all(_lib.tail_on_device(w, a, b) for w, a, b in zip(waves, r_m, r_max))
    cond = np.array([levin_condition(w, a, b) for w, a, b in zip(waves, r_m, r_max)])
    for mode in (0, 1):
        got = _device_tails(waves, r_m, r_max, moms, mode, L_max)
        for k in range(n):
            host = _lib.outer_tails(waves[k], r_m[k], r_max[k], L_max, moms[k], mode, SEG, DPHI)
            scale = np.abs(moms[k]) / r_m[k] ** (np.arange(L_max + 1) + 1) * (r_max[k] - r_m[k])
            rel = 1e-14 + (1e-16 * cond[k] if mode == 0 else 0.0)
            assert got[k, 0] == 0.0
            assert np.all(np.abs(got[k] - host) <= 1e-13 * np.abs(host) + rel * scale), (mode, k, cond[k], got[k], host)
        assert np.all(got[::5, 9:17] == 0.0)
