"""GPU parity: the drop-in module (CUDA engine through the C ABI) against the reference's golden vectors
and the oracle, with the gate |dI| <= 1e-12 |I_ref| + 1e-14 S_L (S_L = |a|^T K_L |b| + |c_L| + |t_L|)."""
import numpy as np
import pytest

import golden_cases as gc
from oracle.folded import fold_pair, folded_eval, semiseparable_eval

pytestmark = pytest.mark.gpu

CALLS = gc.all_calls()


def _scales(call):
    fp = fold_pair(*call["args"], **call["kwargs"])
    r = call["args"][0].r
    L = call["L_max"]
    sd = folded_eval(r, np.abs(fp["a_dir"]), np.abs(fp["b_dir"]), L) + np.abs(fp["tail"])
    se = folded_eval(r, np.abs(fp["a_ex"]), np.abs(fp["b_ex"]), L)
    sd[0] += abs(fp["corr_dir"])
    se[0] += abs(fp["corr_ex"])
    return sd, se


def _check(res, call, sd, se, abs_scale=1e-14):
    L = call["L_max"]
    d = np.array([res.I_L_direct[l] for l in range(L + 1)])
    e = np.array([res.I_L_exchange[l] for l in range(L + 1)])
    assert sorted(res.I_L_direct) == list(range(L + 1)) and sorted(res.I_L_exchange) == list(range(L + 1))
    assert all(type(v) is float for v in res.I_L_direct.values())
    ok_d = np.abs(d - call["ref_dir"]) <= 1e-12 * np.abs(call["ref_dir"]) + abs_scale * sd
    ok_e = np.abs(e - call["ref_exc"]) <= 1e-12 * np.abs(call["ref_exc"]) + abs_scale * se
    assert ok_d.all(), (d, call["ref_dir"])
    assert ok_e.all(), (e, call["ref_exc"])


@pytest.mark.parametrize("engine", ["dense", "semisep"])
@pytest.mark.parametrize("call", CALLS, ids=[c["label"] for c in CALLS])
def test_dropin_matches_reference_goldens(call, engine):
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L
    sd, se = _scales(call)
    res = radial_ME_all_L(*call["args"], **call["kwargs"], engine=engine)
    _check(res, call, sd, se, abs_scale=1e-14 if engine == "dense" else 3e-14)


def test_gpu_signature_with_cache_and_batch_agree():
    from dwba_b200.dwba_matrix_elements import (GPUCache, radial_ME_all_L, radial_ME_all_L_batch,
                                                radial_ME_all_L_gpu)
    common, calls = gc.load_case("h_1s2p_50eV")
    grid = common["grid"]
    cache = GPUCache.from_grid(grid, max_chi_cached=20)
    advanced = [c for c in calls if not c["kwargs"].keys() - {"U_f_array"}]
    singles = [radial_ME_all_L_gpu(*c["args"], gpu_cache=cache, **c["kwargs"]) for c in advanced]
    pairs = [(c["args"][5], c["args"][6]) for c in advanced]
    a = advanced[0]["args"]
    batch = radial_ME_all_L_batch(a[0], a[1], a[2], a[3], a[4], pairs, advanced[0]["L_max"],
                                  U_f_array=advanced[0]["kwargs"]["U_f_array"], gpu_cache=cache)
    for s, b, c in zip(singles, batch, advanced):
        assert s.I_L_direct == b.I_L_direct and s.I_L_exchange == b.I_L_exchange  # same kernels, same order
        cpu_sig = radial_ME_all_L(*c["args"], **c["kwargs"])
        assert cpu_sig.I_L_direct == s.I_L_direct
    # the same batch as two arrays (no result object per pair)
    d, e = radial_ME_all_L_batch(a[0], a[1], a[2], a[3], a[4], pairs, advanced[0]["L_max"],
                                 U_f_array=advanced[0]["kwargs"]["U_f_array"], gpu_cache=cache, as_arrays=True)
    L = advanced[0]["L_max"]
    assert d.shape == e.shape == (len(pairs), L + 1)
    for p, b in enumerate(batch):
        assert list(d[p]) == [b.I_L_direct[l] for l in range(L + 1)]
        assert list(e[p]) == [b.I_L_exchange[l] for l in range(L + 1)]
    cache.clear()


def test_deterministic_repeat():
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L
    call = CALLS[0]
    r1 = radial_ME_all_L(*call["args"], **call["kwargs"])
    r2 = radial_ME_all_L(*call["args"], **call["kwargs"])
    assert r1 == r2


def test_errors_match_reference():
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L, radial_ME_all_L_gpu
    call = CALLS[0]
    args = list(call["args"])
    args[7] = -1
    with pytest.raises(ValueError):
        radial_ME_all_L(*args, **call["kwargs"])
    args = list(call["args"])
    args[1] = args[1][:-5]  # V_core shorter than the grid
    with pytest.raises(ValueError):
        radial_ME_all_L_gpu(*args, **call["kwargs"])


def _synthetic(N, r_max, n_pairs, seed, L_max=8):
    """Seeded config-2-like inputs on an exponential grid (waves sin(kr - l pi/2 + d)(1 - exp(-(r/r0)^(l+1))))."""
    from golden_cases import BoundOrbital, ContinuumWave, Grid
    rng = np.random.default_rng(seed)
    idx = np.linspace(0.0, 1.0, N)
    r = 1e-5 * ((r_max / 1e-5) ** idx)
    dr = np.diff(r)
    wt = np.zeros(N)
    wt[0], wt[-1] = 0.5 * dr[0], 0.5 * dr[-1]
    wt[1:-1] = 0.5 * (r[2:] - r[:-2])
    ws = np.zeros(N)
    for i in range(0, N - 2, 2):
        h1, h2 = dr[i], dr[i + 1]
        ws[i] += (h1 + h2) / 6.0 * (2.0 - h2 / h1)
        ws[i + 1] += (h1 + h2) / 6.0 * ((h1 + h2) ** 2 / (h1 * h2))
        ws[i + 2] += (h1 + h2) / 6.0 * (2.0 - h1 / h2)
    if N % 2 == 0:
        ws[-2] += 0.5 * dr[-1]
        ws[-1] += 0.5 * dr[-1]
    grid = Grid(r=r, dr=np.append(dr, dr[-1]), w_trapz=wt, w_simpson=ws)
    u = []
    for _ in range(2):
        a, b, c = rng.integers(1, 3), rng.uniform(0.5, 2.0), rng.uniform(-1, 1, 3)
        v = r ** a * np.exp(-b * r) * (c[0] + c[1] * r + c[2] * r * r)
        u.append(v / np.sqrt(np.sum(wt * v * v)))
    pairs = []
    for _ in range(n_pairs):
        k = rng.uniform(0.5, 8.0, 2)
        d = rng.uniform(0, np.pi, 2)
        l = rng.integers(0, 64, 2)
        w = [ContinuumWave(l=int(l[j]), k_au=float(k[j]), phase_shift=float(d[j]),
                           chi_of_r=np.sin(k[j] * r - 0.5 * l[j] * np.pi + d[j]) *
                           (1 - np.exp(-(r / ((l[j] + 1) / k[j])) ** (l[j] + 1)))) for j in range(2)]
        pairs.append(tuple(w))
    z = np.zeros(N)
    return grid, z, BoundOrbital(0, -0.5, u[0], 1), BoundOrbital(1, -0.1, u[1], 1), pairs, L_max


def test_engine_vs_oracle_larger_grid():
    """N = 4001 to r = 400 (beyond the golden sizes): engine vs the oracle's folded operands."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch
    grid, z, bi, bf, pairs, L_max = _synthetic(4001, 400.0, 3, seed=11)
    for engine in ("dense", "semisep"):
        res = radial_ME_all_L_batch(grid, z, z, bi, bf, pairs, L_max, U_f_array=z, engine=engine)
        for (ci, cf), rr in zip(pairs, res):
            fp = fold_pair(grid, z, z, bi, bf, ci, cf, L_max, U_f_array=z)
            d = semiseparable_eval(grid.r, fp["a_dir"], fp["b_dir"], L_max)
            e = semiseparable_eval(grid.r, fp["a_ex"], fp["b_ex"], L_max)
            sd = semiseparable_eval(grid.r, np.abs(fp["a_dir"]), np.abs(fp["b_dir"]), L_max)
            se = semiseparable_eval(grid.r, np.abs(fp["a_ex"]), np.abs(fp["b_ex"]), L_max)
            gd = np.array([rr.I_L_direct[l] for l in range(L_max + 1)])
            ge = np.array([rr.I_L_exchange[l] for l in range(L_max + 1)])
            assert np.all(np.abs(gd - d) <= 1e-12 * np.abs(d) + 3e-14 * sd), engine
            assert np.all(np.abs(ge - e) <= 1e-12 * np.abs(e) + 3e-14 * se), engine


def test_engine_vs_oracle_two_multipole_chunks():
    """L_max = 12 (the FP64 kernels take multipoles 0..8 and 9..12 in two launches) on N = 2001:
    dense and semiseparable engines against the oracle's folded operands."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch
    grid, z, bi, bf, pairs, L_max = _synthetic(2001, 200.0, 3, seed=13, L_max=12)
    for engine in ("dense", "semisep"):
        res = radial_ME_all_L_batch(grid, z, z, bi, bf, pairs, L_max, U_f_array=z, engine=engine)
        for (ci, cf), rr in zip(pairs, res):
            fp = fold_pair(grid, z, z, bi, bf, ci, cf, L_max, U_f_array=z)
            d = semiseparable_eval(grid.r, fp["a_dir"], fp["b_dir"], L_max)
            e = semiseparable_eval(grid.r, fp["a_ex"], fp["b_ex"], L_max)
            sd = semiseparable_eval(grid.r, np.abs(fp["a_dir"]), np.abs(fp["b_dir"]), L_max)
            se = semiseparable_eval(grid.r, np.abs(fp["a_ex"]), np.abs(fp["b_ex"]), L_max)
            gd = np.array([rr.I_L_direct[l] for l in range(L_max + 1)])
            ge = np.array([rr.I_L_exchange[l] for l in range(L_max + 1)])
            assert np.all(np.abs(gd - d) <= 1e-12 * np.abs(d) + 3e-14 * sd), engine
            assert np.all(np.abs(ge - e) <= 1e-12 * np.abs(e) + 3e-14 * se), engine


@pytest.mark.parametrize("engine", ["tc_bf16x3", "tc_bf16x6"])
def test_tensor_core_engines_many_multipoles(engine):
    """The split-BF16 forms at L_max = 12 on N = 2001: every integral within 1e-5 of the scale
    S_L = |a|^T K_L |b| of the oracle's folded operands (FP32-accumulated products)."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch
    grid, z, bi, bf, pairs, L_max = _synthetic(2001, 200.0, 3, seed=17, L_max=12)
    res = radial_ME_all_L_batch(grid, z, z, bi, bf, pairs, L_max, U_f_array=z, engine=engine)
    for (ci, cf), rr in zip(pairs, res):
        fp = fold_pair(grid, z, z, bi, bf, ci, cf, L_max, U_f_array=z)
        e = semiseparable_eval(grid.r, fp["a_ex"], fp["b_ex"], L_max)
        se = semiseparable_eval(grid.r, np.abs(fp["a_ex"]), np.abs(fp["b_ex"]), L_max)
        ge = np.array([rr.I_L_exchange[l] for l in range(L_max + 1)])
        assert np.all(np.abs(ge - e) <= 1e-5 * se), (engine, np.max(np.abs(ge - e) / se))


def test_semiseparable_overflow_guard():
    from dwba_b200 import _lib
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L
    call = CALLS[0]
    args = list(call["args"])
    args[7] = 60  # (1e-5)^-(61) overflows FP64
    with pytest.raises(_lib.DWBAError):
        radial_ME_all_L(*args, **call["kwargs"], engine="semisep")


def test_ionization_transitions_in_one_batch_equal_single_calls():
    """Several ejected waves (one transition each, as one ejected energy of the reference's ionization
    loop, ionization.py:526-608) with all (l_i, l_f) pairs in one batch: every (transition, pair)
    equals the single call, and the golden ejected wave equals the reference."""
    import dataclasses
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L, radial_ME_all_L_batch
    common, calls = gc.load_case("h_ionization_100eV")
    grid, V, Ui, bi, bf = common["grid"], common["V_core"], common["U_i"], common["bound_i"], common["bound_f"]
    r = np.asarray(grid.r)
    ejected = [bf] + [dataclasses.replace(bf, chi_of_r=bf.chi_of_r * (1.0 + s * np.exp(-r / 7.0)),
                                          phase_shift=bf.phase_shift + 0.1 * s) for s in (0.3, -0.2)]
    L_max = min(c["L_max"] for c in calls)
    pairs = [(c["args"][5], c["args"][6]) for c in calls]
    kw = dict(calls[0]["kwargs"])
    batch = radial_ME_all_L_batch(grid, V, Ui, [bi] * len(ejected), ejected, pairs, L_max, **kw)
    assert len(batch) == len(ejected) and all(len(b) == len(pairs) for b in batch)
    for t, ej in enumerate(ejected):
        for p, (ci, cf) in enumerate(pairs):
            single = radial_ME_all_L(grid, V, Ui, bi, ej, ci, cf, L_max, **kw)
            assert batch[t][p].I_L_direct == single.I_L_direct
            assert batch[t][p].I_L_exchange == single.I_L_exchange
    for p, c in enumerate(calls):
        d = np.array([batch[0][p].I_L_direct[L] for L in range(L_max + 1)])
        assert np.all(np.abs(d - c["ref_dir"][:L_max + 1]) <= 1e-11 * np.abs(c["ref_dir"][:L_max + 1]) +
                      1e-13 * np.max(np.abs(c["ref_dir"])))
