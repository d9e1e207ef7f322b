"""Ragged multi-energy batches: every energy point with its own grid in shared launches, optionally
replayed from a CUDA graph, must give exactly the per-energy results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _point(N, seed, n_pairs=6):
    import bench
    g, z, bounds, pairs = bench.make_workload(N=N, n_cont=n_pairs, n_bound=1, seed_shift=seed)
    bi, bf = bounds[0]
    return dict(grid=g, V_core_array=z, U_i_array=z, bound_i=bi, bound_f=bf, pairs=pairs, U_f_array=z)


@pytest.mark.parametrize("engine", ["dense", "semisep", "tc_bf16x3"])
@pytest.mark.parametrize("graph", [False, True])
def test_sweep_matches_per_energy(engine, graph):
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch, radial_ME_all_L_sweep
    points = [_point(N, seed) for N, seed in ((801, 1), (1203, 2), (2001, 3))]
    L_max = 5
    swept = radial_ME_all_L_sweep(points, L_max, engine=engine, graph=graph, replays=2)
    for pt, res in zip(points, swept):
        ref = radial_ME_all_L_batch(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"], pt["bound_f"],
                                    pt["pairs"], L_max, U_f_array=pt["U_f_array"], engine=engine)
        for a, b in zip(res, ref):
            for L in range(L_max + 1):
                assert a.I_L_direct[L] == b.I_L_direct[L]
                assert a.I_L_exchange[L] == b.I_L_exchange[L]


@pytest.mark.parametrize("engine", ["semisep", "tc_bf16x3"])
def test_sweep_points_sharing_a_grid_match_per_energy(engine):
    """Two transitions on one grid object (as at one energy of a sweep) share the tensor-core
    launch of their exchange forms; every integral equals the per-point evaluation."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch, radial_ME_all_L_sweep
    first = _point(1203, 2, n_pairs=150)
    second = _point(1203, 5, n_pairs=130)
    second["grid"] = first["grid"]
    points = [first, second, _point(801, 1)]
    L_max = 4
    swept = radial_ME_all_L_sweep(points, L_max, engine=engine, graph=True, replays=1)
    for pt, res in zip(points, swept):
        ref = radial_ME_all_L_batch(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"], pt["bound_f"],
                                    pt["pairs"], L_max, U_f_array=pt["U_f_array"], engine=engine)
        for a, b in zip(res, ref):
            for L in range(L_max + 1):
                assert a.I_L_direct[L] == b.I_L_direct[L]
                assert a.I_L_exchange[L] == b.I_L_exchange[L]


def test_sweep_coulomb_points_with_tails_match_reference():
    """Ragged sweep over the golden energy points (Coulomb waves with n1 < N and outer tails on
    the device, H 1s->2p, the low-k standard path): each point equals the reference's I_L."""
    import golden_cases as gc
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_sweep
    points, refs = [], []
    for name in ("heplus_1s2s_100eV", "h_1s2p_50eV", "low_k_standard"):
        common, calls = gc.load_case(name)
        for c in calls:
            kw = dict(c["kwargs"])
            if kw.get("oscillatory_method", "advanced") != "advanced" or kw.get("CC_nodes", 5) != 5 or \
                    not kw.get("use_oscillatory_quadrature", True):
                continue
            grid, V, Ui, bi, bf, ci, cf, L_max = c["args"]
            points.append(dict(grid=grid, V_core_array=V, U_i_array=Ui, bound_i=bi, bound_f=bf, pairs=[(ci, cf)],
                               U_f_array=kw["U_f_array"], L_max=L_max))
            refs.append(c)
    L_max = min(p["L_max"] for p in points)
    for engine in ("semisep", "auto"):
        swept = radial_ME_all_L_sweep(points, L_max, engine=engine, graph=True)
        for res, c in zip(swept, refs):
            d = np.array([res[0].I_L_direct[L] for L in range(L_max + 1)])
            e = np.array([res[0].I_L_exchange[L] for L in range(L_max + 1)])
            for got, ref in ((d, c["ref_dir"][:L_max + 1]), (e, c["ref_exc"][:L_max + 1])):
                scale = np.max(np.abs(ref))
                assert np.all(np.abs(got - ref) <= 1e-11 * np.abs(ref) + 1e-13 * scale), (c["label"], got, ref)


def test_auto_engine_picks_and_caches():
    from dwba_b200 import tune
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_sweep
    points = [_point(N, seed) for N, seed in ((1501, 5), (2301, 6))]
    L_max = 4
    auto = radial_ME_all_L_sweep(points, L_max, engine="auto")
    keys = [k for k in tune.TUNER.choices if k[2] == L_max and k[3] == ("semisep", "dense")]
    assert keys
    chosen = tune.TUNER.choices[keys[-1]]
    assert set(tune.TUNER.timings_ms[keys[-1]]) == {"semisep", "dense"}
    direct = radial_ME_all_L_sweep(points, L_max, engine=chosen)
    for a_pt, b_pt in zip(auto, direct):
        for a, b in zip(a_pt, b_pt):
            assert a.I_L_direct == b.I_L_direct and a.I_L_exchange == b.I_L_exchange
    n_before = len(tune.TUNER.timings_ms)
    radial_ME_all_L_sweep(points, L_max, engine="auto")
    assert len(tune.TUNER.timings_ms) == n_before  # cached: no second timing round
