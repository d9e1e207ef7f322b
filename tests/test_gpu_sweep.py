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


@pytest.mark.parametrize("engine", ["dense", "semisep"])
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
