"""Node sets applied at once to their pair's folds (dwba_build_nodesets_folded).

When every node set of a batch serves one pair (pairs at different energies), the engine builds
each set's banded operators in registers and applies them to that pair's multi-folds in the same
kernel, instead of storing the operators and folding in a second launch. The arithmetic is the
fold kernel's, so the integrals must be bit-identical to the stored path: plane-wave-like pairs
with n1 = N, and Coulomb-like pairs (breakpoint lists, eta != 0) with n1 < N.
"""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


def _inputs(kind):
    """(grid, V, U, bounds, pairs) of the two test batches."""
    if kind == "log":
        g, z, bounds, pairs = bench.make_workload(N=3001, n_cont=96, n_bound=4, seed_shift=21)
        V = U = z
    else:
        # Coulomb-like waves (eta = -1/k, matching index inside the grid: n1 < N) at a different
        # energy per pair, on a log grid to r = 200, hydrogenic bound states
        rng = np.random.default_rng(8)
        g = bench.make_grid(2500, 1e-5, 200.0)
        r = g.r
        im = int(np.searchsorted(r, 120.0))
        pairs = []
        for _ in range(70):
            w = []
            k0 = float(rng.uniform(1.5, 6.0))
            for l, k in ((int(rng.integers(0, 30)), k0), (int(rng.integers(0, 30)), k0 * 0.9)):
                eta, d, sig = -1.0 / k, float(rng.uniform(0, np.pi)), float(rng.uniform(-1, 1))
                chi = np.sin(k * r - 0.5 * l * np.pi + eta * np.log(2 * k * r) + sig + d) * \
                    (1.0 - np.exp(-(r / ((l + 1) / k)) ** (l + 1)))
                wv = bench._Wave(l, k, d, chi)
                wv.eta, wv.sigma_l, wv.idx_match = eta, sig, im
                w.append(wv)
            pairs.append(tuple(w))
        Z = 2.0
        u1s = 2.0 * Z ** 1.5 * r * np.exp(-Z * r)
        u2p = (Z / 2) ** 2.5 / np.sqrt(6.0) * r * r * np.exp(-Z * r / 2)
        bounds = [(bench._Bound(0, u1s), bench._Bound(1, u2p))]
        V = U = -Z / r
    return g, V, U, bounds, pairs


def _job(kind):
    from dwba_b200.dwba_matrix_elements import GPUCache, _make_job
    g, V, U, bounds, pairs = _inputs(kind)
    cache = GPUCache.from_grid(g)
    job = _make_job(g, V, U, [b[0] for b in bounds], [b[1] for b in bounds], pairs, 6, U, {}, cache)
    return job, cache


@pytest.mark.parametrize("kind", ["log", "coulomb"])
def test_fused_node_sets_match_stored_operators(kind):
    from dwba_b200.engine import PreparedJob
    job, cache = _job(kind)
    fu = PreparedJob(job, cache.dg, "semisep", rebuild_nodesets=True, fuse_folds=True)
    un = PreparedJob(job, cache.dg, "semisep", plans=fu.plans, rebuild_nodesets=True, fuse_folds=False)
    assert fu.nodesets.n_fused > 0 and len(fu.multi_host) < len(un.multi_host)
    fu.launch()
    d1, e1 = fu.collect()
    un.launch()
    d2, e2 = un.collect()
    assert np.array_equal(d1, d2) and np.array_equal(e1, e2)
    assert np.isfinite(d1).all() and np.abs(e1).max() > 0


def test_chunked_wave_upload_gives_the_same_integrals():
    """A batch whose waves are rows of one pinned host matrix goes to the device in parts on a copy
    stream, and the fused node sets of each part start as soon as it has arrived (their launch
    order changes). The integrals must be bit-identical to those of the same waves from pageable
    memory (one synchronous upload, sets in their planned order) and repeatable."""
    from dwba_b200.dwba_matrix_elements import GPUCache, radial_ME_all_L_batch
    from dwba_b200 import engine
    g, z, bounds, pairs_pinned = bench.make_workload(N=3001, n_cont=96, n_bound=3, seed_shift=31, pinned=True)
    _, _, _, pairs_plain = bench.make_workload(N=3001, n_cont=96, n_bound=3, seed_shift=31, pinned=False)
    b_i, b_f = [b[0] for b in bounds], [b[1] for b in bounds]
    cache = GPUCache.from_grid(g)
    seen = []
    orig = engine.NodeSetBatch.reorder_fused

    def spy(self, perm, groups):
        seen.append(len(groups))
        return orig(self, perm, groups)
    engine.NodeSetBatch.reorder_fused = spy
    try:
        res = []
        for pairs in (pairs_pinned, pairs_plain, pairs_pinned):
            cache.clear()
            res.append(radial_ME_all_L_batch(g, z, z, b_i, b_f, pairs, 6, U_f_array=z, gpu_cache=cache,
                                             engine="semisep", as_arrays=True))
    finally:
        engine.NodeSetBatch.reorder_fused = orig
    assert seen and max(seen) > 1, "the pinned batch was not uploaded in parts"
    for d, e in res[1:]:
        assert np.array_equal(d, res[0][0]) and np.array_equal(e, res[0][1])
    assert np.isfinite(res[0][0]).all() and np.abs(res[0][1]).max() > 0


@pytest.mark.parametrize("kind", ["log", "coulomb"])
def test_result_objects_with_direct_rows_first_match_the_arrays(kind, monkeypatch):
    """Returning result objects, the batch entry point copies the direct rows (dot forms and device
    tails) back before the exchange forms run and fills their dicts meanwhile; every value must equal
    the as_arrays call's (which collects everything at the end), including the tails' contribution."""
    from dwba_b200 import dwba_matrix_elements as dme
    from dwba_b200.dwba_matrix_elements import GPUCache, RadialDWBAIntegrals, radial_ME_all_L_batch
    monkeypatch.setattr(dme, "EARLY_DIRECT_MIN_FORMS", 1)  # the small Coulomb batch (with tails) too
    g, V, U, bounds, pairs = _inputs(kind)
    cache = GPUCache.from_grid(g)
    b_i, b_f = [b[0] for b in bounds], [b[1] for b in bounds]
    I_d, I_e = radial_ME_all_L_batch(g, V, U, b_i, b_f, pairs, 6, U_f_array=U, gpu_cache=cache, engine="semisep",
                                     as_arrays=True)
    res = radial_ME_all_L_batch(g, V, U, b_i, b_f, pairs, 6, U_f_array=U, gpu_cache=cache, engine="semisep")
    assert len(res) == len(bounds) and all(len(r) == len(pairs) for r in res)
    for t, row in enumerate(res):
        for p, x in enumerate(row):
            assert type(x) is RadialDWBAIntegrals
            assert [x.I_L_direct[L] for L in range(7)] == I_d[t, p].tolist()
            assert [x.I_L_exchange[L] for L in range(7)] == I_e[t, p].tolist()
