"""Host packing of a batch's waves (the C extension dwba_b200._hostpack) against the Python path.

pack_pairs reads every wave's scalars and numbers its chi array in one pass; the planner and the
upload then use arrays instead of walking the wave objects. The packed scalars and rows must equal
what the general Python path computes, a wave that does not qualify (chi not exactly N float64
values in C order, a missing l / k_au) must send the whole call to the general path, and the rows of
a batch's chi matrix must be grouped into one transfer by address arithmetic.
"""
import numpy as np
import pytest
import torch

import bench
from dwba_b200 import _hostpack
from dwba_b200.dwba_matrix_elements import _pack
from dwba_b200.engine import WaveMatrix, _pair_arrays


def test_packed_scalars_and_rows_match_the_python_path():
    g, z, bounds, pairs = bench.make_workload(N=501, n_cont=40, n_bound=1, seed_shift=3)
    pairs = pairs + [pairs[3], (pairs[5][0], pairs[7][1])]  # repeated wave objects share rows
    pk = _pack(pairs, 501)
    assert pk is not None
    pa = _pair_arrays(pairs)
    for j, k in enumerate(("k_i", "l_i", "im_i", "e_i", "d_i", "s_i", "k_f", "l_f", "im_f", "e_f", "d_f", "s_f")):
        assert np.array_equal(pk.scalars[:, j], pa[k].astype(np.float64)), k
    w = WaveMatrix(501)
    rows_i, rows_f = [], []
    for ci, cf in pairs:  # numbered pair by pair, cont_i before cont_f
        rows_i.append(w.add(ci.chi_of_r))
        rows_f.append(w.add(cf.chi_of_r))
    assert list(pk.rows_i) == rows_i and list(pk.rows_f) == rows_f
    assert len(pk.arrays) == len(w.arrays) and all(a is b for a, b in zip(pk.arrays, w.arrays))
    assert list(pk.ptrs) == [a.__array_interface__["data"][0] for a in pk.arrays]


@pytest.mark.parametrize("bad", ["float32", "short", "strided", "no_l", "list"])
def test_waves_that_do_not_qualify_take_the_general_path(bad):
    g, z, bounds, pairs = bench.make_workload(N=301, n_cont=6, n_bound=1, seed_shift=4)
    w = pairs[2][1]
    if bad == "float32":
        w.chi_of_r = w.chi_of_r.astype(np.float32)
    elif bad == "short":
        w.chi_of_r = w.chi_of_r[:300]
    elif bad == "strided":
        w.chi_of_r = np.repeat(w.chi_of_r, 2)[::2]
    elif bad == "no_l":
        del w.l
    else:
        w.chi_of_r = list(w.chi_of_r)
    assert _hostpack.pack_pairs(pairs, 301, np.ndarray) is None


def test_upload_groups_packed_rows_by_address():
    """The chi matrix behind a batch's waves goes as one gather; the rows match the arrays."""
    g, z, bounds, pairs = bench.make_workload(N=257, n_cont=30, n_bound=2, seed_shift=6)
    pk = _pack(pairs, 257)
    w = WaveMatrix(257)
    pk.first, pk.owner = w.add_distinct(pk.arrays, pk.ptrs), w
    for b in bounds:
        w.add(b[0].u_of_r)
        w.add(b[1].u_of_r)
    out = w.upload(torch.device("cpu")).numpy()
    for i, a in enumerate(w.arrays):
        assert np.array_equal(out[i], a)


def test_result_objects_match_the_python_path():
    """make_results + fill_results give the same RadialDWBAIntegrals (frozen, {L: float} dicts in L
    order) as constructing them in Python, and reject arrays of the wrong size."""
    import dataclasses
    from dwba_b200 import dwba_matrix_elements as dme
    rng = np.random.default_rng(12)
    for T, P, nl in ((1, 1, 1), (3, 17, 9), (2, 5, 300)):
        I_d, I_e = rng.standard_normal((T, P, nl)), rng.standard_normal((T, P, nl))
        fast = dme._results(I_d, I_e, dme._skeleton(T, P, nl))
        ref = [[dme.RadialDWBAIntegrals(I_L_direct={L: float(I_d[t, p, L]) for L in range(nl)},
                                        I_L_exchange={L: float(I_e[t, p, L]) for L in range(nl)})
                for p in range(P)] for t in range(T)]
        assert fast == ref
        x = fast[-1][-1]
        assert type(x) is dme.RadialDWBAIntegrals and list(x.I_L_direct) == list(range(nl))
        assert all(type(v) is float for v in x.I_L_exchange.values())
        with pytest.raises(dataclasses.FrozenInstanceError):
            x.I_L_direct = {}
    # the direct and the exchange halves filled separately (direct rows first, as the batch entry
    # point does while the exchange forms still run) give the same objects
    I_d, I_e = rng.standard_normal((2, 5, 9)), rng.standard_normal((2, 5, 9))
    res, dicts = dme._skeleton(2, 5, 9)
    _hostpack.fill_half(dicts, I_d, 9, 0)
    _hostpack.fill_half(dicts, I_e, 9, 1)
    assert res == dme._results(I_d, I_e)
    with pytest.raises(ValueError):
        _hostpack.fill_half(dicts, I_d, 9, 2)
    with pytest.raises(ValueError):
        _hostpack.fill_half(dicts, I_d[:1], 9, 0)
    _, dicts = dme._skeleton(2, 3, 4)
    with pytest.raises(ValueError):
        _hostpack.fill_results(dicts, np.zeros(2 * 3 * 4 - 1), np.zeros(2 * 3 * 4), 4)
    with pytest.raises(ValueError):
        _hostpack.fill_results(dicts, np.zeros(24, dtype=np.float32), np.zeros(24), 4)


def test_prestaged_block_is_taken_only_for_its_exact_rows():
    """A wave copy started before packing (engine.prestage_waves) is used only when the packed waves
    are exactly the block's rows, in order; chunk_of maps rows to the parts of such an upload."""
    from dwba_b200.engine import Prestaged
    g, z, bounds, pairs = bench.make_workload(N=129, n_cont=10, n_bound=1, seed_shift=8)
    base = pairs[0][0].chi_of_r.base
    bp, rb = base.__array_interface__["data"][0], 8 * 129
    pre = Prestaged(torch.empty((20 + 2, 129), dtype=torch.float64), bp, rb, 0, 20, [])
    pk = _pack(pairs, 129)
    w = WaveMatrix(129)
    pk.first, pk.owner = w.add_distinct(pk.arrays, pk.ptrs), w
    assert w._takes(pre)
    assert not w._takes(pre._replace(base_ptr=bp + rb))  # the block one row off
    assert not w._takes(pre._replace(n=19))
    shuffled = pairs[1:] + pairs[:1]
    pk2 = _pack(shuffled, 129)
    w2 = WaveMatrix(129)
    pk2.first, pk2.owner = w2.add_distinct(pk2.arrays, pk2.ptrs), w2
    assert not w2._takes(pre)
    w.chunks = [(0, 8, None), (8, 20, None)]
    assert list(w.chunk_of(np.array([0, 7, 8, 19, 20, 21]))) == [0, 0, 1, 1, 2, 2]
    w.chunks = None
    assert list(w.chunk_of(np.array([3, 30]))) == [0, 0]
