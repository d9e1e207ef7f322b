"""Large batches on the exact engines are planned and launched in chunks (the host plans chunk k+1
while the kernels of chunk k run); every integral depends on its own pair only, so the chunked call
must return exactly the unchunked one, for the semiseparable and the plain FP64 engines, with the
reference's result objects and as arrays, and with pairs that share a wave object across chunks."""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("engine", ["semisep", "dense"])
def test_chunked_batch_equals_one_call(engine, monkeypatch):
    from dwba_b200 import dwba_matrix_elements as dm
    g, z, bounds, pairs = bench.make_workload(N=2001, n_cont=150, n_bound=2, seed_shift=31, pinned=True)
    pairs = pairs + [(pairs[0][0], pairs[140][1]), pairs[7]]  # shared waves across chunks
    b_i, b_f = [b[0] for b in bounds], [b[1] for b in bounds]
    monkeypatch.setattr(dm, "PIPELINE_PAIRS", 10 ** 9)
    d1, e1 = dm.radial_ME_all_L_batch(g, z, z, b_i, b_f, pairs, 6, U_f_array=z, engine=engine, as_arrays=True)
    monkeypatch.setattr(dm, "PIPELINE_PAIRS", 48)
    d2, e2 = dm.radial_ME_all_L_batch(g, z, z, b_i, b_f, pairs, 6, U_f_array=z, engine=engine, as_arrays=True)
    assert np.array_equal(d1, d2) and np.array_equal(e1, e2)
    res = dm.radial_ME_all_L_batch(g, z, z, b_i, b_f, pairs, 6, U_f_array=z, engine=engine)
    for t in range(len(b_i)):
        for p in (0, 47, 48, 151):
            assert [res[t][p].I_L_direct[L] for L in range(7)] == list(d1[t, p])
            assert [res[t][p].I_L_exchange[L] for L in range(7)] == list(e1[t, p])
