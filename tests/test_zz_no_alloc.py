"""The allocation-free entry point against the regular dense FP64 entry point.

``dwba_bilinear_dense_fp64_noalloc`` exists for callers whose device memory is
owned by another allocator, or whose loop must not call cudaMalloc/cudaFree:
they pass only inputs and the output, and the library keeps its partial sums
in a fixed array of its own. This test builds the forms of one energy point,
evaluates them once with the regular entry point (caller-provided scratch),
then twice in a row with the allocation-free one through the C ABI, and checks
both calls against the first within the parity tolerance of the other GPU
tests. It lives in its own file, named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import golden_cases as gc

pytestmark = pytest.mark.gpu


def _prepared_job():
    import torch
    from dwba_b200.dwba_matrix_elements import GPUCache, _make_job
    from dwba_b200.engine import PreparedJob
    common, calls = gc.load_case("h_1s2p_50eV")
    adv = [c for c in calls if not c["kwargs"].keys() - {"U_f_array"}]
    grid = common["grid"]
    cache = GPUCache.from_grid(grid)
    pairs = [(c["args"][5], c["args"][6]) for c in adv]
    a = adv[0]["args"]
    job = _make_job(grid, a[1], a[2], a[3], a[4], pairs, 6, adv[0]["kwargs"]["U_f_array"], {}, cache)
    pj = PreparedJob(job, cache.dg, "dense")
    pj.nodesets.launch()
    pj.launch_folds()
    torch.cuda.synchronize()
    return pj


def test_noalloc_matches_dense_entry_point_twice():
    import torch
    from dwba_b200 import _lib
    lib = _lib.load()
    pj = _prepared_job()
    stream = torch.cuda.current_stream().cuda_stream
    # the regular entry point with caller-provided scratch
    pj.launch_forms()
    torch.cuda.synchronize()
    ref = pj.out.cpu().numpy().copy()
    m = np.maximum(pj.forms_host["n_rows"], pj.forms_host["n_cols"])
    max_m = int(m.max())
    scale = np.abs(ref) + 1e-300
    for attempt in range(2):
        out = torch.full_like(pj.out, float("nan"))
        rc = lib.dwba_bilinear_dense_fp64_noalloc(ctypes.c_void_p(pj.forms_d.data_ptr()), pj.n_forms, max_m,
                                                  pj.job.L_max, pj.ds.ctypes.data, ctypes.c_void_p(out.data_ptr()),
                                                  ctypes.c_void_p(stream))
        assert rc == _lib.DWBA_OK, _lib.status_string(rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), attempt
        assert np.all(np.abs(got - ref) <= 1e-12 * scale), (attempt, np.max(np.abs(got - ref) / scale))


def test_noalloc_rejects_requests_beyond_its_array():
    import torch
    from dwba_b200 import _lib
    lib = _lib.load()
    pj = _prepared_job()
    out = torch.empty_like(pj.out)
    stream = torch.cuda.current_stream().cuda_stream
    # 65535 forms of up to 10^6 points each need far more partials than the fixed array holds
    rc = lib.dwba_bilinear_dense_fp64_noalloc(ctypes.c_void_p(pj.forms_d.data_ptr()), 65535, 1_000_000,
                                              pj.job.L_max, pj.ds.ctypes.data, ctypes.c_void_p(out.data_ptr()),
                                              ctypes.c_void_p(stream))
    assert rc == _lib.DWBA_ERR_WORKSPACE
    rc = lib.dwba_bilinear_dense_fp64_noalloc(None, 1, 10, 4, pj.ds.ctypes.data, None, None)
    assert rc == _lib.DWBA_ERR_INVALID_ARG
