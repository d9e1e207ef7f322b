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


def _forms_dense(pj, idx, L_max):
    """The regular dense entry point on the forms idx (a fresh descriptor array), L = 0..L_max."""
    import torch
    from dwba_b200 import _lib
    lib = _lib.load()
    f = np.ascontiguousarray(pj.forms_host[idx])
    fd = torch.from_numpy(f.view(np.uint8).copy()).cuda()
    m = np.maximum(f["n_rows"], f["n_cols"]).astype(np.int32)
    prefix = np.zeros(len(f) + 1, dtype=np.int64)
    n_cta = int(lib.dwba_dense_chunk_prefix(m.ctypes.data, len(f), prefix.ctypes.data))
    prefix_d = torch.from_numpy(prefix).cuda()
    part = torch.empty(n_cta * (L_max + 1), dtype=torch.float64, device="cuda")
    out = torch.empty((len(f), L_max + 1), dtype=torch.float64, device="cuda")
    ds = np.array([(1.0 - 1e-12) ** L for L in range(L_max + 1)])
    _lib.check(lib.dwba_bilinear_dense_fp64(fd.data_ptr(), len(f), L_max, ds.ctypes.data, prefix_d.data_ptr(), n_cta,
                                            part.data_ptr(), part.numel(), out.data_ptr(),
                                            torch.cuda.current_stream().cuda_stream), "dwba_bilinear_dense_fp64")
    torch.cuda.synchronize()
    return fd, out.cpu().numpy(), ds


def _noalloc(fd, n_forms, max_m, L_max, ds):
    import torch
    from dwba_b200 import _lib
    out = torch.full((n_forms, L_max + 1), float("nan"), dtype=torch.float64, device="cuda")
    rc = _lib.load().dwba_bilinear_dense_fp64_noalloc(ctypes.c_void_p(fd.data_ptr()), n_forms, max_m, L_max,
                                                      ds.ctypes.data, ctypes.c_void_p(out.data_ptr()),
                                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def test_noalloc_many_multipoles_in_two_passes():
    """L_max = 18: the multipoles go in two launches (0..15, 16..18); both calls in a row equal the
    regular entry point."""
    from dwba_b200 import _lib
    pj = _prepared_job()
    idx = np.arange(pj.n_forms)
    fd, ref, ds = _forms_dense(pj, idx, 18)
    max_m = int(np.max(np.maximum(pj.forms_host["n_rows"], pj.forms_host["n_cols"])))
    for _ in range(2):
        rc, got = _noalloc(fd, pj.n_forms, max_m, 18, ds)
        assert rc == _lib.DWBA_OK
        assert np.all(np.abs(got - ref) <= 1e-12 * (np.abs(ref) + 1e-300))


def test_noalloc_form_above_max_m_and_empty_form():
    """A form longer than max_m gets NaN in its row only; an empty form gets the empty sum 0."""
    import torch
    from dwba_b200 import _lib
    pj = _prepared_job()
    f = np.ascontiguousarray(pj.forms_host[:4]).copy()
    m = np.maximum(f["n_rows"], f["n_cols"])
    f["n_rows"][1] = f["n_cols"][1] = 0                 # empty form
    f["n_rows"][2] = min(int(f["n_rows"][2]), 100)      # short forms: within max_m
    f["n_cols"][2] = min(int(f["n_cols"][2]), 100)
    f["n_rows"][3] = min(int(f["n_rows"][3]), 120)
    f["n_cols"][3] = min(int(f["n_cols"][3]), 120)
    assert m[0] > 256
    fd = torch.from_numpy(f.view(np.uint8).copy()).cuda()
    ds = np.array([(1.0 - 1e-12) ** L for L in range(5)])
    rc, got = _noalloc(fd, 4, 128, 4, ds)   # max_m = 128 < M of form 0
    assert rc == _lib.DWBA_OK
    assert np.all(np.isnan(got[0])) and np.all(got[1] == 0.0)
    assert np.all(np.isfinite(got[2:]))
    pj.forms_host = f
    _, ref, _ = _forms_dense(pj, np.array([2, 3]), 4)
    assert np.all(np.abs(got[2:] - ref) <= 1e-12 * (np.abs(ref) + 1e-300))


def test_noalloc_request_exactly_at_the_array_size():
    """n_forms * ceil(ceil(max_m/128)/2) * (L_max+1) == DWBA_NOALLOC_SCRATCH_DOUBLES is accepted and
    gives the regular entry point's values; one form more is rejected."""
    from dwba_b200 import _lib
    pj = _prepared_job()
    L_max, max_m = 15, 128 * 128           # 16 multipoles x 64 chunks per form
    n_forms = (1 << 20) // (16 * 64)       # 1024 forms
    idx = np.arange(n_forms) % pj.n_forms  # the job's forms, repeated
    fd, ref, ds = _forms_dense(pj, idx, L_max)
    rc, got = _noalloc(fd, n_forms, max_m, L_max, ds)
    assert rc == _lib.DWBA_OK
    assert np.all(np.abs(got - ref) <= 1e-12 * (np.abs(ref) + 1e-300))
    fd2, _, _ = _forms_dense(pj, np.arange(n_forms + 1) % pj.n_forms, L_max)
    rc, _ = _noalloc(fd2, n_forms + 1, max_m, L_max, ds)
    assert rc == _lib.DWBA_ERR_WORKSPACE
