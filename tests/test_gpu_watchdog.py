"""The bounded waits of the tensor-core kernels, made to run out on a normal input.

Every mbarrier wait of the split-BF16 pipeline (tc_gemm.cu) is bounded; dwba_tc_set_wait_cycles
sets that bound for the next launches. With a bound of a few clock cycles the pipeline's waits
expire on an ordinary small batch: the call must report status 2 through its status word (the
engine raises DWBAError), each CTA must drain its own copies and products and free its tensor
memory, and the next call with the default bound must run normally and give the same values as
before. Nothing here faults or hangs the GPU: the expired waits return, and the drain keeps its
own default bound of about a second.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _job(N=2001, n_pairs=24, L_max=4):
    import bench
    from dwba_b200.dwba_matrix_elements import GPUCache, _make_job
    g, z, bounds, pairs = bench.make_workload(N=N, n_cont=n_pairs, n_bound=1, seed_shift=77)
    cache = GPUCache.from_grid(g)
    job = _make_job(g, z, z, bounds[0][0], bounds[0][1], pairs, L_max, z, {}, cache)
    return job, cache


def _run(job, cache, engine="tc_bf16x3"):
    from dwba_b200.engine import PreparedJob
    pj = PreparedJob(job, cache.dg, engine)
    pj.launch()
    return pj.collect()


@pytest.mark.parametrize("engine", ["tc_bf16x3", "tc_bf16x6"])
def test_expired_waits_report_status_and_next_call_runs(engine):
    import torch
    from dwba_b200 import _lib
    lib = _lib.load()
    job, cache = _job()
    ref_d, ref_e = _run(job, cache, engine)
    try:
        assert lib.dwba_tc_set_wait_cycles(1) == _lib.DWBA_OK
        with pytest.raises(_lib.DWBAError, match="bounded wait"):
            _run(job, cache, engine)
    finally:
        assert lib.dwba_tc_set_wait_cycles(0) == _lib.DWBA_OK
    torch.cuda.synchronize()
    d, e = _run(job, cache, engine)
    assert np.array_equal(d, ref_d) and np.array_equal(e, ref_e)
    assert lib.dwba_tc_set_wait_cycles(-1) == _lib.DWBA_ERR_INVALID_ARG


def test_expired_waits_in_the_backward():
    """The backward kernel shares the pipeline: an expired wait sets its status word to 2 and the
    next backward call with the default bound gives the same gradients as before."""
    import torch
    from dwba_b200 import _lib
    from dwba_b200.engine import _ptr, _stream
    lib = _lib.load()
    job, cache = _job(N=1501, n_pairs=8, L_max=3)
    dev = cache.dg.device
    N, nl, n = job.grid.N, job.L_max + 1, len(job.pairs)
    rng = np.random.default_rng(5)
    a = torch.tensor(rng.normal(size=(n, N)), device=dev)
    b = torch.tensor(rng.normal(size=(n, N)), device=dev)
    grad = torch.tensor(rng.normal(size=(n, nl)), device=dev)
    ga, gb = torch.zeros_like(a), torch.zeros_like(b)
    rec = np.zeros(n, dtype=_lib.FORM_GRAD_DTYPE)
    rec["r"] = _ptr(cache.dg.r)
    rec["a"] = _ptr(a) + 8 * N * np.arange(n, dtype=np.uint64)
    rec["b"] = _ptr(b) + 8 * N * np.arange(n, dtype=np.uint64)
    rec["ga"] = _ptr(ga) + 8 * N * np.arange(n, dtype=np.uint64)
    rec["gb"] = _ptr(gb) + 8 * N * np.arange(n, dtype=np.uint64)
    rec["n_rows"] = rec["n_cols"] = N
    rec_d = torch.from_numpy(rec.view(np.uint8).copy()).to(dev)
    ds = np.array([(1.0 - 1e-12) ** L for L in range(nl)])
    ws_bytes = int(lib.dwba_tc_backward_workspace_bytes(n, N, job.L_max, 2))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)

    def call():
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        _lib.check(lib.dwba_bilinear_tc_bf16_backward(_ptr(rec_d), n, _ptr(cache.dg.r), N, job.L_max, 2,
                                                      ds.ctypes.data, _ptr(grad), _ptr(ws), ws_bytes,
                                                      _ptr(status), _stream()), "dwba_bilinear_tc_bf16_backward")
        torch.cuda.synchronize()
        return int(status.item()), ga.clone(), gb.clone()
    st0, ga0, gb0 = call()
    assert st0 == 0
    try:
        lib.dwba_tc_set_wait_cycles(1)
        st1, _, _ = call()
    finally:
        lib.dwba_tc_set_wait_cycles(0)
    assert st1 == 2
    st2, ga2, gb2 = call()
    assert st2 == 0 and torch.equal(ga2, ga0) and torch.equal(gb2, gb0)
