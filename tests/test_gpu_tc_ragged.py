"""The ragged split-BF16 launch: forms on several grids in one tensor-core launch.

dwba_bilinear_tc_bf16_ragged takes one segment per grid (its forms, grid and result rows) and
runs all of them in one launch of the tensor-core kernel, segments largest grid first, with a
tile chosen at run time (forms per CTA 128 or 256, pipeline depth, CTA order). Every CTA works on
one (row block, form block, multipole) of one segment exactly as in a single-grid launch, so each
segment's results must be bit-identical to dwba_bilinear_tc_bf16 on that segment alone, for every
tile and both splits. Through the sweep entry point, the tile tuner (tile="auto") must time every
valid tile (median of repeated launches), record its choice, and give the same results as the
default tile.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _segments(rng, dev):
    import torch
    from dwba_b200 import _lib
    from dwba_b200.engine import _ptr
    segs = []
    for N, nf in ((1501, 300), (4001, 520), (2600, 64), (1024, 1)):
        r = np.geomspace(1e-4, 60.0, N)
        x = rng.normal(size=(2, nf, N))
        env = np.exp(-r / rng.uniform(2.0, 20.0, size=(2, nf, 1)))
        a = torch.tensor(x[0] * env[0], device=dev)
        b = torch.tensor(x[1] * env[1] * np.sin(rng.uniform(0.5, 4.0, size=(nf, 1)) * r), device=dev)
        r_d = torch.tensor(r, device=dev)
        f = np.zeros(nf, dtype=_lib.FORM_DTYPE)
        f["r"] = _ptr(r_d)
        f["a"] = _ptr(a) + 8 * N * np.arange(nf, dtype=np.uint64)
        f["b"] = _ptr(b) + 8 * N * np.arange(nf, dtype=np.uint64)
        f["n_rows"] = rng.integers(N // 2, N + 1, size=nf)
        f["n_cols"] = N
        segs.append(dict(N=N, nf=nf, r=r_d, a=a, b=b, forms=torch.from_numpy(f.view(np.uint8).copy()).to(dev)))
    return segs


@pytest.mark.parametrize("nt", [2, 3])
def test_ragged_launch_matches_single_grid_launches_for_every_tile(nt):
    import torch
    from dwba_b200 import _lib, tune
    from dwba_b200.engine import _ptr, _stream
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(40 + nt)
    segs = _segments(rng, dev)
    L_max = 6
    nl = L_max + 1
    ds = np.array([(1.0 - 1e-12) ** L for L in range(nl)])
    # single-grid launches
    ref = []
    for sg in segs:
        ws = torch.empty(int(lib.dwba_tc_workspace_bytes(sg["nf"], sg["N"], L_max, nt)), dtype=torch.uint8, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        out = torch.empty((sg["nf"], nl), dtype=torch.float64, device=dev)
        _lib.check(lib.dwba_bilinear_tc_bf16(_ptr(sg["forms"]), sg["nf"], _ptr(sg["r"]), sg["N"], L_max, nt,
                                             ds.ctypes.data, _ptr(ws), ws.numel(), _ptr(status), _ptr(out), _stream()),
                   "dwba_bilinear_tc_bf16")
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        ref.append(out.cpu().numpy())
    # one ragged launch per tile
    outs = [torch.empty((sg["nf"], nl), dtype=torch.float64, device=dev) for sg in segs]
    rec = np.zeros(len(segs), dtype=_lib.TC_SEGMENT_DTYPE)
    for q, (sg, o) in enumerate(zip(segs, outs)):
        rec[q] = (_ptr(sg["forms"]), _ptr(sg["r"]), _ptr(o), sg["nf"], sg["N"])
    for tile in tune.TILES[nt]:
        t = np.zeros(1, dtype=_lib.TC_TILE_DTYPE)
        t["bn"], t["stages"], t["order"] = tile["bn"], tile["stages"], tile["order"]
        nbytes = int(lib.dwba_tc_ragged_workspace_bytes(rec.ctypes.data, len(rec), L_max, nt, t.ctypes.data))
        assert nbytes > 0
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        for o in outs:
            o.fill_(float("nan"))
        _lib.check(lib.dwba_bilinear_tc_bf16_ragged(rec.ctypes.data, len(rec), L_max, nt, t.ctypes.data,
                                                    ds.ctypes.data, _ptr(ws), ws.numel(), _ptr(status), _stream()),
                   "dwba_bilinear_tc_bf16_ragged")
        torch.cuda.synchronize()
        assert int(status.item()) == 0, tile
        for q, (o, rf) in enumerate(zip(outs, ref)):
            assert np.array_equal(o.cpu().numpy(), rf), (tile, q)


def test_sweep_tile_tuner_records_its_choice():
    import bench
    from dwba_b200 import tune
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_sweep
    pts = bench.make_ragged_points(64, select=(0, 40))
    keys = ("grid", "V_core_array", "U_i_array", "bound_i", "bound_f", "pairs", "U_f_array")
    args = [{k: pt[k] for k in keys} for pt in pts]
    base = radial_ME_all_L_sweep(args, 6, engine="tc_bf16x3")
    tuned = radial_ME_all_L_sweep(args, 6, engine="tc_bf16x3", tile="auto", graph=True)
    for rb, rt in zip(base, tuned):
        for x, y in zip(rb, rt):
            assert x.I_L_direct == y.I_L_direct and x.I_L_exchange == y.I_L_exchange
    (key, tile), = [(k, v) for k, v in tune.TILE_TUNER.choices.items() if k[0] == 2]
    times = tune.TILE_TUNER.timings_ms[key]
    assert len(times) == len(tune.TILES[2]) and all(v > 0 for v in times.values())
    assert tune._tile_name(tile) == min(times, key=times.get)
