"""Drop-in replacement for the reference module ``dwba_matrix_elements``.

Same names, call signatures and result layout as the reference
(``dwba_matrix_elements.py``: ``radial_ME_all_L`` :780, ``radial_ME_all_L_gpu``
:1563, ``RadialDWBAIntegrals`` :670, ``GPUCache`` :203, ``HAS_CUPY`` :73-77,
``check_cupy_runtime`` :178, ``OscillatoryMethod`` :70), so ``driver.py`` and
``ionization.py`` import it unchanged::

    from dwba_b200.dwba_matrix_elements import (radial_ME_all_L, radial_ME_all_L_gpu,
                                                HAS_CUPY, check_cupy_runtime, GPUCache)

Both entry points evaluate the reference's CPU quadrature semantics on the
GPU (sm_100a kernels behind ``libdwba_b200.so``); there is no CPU fallback, so
without a usable GPU they raise ``RuntimeError`` like the reference's GPU path
does without CuPy. ``radial_ME_all_L_batch`` is the added batched entry point:
all (l_i, l_f) pairs of one energy point in one set of launches. The GPU and
batched entry points take ``semantics="cupy"`` for the quadrature of the
reference's CuPy function instead (``cupy_mode.py``).

Engine selection: ``DWBA_B200_ENGINE`` = ``dense`` (default; the plain FP64
form that generates every kernel element) or ``semisep`` (exact FP64 O(N L)
evaluation of the same bilinear forms).
"""
from __future__ import annotations

import os
from collections import OrderedDict
from dataclasses import dataclass
from typing import Dict, List, Literal, Optional, Sequence, Tuple, Union

import numpy as np

from . import _lib

try:  # host packing of a batch's waves (csrc/hostpack.c); the general Python path works without it
    from . import _hostpack
except ImportError:  # pragma: no cover - only when the extension was not built
    _hostpack = None

OscillatoryMethod = Literal["legacy", "advanced", "full_split"]
EARLY_DIRECT_MIN_FORMS = 256  # (transition, pair) count from which results come back in two parts
SEMANTICS = ("cpu", "cupy")

try:
    _lib.load()
    HAS_CUPY = True  # the GPU engine is importable (the reference's flag name is kept for its callers)
except ImportError:  # pragma: no cover - exercised only when the library was not built
    HAS_CUPY = False


@dataclass(frozen=True)
class RadialDWBAIntegrals:
    """I_L_direct / I_L_exchange: ``{L: float}`` for L = 0..L_max (``dwba_matrix_elements.py:670-685``)."""
    I_L_direct: Dict[int, float]
    I_L_exchange: Dict[int, float]


def check_cupy_runtime() -> bool:
    """True when the engine can run: library loaded, torch sees a CUDA device, and it is sm_100."""
    if not HAS_CUPY:
        return False
    try:
        import torch
        if not torch.cuda.is_available():
            return False
        return _lib.device_ok()
    except Exception as e:  # pragma: no cover
        print(f"[Warning] GPU initialization failed: {e}")
        return False


ENGINE_NAMES = ("dense", "semisep", "tc_bf16x3", "tc_bf16x6", "auto", "auto_split")


def _engine_name(engine: Optional[str]) -> str:
    """Engine of a call: the argument, else DWBA_B200_ENGINE, else the plain FP64 kernel. ``auto``
    times the FP64 engines per shape class and keeps the fastest; ``auto_split`` also admits the
    split-BF16 tensor-core form."""
    e = engine or os.environ.get("DWBA_B200_ENGINE", "dense")
    if e not in ENGINE_NAMES:
        raise ValueError(f"unknown engine {e!r} ({' | '.join(ENGINE_NAMES)})")
    return e


class GPUCache:
    """Energy-level device cache (grid arrays and quadrature node sets); ``dwba_matrix_elements.py:203-615``.

    ``GPUCache.from_grid(grid, max_chi_cached=20)`` builds it; ``clear()`` releases it.
    """

    def __init__(self, grid, max_chi_cached: int = 20, device=None):
        import torch
        from .engine import DeviceGrid
        from .plan import GridInfo
        if not torch.cuda.is_available():
            raise RuntimeError("GPUCache requires a CUDA device")
        self.grid = grid
        self.max_chi_cached = int(max_chi_cached)
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.info = GridInfo(grid.r, grid.w_simpson, getattr(grid, "w_trapz", None)
                             if getattr(grid, "w_trapz", None) is not None else np.gradient(grid.r))
        self.dg = DeviceGrid(self.info, self.device)

    @classmethod
    def from_grid(cls, grid, max_chi_cached: int = 20) -> "GPUCache":
        return cls(grid, max_chi_cached=max_chi_cached)

    def matches(self, grid) -> bool:
        r = np.asarray(grid.r)
        return len(r) == self.info.N and (r is self.grid.r or np.array_equal(r, self.info.r))

    def clear(self) -> None:
        self.dg.nodesets.clear()


_GRID_CACHE: "OrderedDict[tuple, GPUCache]" = OrderedDict()


def _grid_key(grid):
    r = np.asarray(grid.r)
    w = np.asarray(grid.w_simpson)
    return (r.__array_interface__["data"][0], w.__array_interface__["data"][0], len(r), float(r[0]), float(r[-1]))


def _cache_for(grid, gpu_cache: Optional[GPUCache]) -> GPUCache:
    if gpu_cache is not None and gpu_cache.matches(grid):
        return gpu_cache
    key = _grid_key(grid)
    c = _GRID_CACHE.get(key)
    if c is None:
        c = GPUCache(grid)
        _GRID_CACHE[key] = c
        while len(_GRID_CACHE) > 4:
            _GRID_CACHE.popitem(last=False)
    else:
        _GRID_CACHE.move_to_end(key)
    return c


def _fit(arr, N, what):
    """Length check of the reference's GPU path (dwba_matrix_elements.py:1637-1672, :1754-1783)."""
    a = np.asarray(arr, dtype=np.float64)
    if len(a) > N:
        return a[:N]
    if len(a) < N:
        raise ValueError(f"{what} has {len(a)} pts but grid has {N}")
    return a


class _WaveView:
    """A continuum wave with chi truncated to the grid (attributes as the reference's ContinuumWave)."""

    __slots__ = ("l", "k_au", "chi_of_r", "phase_shift", "idx_match", "eta", "sigma_l")

    def __init__(self, w, N, what):
        self.l = int(w.l)
        self.k_au = float(w.k_au)
        self.chi_of_r = _fit(w.chi_of_r, N, what)
        self.phase_shift = float(getattr(w, "phase_shift", 0.0))
        self.idx_match = int(getattr(w, "idx_match", -1))
        self.eta = float(getattr(w, "eta", 0.0))
        self.sigma_l = float(getattr(w, "sigma_l", 0.0))


class _Packed:
    """A batch's waves packed in one pass by the host extension: scalars (P x 12), the rows of each
    pair's two chi arrays among the distinct ones (``arrays``, pair by pair) and, once they are in a
    WaveMatrix (``owner``), the row of the first (``first``)."""
    __slots__ = ("scalars", "rows_i", "rows_f", "arrays", "ptrs", "first", "owner")

    def __init__(self, scalars, rows_i, rows_f, arrays, ptrs):
        self.scalars, self.rows_i, self.rows_f, self.arrays = scalars, rows_i, rows_f, arrays
        self.ptrs = np.asarray(ptrs, dtype=np.int64)
        self.first, self.owner = None, None


def _pack(pairs, N):
    """_Packed for the pairs, or None when a wave needs the general path (or the extension is absent)."""
    if _hostpack is None or len(pairs) == 0:
        return None
    res = _hostpack.pack_pairs(pairs, int(N), np.ndarray)
    if res is None:
        return None
    scal, ri, rf, arrays, ptrs = res
    return _Packed(np.frombuffer(scal, dtype=np.float64).reshape(-1, 12), np.frombuffer(ri, dtype=np.int64),
                   np.frombuffer(rf, dtype=np.int64), arrays, ptrs)


def _make_job(grid, V_core_array, U_i_array, bound_i, bound_f, pairs, L_max, U_f_array, kw, cache):
    """Job for one or several transitions: bound_i/bound_f are single objects or equal-length sequences."""
    from .engine import Job, Transition
    from .plan import is_excitation
    if L_max < 0:
        raise ValueError("radial_ME_all_L: L_max must be >= 0.")
    N = cache.info.N
    V = _fit(V_core_array, N, "V_core")
    Ui = _fit(U_i_array, N, "U_i")
    Uf = _fit(U_f_array, N, "U_f") if U_f_array is not None else None
    bis = list(bound_i) if isinstance(bound_i, (list, tuple)) else [bound_i]
    bfs = list(bound_f) if isinstance(bound_f, (list, tuple)) else [bound_f]
    if len(bis) != len(bfs):
        raise ValueError("bound_i and bound_f must have the same number of transitions")
    trans = [Transition(u_i=_fit(bi.u_of_r, N, "Bound state u_i"), u_f=_fit(bf.u_of_r, N, "u_f"),
                        excitation=is_excitation(bf)) for bi, bf in zip(bis, bfs)]
    cache_w: Dict[int, object] = {}

    def view(w, what):
        # a wave whose chi is already N float64 values is used as it is; others get a truncated view
        v = cache_w.get(id(w))
        if v is None:
            chi = getattr(w, "chi_of_r", None)
            ok = (type(chi) is np.ndarray and chi.dtype == np.float64 and chi.ndim == 1 and len(chi) == N and
                  hasattr(w, "l") and hasattr(w, "k_au"))
            v = cache_w[id(w)] = w if ok else _WaveView(w, N, what)
        return v
    packed = _pack(pairs, N)
    if packed is not None:
        wp = [(ci, cf) for ci, cf in pairs]  # every wave qualifies as it is
    else:
        wp = [(view(ci, "cont_i.chi"), view(cf, "cont_f.chi")) for ci, cf in pairs]
    meth = kw.get("oscillatory_method", "advanced")
    if meth not in ("legacy", "advanced", "full_split"):
        meth = "advanced"  # the reference treats any other value as "advanced" (dwba_matrix_elements.py:1183)
    job = Job(grid=cache.info, V_core=V, U_i=Ui, U_f=Uf, transitions=trans, pairs=wp, L_max=int(L_max),
               use_oscillatory_quadrature=bool(kw.get("use_oscillatory_quadrature", True)),
               oscillatory_method=meth, CC_nodes=int(kw.get("CC_nodes", 5)),
               phase_increment=float(kw.get("phase_increment", 1.5708)),
               min_grid_fraction=float(kw.get("min_grid_fraction", 0.10)),
               k_threshold=float(kw.get("k_threshold", 0.5)),
               tails_on_device=os.environ.get("DWBA_B200_TAILS", "device").strip().lower() != "host")
    job._packed = packed
    return job


def _no_gc(fn):
    """Run ``fn`` with the cyclic garbage collector paused (a call allocates many small host
    objects -- descriptors, keys, result dicts -- none of which form cycles), restoring its state."""
    import functools
    import gc

    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        enabled = gc.isenabled()
        gc.disable()
        try:
            return fn(*args, **kwargs)
        finally:
            if enabled:
                gc.enable()
    return wrapper


def _early_upload(job, device, prestaged=None):
    """The job's functions (continuum waves, bound pairs) as rows of one device matrix, copied before
    the host planning so that a copy from pinned memory overlaps it; planning and preparation then
    find them uploaded. ``prestaged``: a copy of the waves started before the job was made
    (engine.prestage_waves), used when the packed waves turn out to be exactly its rows."""
    from .engine import WaveMatrix
    waves = WaveMatrix(job.grid.N)
    waves.prestaged = prestaged
    packed = getattr(job, "_packed", None)
    if packed is not None:
        packed.first, packed.owner = waves.add_distinct(packed.arrays, packed.ptrs), waves
    else:
        for ci, _ in job.pairs:
            waves.add(ci.chi_of_r)
        for _, cf in job.pairs:
            waves.add(cf.chi_of_r)
    for t in job.transitions:
        waves.add(t.u_i)
        waves.add(t.u_f)
    waves.upload(device, side_stream=True)  # the kernels' launch waits for it (WaveMatrix.wait_ready)
    return waves


def _skeleton(T: int, P: int, nl: int):
    """results[t][p] as RadialDWBAIntegrals whose dicts hold the keys 0..nl-1 and no values yet,
    with the list of those dicts, made while the device computes (None without the extension)."""
    if _hostpack is None:
        return None
    return _hostpack.make_results(RadialDWBAIntegrals, int(T), int(P), int(nl))


def _results(I_dir: np.ndarray, I_exc: np.ndarray, skeleton=None):
    """(T, P, L_max+1) arrays -> results[t][p] as RadialDWBAIntegrals of Python floats (the values
    filled into ``skeleton`` from _skeleton when given)."""
    T, P, nl = I_dir.shape
    if _hostpack is not None and I_exc.shape == I_dir.shape:
        res, dicts = skeleton if skeleton is not None else _skeleton(T, P, nl)
        _hostpack.fill_results(dicts, np.ascontiguousarray(I_dir, dtype=np.float64),
                               np.ascontiguousarray(I_exc, dtype=np.float64), nl)
        return res
    d, e = I_dir.tolist(), I_exc.tolist()
    return [[RadialDWBAIntegrals(I_L_direct=dict(enumerate(dp)), I_L_exchange=dict(enumerate(ep)))
             for dp, ep in zip(dt, et)] for dt, et in zip(d, e)]


@_no_gc
def _run(grid, V_core_array, U_i_array, bound_i, bound_f, pairs, L_max, U_f_array, kw, gpu_cache, engine,
         as_arrays: bool = False, semantics: str = "cpu"):
    """Evaluate a job; returns results[t][p] (a list of RadialDWBAIntegrals per transition), or
    the (T, P, L_max+1) arrays (I_dir, I_exc) with ``as_arrays``. ``semantics``: "cpu" for the
    quadrature of the reference's CPU path, "cupy" for that of its CuPy path (cupy_mode.py)."""
    if semantics not in SEMANTICS:
        raise ValueError(f"unknown semantics {semantics!r}; choose from {SEMANTICS}")
    if not HAS_CUPY:
        raise RuntimeError("dwba_b200 engine library is not available (build it with python -m dwba_b200.build)")
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("radial_ME_all_L: no CUDA device available (the B200 engine has no CPU fallback)")
    from .engine import PreparedJob, plan_job, prestage_waves
    from . import tune
    cache = _cache_for(grid, gpu_cache)
    eng = _engine_name(engine)
    with torch.cuda.device(cache.device):
        # the waves' copy starts before packing when they are rows of one pinned matrix
        n_bound = len(bound_i) if isinstance(bound_i, (list, tuple)) else 1
        pre = prestage_waves(pairs, cache.info.N, 2 * n_bound, cache.device) if semantics == "cpu" else None
        job = _make_job(grid, V_core_array, U_i_array, bound_i, bound_f, pairs, L_max, U_f_array, kw, cache)
        if semantics == "cupy":
            from .cupy_mode import CupyPreparedJob
            pj = CupyPreparedJob(job, cache.dg)
            pj.launch()
            I_dir, I_exc = pj.collect()
            return (I_dir, I_exc) if as_arrays else _results(I_dir, I_exc)
        plans = plan_job(job, _early_upload(job, cache.device, pre))
        if tune.is_auto(eng):
            cands = tune.candidates(eng)
            key = tune.TUNER.key(cache.info.N, 2 * len(job.transitions) * len(job.pairs), L_max, cands)
            _, pj = tune.TUNER.select(key, cands, lambda e: PreparedJob(job, cache.dg, e, plans=plans),
                                      lambda p: p.launch())
            pj.launch()
        else:
            # direct rows copied back first only where the fill of their dicts is worth overlapping
            early = not as_arrays and len(job.transitions) * len(job.pairs) >= EARLY_DIRECT_MIN_FORMS
            pj = PreparedJob(job, cache.dg, eng, plans=plans, early_direct=early, early_nodesets=True)
            pj.launch()
        # the result objects are made while the kernels run; collect() then waits for them
        skel = None if as_arrays else _skeleton(len(job.transitions), len(job.pairs), job.L_max + 1)
        if skel is not None and getattr(pj, "early_direct", None) is not None:
            # the direct integrals arrive before the exchange forms have run: their values are
            # filled in meanwhile
            _hostpack.fill_half(skel[1], pj.collect_direct(), job.L_max + 1, 0)
            I_dir, I_exc = pj.collect()
            _hostpack.fill_half(skel[1], np.ascontiguousarray(I_exc), job.L_max + 1, 1)
            return skel[0]
        I_dir, I_exc = pj.collect()
    if as_arrays:
        return I_dir, I_exc
    return _results(I_dir, I_exc, skel)


def radial_ME_all_L(grid, V_core_array, U_i_array, bound_i, bound_f, cont_i, cont_f, L_max: int,
                    use_oscillatory_quadrature: bool = True, oscillatory_method: OscillatoryMethod = "advanced",
                    CC_nodes: int = 5, phase_increment: float = 1.5708, min_grid_fraction: float = 0.10,
                    k_threshold: float = 0.5, U_f_array: Optional[np.ndarray] = None,
                    engine: Optional[str] = None) -> RadialDWBAIntegrals:
    """I_L^dir and I_L^exc for L = 0..L_max of one (cont_i, cont_f) pair (``dwba_matrix_elements.py:780``)."""
    kw = dict(use_oscillatory_quadrature=use_oscillatory_quadrature, oscillatory_method=oscillatory_method,
              CC_nodes=CC_nodes, phase_increment=phase_increment, min_grid_fraction=min_grid_fraction,
              k_threshold=k_threshold)
    return _run(grid, V_core_array, U_i_array, bound_i, bound_f, [(cont_i, cont_f)], L_max, U_f_array, kw, None,
                engine)[0][0]


def radial_ME_all_L_gpu(grid, V_core_array, U_i_array, bound_i, bound_f, cont_i, cont_f, L_max: int,
                        use_oscillatory_quadrature: bool = True, oscillatory_method: OscillatoryMethod = "advanced",
                        CC_nodes: int = 5, phase_increment: float = 1.5708, gpu_block_size=0,
                        min_grid_fraction: float = 0.10, k_threshold: float = 0.5, gpu_memory_mode: str = "auto",
                        gpu_memory_threshold: float = 0.8, gpu_cache: Optional[GPUCache] = None,
                        U_f_array: Optional[np.ndarray] = None, engine: Optional[str] = None,
                        semantics: str = "cpu") -> RadialDWBAIntegrals:
    """GPU signature of the reference (``dwba_matrix_elements.py:1563``). ``gpu_block_size``,
    ``gpu_memory_mode`` and ``gpu_memory_threshold`` are accepted for compatibility: kernel tiles are
    generated in registers, so device memory is O(N) per pair and no block-size policy is needed.

    ``semantics="cpu"`` (default) gives the values of the reference's CPU path ``radial_ME_all_L``,
    which its drivers use as ground truth; ``semantics="cupy"`` reproduces the quadrature of the
    reference's own GPU function (un-adapted phase step, linear interpolation on r[:idx_limit],
    kernel at the CC nodes, ungated L=0 corrections), evaluated exactly in FP64 (``engine`` is
    ignored there)."""
    kw = dict(use_oscillatory_quadrature=use_oscillatory_quadrature, oscillatory_method=oscillatory_method,
              CC_nodes=CC_nodes, phase_increment=phase_increment, min_grid_fraction=min_grid_fraction,
              k_threshold=k_threshold)
    return _run(grid, V_core_array, U_i_array, bound_i, bound_f, [(cont_i, cont_f)], L_max, U_f_array, kw,
                gpu_cache, engine, semantics=semantics)[0][0]


def radial_ME_all_L_batch(grid, V_core_array, U_i_array, bound_i, bound_f,
                          pairs: Sequence[Tuple[object, object]], L_max: int,
                          use_oscillatory_quadrature: bool = True, oscillatory_method: OscillatoryMethod = "advanced",
                          CC_nodes: int = 5, phase_increment: float = 1.5708, min_grid_fraction: float = 0.10,
                          k_threshold: float = 0.5, U_f_array: Optional[np.ndarray] = None,
                          gpu_cache: Optional[GPUCache] = None,
                          engine: Optional[str] = None, as_arrays: bool = False, semantics: str = "cpu"):
    """Batched entry point (new): the same values as calling ``radial_ME_all_L`` per pair.

    All pairs share one grid and the potentials. With single ``bound_i``/``bound_f`` objects the
    result is one ``RadialDWBAIntegrals`` per pair; with equal-length sequences of them (several
    transitions, e.g. one per ejected wave in ionization) it is a list per transition. With
    ``as_arrays=True`` the same values come as two float64 arrays (I_direct, I_exchange) of shape
    (P, L_max+1), or (T, P, L_max+1) for several transitions, without building a result object
    per pair. ``semantics`` as for ``radial_ME_all_L_gpu``."""
    kw = dict(use_oscillatory_quadrature=use_oscillatory_quadrature, oscillatory_method=oscillatory_method,
              CC_nodes=CC_nodes, phase_increment=phase_increment, min_grid_fraction=min_grid_fraction,
              k_threshold=k_threshold)
    multi = isinstance(bound_i, (list, tuple))
    if len(pairs) == 0:
        if as_arrays:
            shape = ((len(bound_i),) if multi else ()) + (0, L_max + 1)
            return np.zeros(shape), np.zeros(shape)
        return [[] for _ in bound_i] if multi else []
    res = _run(grid, V_core_array, U_i_array, bound_i, bound_f, list(pairs), L_max, U_f_array, kw, gpu_cache, engine,
               as_arrays=as_arrays, semantics=semantics)
    if as_arrays:
        return res if multi else (res[0][0], res[1][0])
    return res if multi else res[0]


@_no_gc
def radial_ME_all_L_sweep(points: Sequence[dict], L_max: int, engine: Optional[str] = None, graph: bool = False,
                          replays: int = 0, tile: Union[None, str, dict] = None, **options):
    """Many energy points in shared launches (new entry point; the reference loops over energies).

    ``points``: one dict per energy point with the arguments of ``radial_ME_all_L_batch``:
    ``grid``, ``V_core_array``, ``U_i_array``, ``bound_i``, ``bound_f`` (objects or equal-length
    sequences), ``pairs`` and optionally ``U_f_array``. Every point keeps its own grid (LOCAL
    adaptive grids of any size); all node sets, operand folds and bilinear forms of all points
    are evaluated in one launch each. With ``graph=True`` the launch sequence is captured once
    in a CUDA graph and replayed (``replays`` extra replays, e.g. for timing). With a split-BF16
    engine the exchange forms of all points go in one ragged tensor-core launch; ``tile`` chooses
    its tile: None (the default), a dict(bn=, stages=, order=) or "auto" (timed per shape class by
    ``tune.TILE_TUNER``, which records its choices).
    Returns, per point, what ``radial_ME_all_L_batch`` returns for it.
    """
    if not HAS_CUPY:
        raise RuntimeError("dwba_b200 engine library is not available (build it with python -m dwba_b200.build)")
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("radial_ME_all_L_sweep: no CUDA device available (the B200 engine has no CPU fallback)")
    from .engine import MultiPrepared, PreparedJob, plan_job
    from . import tune
    kw = dict(use_oscillatory_quadrature=options.get("use_oscillatory_quadrature", True),
              oscillatory_method=options.get("oscillatory_method", "advanced"),
              CC_nodes=options.get("CC_nodes", 5), phase_increment=options.get("phase_increment", 1.5708),
              min_grid_fraction=options.get("min_grid_fraction", 0.10), k_threshold=options.get("k_threshold", 0.5))
    eng = _engine_name(engine)
    jobs, shapes = [], []
    for pt in points:
        cache = pt.get("gpu_cache") or GPUCache(pt["grid"])
        job = _make_job(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"], pt["bound_f"],
                        list(pt["pairs"]), L_max, pt.get("U_f_array"), kw, cache)
        jobs.append((job, cache, plan_job(job)))
        shapes.append(isinstance(pt["bound_i"], (list, tuple)))

    def build(e):
        return MultiPrepared([PreparedJob(j, c.dg, e, plans=pl, rebuild_nodesets=True) for j, c, pl in jobs])
    if tune.is_auto(eng):
        cands = tune.candidates(eng)
        n_forms = sum(2 * len(j.transitions) * len(j.pairs) for j, _, _ in jobs)
        key = tune.TUNER.key(max(c.info.N for _, c, _ in jobs), n_forms, L_max, cands)
        _, mp = tune.TUNER.select(key, cands, build, lambda m: m.launch())
    else:
        mp = build(eng)
    if mp.tc is not None and tile is not None:
        if tile == "auto":
            n_ex = int(mp.tc["n"])
            tune.TILE_TUNER.select(tune.TILE_TUNER.key(mp.tc["nt"], mp.max_grid, n_ex, L_max), mp)
        else:
            mp.set_tile(tile)
    if graph:
        mp.capture()
        for _ in range(max(0, int(replays)) + 1):
            mp.replay()
    else:
        mp.launch()
    outs = mp.collect()
    results = []
    for (I_dir, I_exc), multi, pt in zip(outs, shapes, points):
        per_t = _results(I_dir, I_exc)
        results.append(per_t if multi else per_t[0])
    return results
