"""Autotuners for the batched entry points (new; the reference has one fixed code path).

Engines: ``engine="auto"`` picks, per shape class, the fastest FP64 engine (``semisep``, ``dense``);
``engine="auto_split"`` also admits the split-BF16 tensor-core form (``tc_bf16x3``, <= 1e-6
relative on cross sections with its accuracy guard). The first job of a shape class times every
admissible candidate -- one warm-up launch, then the median of ``REPEATS`` launches timed with CUDA
events on the current stream -- and keeps the fastest; later jobs of that class reuse the choice.
A candidate that refuses the job (e.g. the semiseparable form when r^L would leave the FP64 range)
is skipped.

Tiles: ``tile="auto"`` in the sweep entry point times the ragged tensor-core launch with every valid
tile (forms per CTA, pipeline depth, CTA order; ``TILES``) the same way and keeps the fastest per
shape class; ``TILE_TUNER.choices`` / ``timings_ms`` record the decisions.

Shape class: (next power of two of the largest grid, next power of two of the number of forms,
L_max, candidate set).
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Sequence, Tuple

import torch

from . import _lib

AUTO_ENGINES = {"auto": ("semisep", "dense"), "auto_split": ("semisep", "dense", "tc_bf16x3")}
REPEATS = 5  # timed launches per candidate (median)

# valid tiles of the ragged split-BF16 launch per number of bf16 terms: forms per CTA and pipeline
# depth (tensor memory: bn + stages * terms * 32 columns <= 512; shared memory <= 227 KB), each with
# both CTA orders (0: row blocks fastest, 1: form blocks fastest)
TILES = {nt: [dict(bn=bn, stages=sg, order=o) for bn, sg in shapes for o in (0, 1)]
         for nt, shapes in ((2, ((256, 3), (128, 3), (128, 4))), (3, ((256, 2), (128, 2), (128, 3))))}


def _median_ms(launch: Callable[[], None], repeats: int = REPEATS) -> float:
    """Median device time of ``launch()`` over ``repeats`` launches (events on the current stream)."""
    st = torch.cuda.current_stream()
    times = []
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        launch()
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    times.sort()
    return times[len(times) // 2]


def _pow2(n: int) -> int:
    p = 1
    while p < n:
        p <<= 1
    return p


class EngineTuner:
    """Chooses an engine per shape class by timing; ``choices`` and ``timings_ms`` record the decisions."""

    def __init__(self):
        self.choices: Dict[Tuple, str] = {}
        self.timings_ms: Dict[Tuple, Dict[str, float]] = {}

    @staticmethod
    def key(max_grid: int, n_forms: int, L_max: int, candidates: Sequence[str]) -> Tuple:
        return (_pow2(int(max_grid)), _pow2(int(n_forms)), int(L_max), tuple(candidates))

    def select(self, key: Tuple, candidates: Sequence[str], build: Callable[[str], object],
               launch: Callable[[object], None]):
        """Returns (engine, prepared object) for the key, building with ``build(engine)`` and timing
        ``launch(prepared)`` for every candidate the first time a key is seen."""
        eng = self.choices.get(key)
        if eng is not None:
            return eng, build(eng)
        times: Dict[str, float] = {}
        built: Dict[str, object] = {}
        for cand in candidates:
            try:
                obj = build(cand)
                launch(obj)  # warm-up (node sets, workspaces, library set-up)
                times[cand] = _median_ms(lambda: launch(obj))
            except (_lib.DWBAError, ValueError):
                times.pop(cand, None)
                continue
            built[cand] = obj
        if not times:
            raise _lib.DWBAError(_lib.DWBA_ERR_UNSUPPORTED, "no engine accepts this job")
        eng = min(times, key=times.get)
        self.choices[key] = eng
        self.timings_ms[key] = times
        return eng, built[eng]


TUNER = EngineTuner()


class TileTuner:
    """Chooses the tile of the ragged split-BF16 launch per shape class by timing."""

    def __init__(self):
        self.choices: Dict[Tuple, dict] = {}
        self.timings_ms: Dict[Tuple, Dict[str, float]] = {}

    @staticmethod
    def key(n_terms: int, max_grid: int, n_forms: int, L_max: int) -> Tuple:
        return (int(n_terms), _pow2(int(max_grid)), _pow2(int(n_forms)), int(L_max))

    def select(self, key: Tuple, mp) -> dict:
        """The tile for ``mp`` (a MultiPrepared of a tensor-core engine), timing ``mp.launch_tensor()``
        with every valid tile the first time a key is seen; ``mp`` is left set to the choice."""
        tile = self.choices.get(key)
        if tile is None:
            times: Dict[str, float] = {}
            for cand in TILES[key[0]]:
                mp.set_tile(cand)
                mp.launch_tensor()  # warm-up
                times[_tile_name(cand)] = _median_ms(mp.launch_tensor)
            best = min(times, key=times.get)
            tile = next(c for c in TILES[key[0]] if _tile_name(c) == best)
            self.choices[key] = tile
            self.timings_ms[key] = times
        mp.set_tile(tile)
        return tile


def _tile_name(t: dict) -> str:
    return f"bn{t['bn']}_s{t['stages']}_o{t['order']}"


TILE_TUNER = TileTuner()


def is_auto(engine: Optional[str]) -> bool:
    return engine in AUTO_ENGINES


def candidates(engine: str) -> List[str]:
    return list(AUTO_ENGINES[engine])
