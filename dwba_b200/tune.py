"""Engine autotuner for the batched entry points (new; the reference has one fixed code path).

``engine="auto"`` picks, per shape class, the fastest FP64 engine (``semisep``, ``dense``);
``engine="auto_split"`` also admits the split-BF16 tensor-core form (``tc_bf16x3``, ~1e-7
relative error per integral, <= 1e-6 relative on cross sections). The first job of a shape class
times one launch of every admissible candidate with CUDA events on the current stream (after one
warm-up launch each) and keeps the fastest; later jobs of that class reuse the choice. A candidate
that refuses the job (e.g. the semiseparable form when r^L would leave the FP64 range) is skipped.

Shape class: (next power of two of the largest grid, next power of two of the number of forms,
L_max, candidate set).
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Sequence, Tuple

import torch

from . import _lib

AUTO_ENGINES = {"auto": ("semisep", "dense"), "auto_split": ("semisep", "dense", "tc_bf16x3")}


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
        st = torch.cuda.current_stream()
        times: Dict[str, float] = {}
        built: Dict[str, object] = {}
        for cand in candidates:
            try:
                obj = build(cand)
                launch(obj)  # warm-up (node sets, workspaces, library set-up)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                launch(obj)
                e1.record(st)
                e1.synchronize()
            except (_lib.DWBAError, ValueError):
                continue
            times[cand] = e0.elapsed_time(e1)
            built[cand] = obj
        if not times:
            raise _lib.DWBAError(_lib.DWBA_ERR_UNSUPPORTED, "no engine accepts this job")
        eng = min(times, key=times.get)
        self.choices[key] = eng
        self.timings_ms[key] = times
        return eng, built[eng]


TUNER = EngineTuner()


def is_auto(engine: Optional[str]) -> bool:
    return engine in AUTO_ENGINES


def candidates(engine: str) -> List[str]:
    return list(AUTO_ENGINES[engine])
