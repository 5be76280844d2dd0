"""Launch autotuner of the CUDA route (no counterpart in the reference, whose shader has
fixed workgroups and one form).

For a job it measures, on a sample of row bands spread over the frame, every candidate
launch setting (fdc_tuning: BLA deferral, resident blocks per SM, tile width) and both
delta forms (FP64 plain and FP32-mantissa floatexp), and keeps the fastest. The FP32
form is chosen only where its escape counts equal the plain form's on at least
`min_match` of the sampled samples (the route's acceptance bar), so the cut-over between
the forms is made per job kind from measured speed and measured agreement. Choices are
cached per job kind: tier, derivative, BLA.
"""
import ctypes as C
import dataclasses
import itertools
from typing import Callable, Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib

DEFERS = (1, 4, 8, 12, 16)
BLOCKS = (0, 4, 3)          # 0: the occupancy limit
TILE_WIDTHS = (8, 16, 4, 32)
MIN_MATCH = 0.999


@dataclasses.dataclass(frozen=True)
class Setting:
    defer: int = 0
    blocks_per_sm: int = 0
    tile_w: int = 0
    f32: bool = False


@dataclasses.dataclass
class Choice:
    setting: Setting
    ms: float                    # sampled kernel time of the chosen setting
    plain_ms: float              # sampled kernel time of the best plain-form setting
    match: Optional[float]       # FP32 count agreement with the plain form (None: not measured)
    table: List[Tuple[Setting, float]]


def kind(job: _lib.Job) -> Tuple[int, bool, bool]:
    return (int(job.tier), bool(job.flags & _lib.DERIVATIVE), bool(job.flags & _lib.BLA))


def bands(ny: int, count: int = 4, height: int = 16) -> List[Tuple[int, int]]:
    """`count` bands of `height` rows centred on evenly spaced rows of the frame."""
    height = min(height, ny)
    out = []
    for k in range(count):
        centre = int((k + 0.5) * ny / count)
        first = min(max(centre - height // 2, 0), ny - height)
        if (first, height) not in out:
            out.append((first, height))
    return out


def candidates(bla: bool, defers=DEFERS, blocks=BLOCKS, tiles=TILE_WIDTHS) -> List[Setting]:
    return [Setting(d if bla else 0, b, t) for d, b, t in itertools.product(defers if bla else (0,), blocks, tiles)]


def count_match(a: Dict[str, np.ndarray], b: Dict[str, np.ndarray]) -> float:
    """Share of samples whose class agrees and, where escaped, whose count is equal."""
    ea, eb = a["cls"] == 0, b["cls"] == 0
    same = (ea == eb) & (~ea | (a["n"] == b["n"]))
    return float(same.mean()) if same.size else 1.0


def choose(measure: Callable[[Setting], Tuple[float, Dict[str, np.ndarray]]], settings: Sequence[Setting],
           try_f32: bool = True, min_match: float = MIN_MATCH) -> Choice:
    """Measure each plain-form setting, then the best one's launch shape in the FP32
    form; keep the FP32 form only if it is faster and agrees on >= min_match."""
    table = []
    best, best_ms, ref = None, float("inf"), None
    for s in settings:
        ms, out = measure(s)
        table.append((s, ms))
        if ms < best_ms:
            best, best_ms, ref = s, ms, out
    chosen, chosen_ms, match = best, best_ms, None
    if try_f32:
        f = dataclasses.replace(best, f32=True)
        ms, out = measure(f)
        table.append((f, ms))
        match = count_match(ref, out)
        if ms < best_ms and match >= min_match:
            chosen, chosen_ms = f, ms
    return Choice(chosen, chosen_ms, best_ms, match, table)


class Tuner:
    """Per-device cache of choices; `apply(job)` sets the device's tuning and the job's
    form for its kind, measuring it first when the kind is new."""

    def __init__(self, dev, settings: Optional[Iterable[Setting]] = None, try_f32: bool = True,
                 min_match: float = MIN_MATCH, reps: int = 2):
        self.dev, self.try_f32, self.min_match, self.reps = dev, try_f32, min_match, reps
        self.settings = list(settings) if settings is not None else None
        self.cache: Dict[Tuple[int, bool, bool], Choice] = {}

    def _measure(self, job: _lib.Job) -> Callable[[Setting], Tuple[float, Dict[str, np.ndarray]]]:
        parts = bands(job.ny)

        def run(s: Setting):
            self.dev.tune(defer=s.defer, blocks_per_sm=s.blocks_per_sm, tile_w=s.tile_w)
            total, cols = 0.0, []
            for first, rows in parts:
                j = _lib.Job()
                C.memmove(C.byref(j), C.byref(job), C.sizeof(_lib.Job))
                j.first_row, j.rows = first, rows
                j.flags = (job.flags | _lib.F32) if s.f32 else (job.flags & ~_lib.F32)
                j.flags &= ~_lib.DEVICE_OUT
                best = float("inf")
                for _ in range(self.reps):
                    arrays, cnt, _ = self.dev.render_job(j, columns=())
                    best = min(best, cnt.kernel_ms)
                total += best
                lo, hi = first * job.nx, (first + rows) * job.nx
                cols.append({k: arrays[k][lo:hi] for k in ("cls", "n")})
            return total, {k: np.concatenate([c[k] for c in cols]) for k in ("cls", "n")}

        return run

    def choice(self, job: _lib.Job) -> Choice:
        key = kind(job)
        if key not in self.cache:
            settings = self.settings if self.settings is not None else candidates(key[2])
            saved = self.dev.tuning
            try:
                self.cache[key] = choose(self._measure(job), settings, self.try_f32, self.min_match)
            finally:
                self.dev.tune(defer=saved.defer, blocks_per_sm=saved.blocks_per_sm, tile_w=saved.tile_w)
        return self.cache[key]

    def apply(self, job: _lib.Job) -> Setting:
        s = self.choice(job).setting
        self.dev.tune(defer=s.defer, blocks_per_sm=s.blocks_per_sm, tile_w=s.tile_w)
        job.flags = (job.flags | _lib.F32) if s.f32 else (job.flags & ~_lib.F32)
        return s
