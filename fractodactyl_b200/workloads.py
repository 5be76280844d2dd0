"""Job sets of the batched and jittered benchmark configurations, built on the route's
public pieces (Plane, Reference, Bla, make_job, Device.batch).

- film(): zoom frames toward one centre sharing one reference orbit (computed at the
  deepest frame's precision, which the reference allows: a reference may carry more
  bits than a view needs), with a BLA table per frame over it (or one shared table).
  Frames keep their own tier, except that F64-tier frames take the Fixed tier so the
  shared fixed-point orbit serves them.
- tiles(): locations each with its own orbit and table; each location's frame is cut
  into column x row windows, one job per window.
- jittered(): one frame whose samples are moved by seeded jitter (fdc_job.offsets).
"""
import dataclasses
import math
import time
from concurrent.futures import ThreadPoolExecutor
from typing import List, Optional, Tuple

import numpy as np

from . import _lib
from .locations import Frame, jitter_offsets
from .route import Bla, Plane, Reference, TIERS, _setup, bla_dc_bound, make_job


@dataclasses.dataclass
class JobSet:
    jobs: List[_lib.Job]
    handles: List[int]
    refs: List[Reference]
    blas: List[Optional[Bla]]
    planes: List[Plane]
    tiers: List[int]
    windows: List[Tuple[int, int, int, int]]  # (first_col, cols, first_row, rows) per job
    orbit_seconds: float
    bla_seconds: float
    keep: list = dataclasses.field(default_factory=list)  # host arrays jobs point to
    # per job, the frame it is a window of (jobs of one frame may share output buffers:
    # Batch groups); None: every job its own frame
    groups: Optional[List[int]] = None

    def free(self, dev):
        for h in set(self.handles):
            dev.free(h)
        self.handles = []


def _flags(derivative: bool, bla: Optional[Bla], extra: int = 0) -> int:
    return (_lib.DERIVATIVE if derivative else 0) | (_lib.BLA if bla is not None else 0) | extra


def _log2_bound(dc_e):
    dc, e = dc_e
    return math.log2(dc) + e if dc > 0 else -math.inf


def film(dev, frames: List[Frame], extra_flags: int = 0, max_iter: Optional[int] = None,
         tables: str = "per-frame") -> JobSet:
    """tables "per-frame": one BLA table per frame over the shared orbit, each for its
    frame's |dc| bound (the reference's per-frame BLA film mode). "shared": one table for
    the largest bound of all frames; across widths 1e-10..1e-500 that table has no level
    (every radius is negative), so the film then runs without block skips."""
    planes = [Plane.new(f.view, f.params.nx, f.params.ny) for f in frames]
    bits = max(pl.bits for pl in planes)
    f0 = frames[0]
    mi = max_iter or f0.params.max_iter
    t = time.perf_counter()
    r = Reference.from_fixed(f0.view.center_re, f0.view.center_im, bits, mi)
    orbit_s = time.perf_counter() - t
    tiers = [max(pl.tier, TIERS["fixed"]) for pl in planes]
    bounds = []
    for f, tier in zip(frames, tiers):
        p = dataclasses.replace(f.params, tier={1: "fixed", 2: "scaled"}[tier])
        bounds.append(bla_dc_bound(f.view, p))
    t = time.perf_counter()
    blas: List[Optional[Bla]] = [None] * len(frames)
    if f0.bla_eps is not None:
        if tables == "shared":
            dc, e = max(bounds, key=_log2_bound)
            b = Bla.build_scaled(r, f0.bla_eps, dc, e)
            blas = [b if b.levels else None] * len(frames)
        else:
            blas = [Bla.build_scaled(r, f0.bla_eps, dc, e) for dc, e in bounds]
            blas = [b if b.levels else None for b in blas]
    bla_s = time.perf_counter() - t
    nuc = r.nucleus_period()
    jobs, windows, handles = [], [], []
    shared = None
    for f, pl, tier, b in zip(frames, planes, tiers, blas):
        if tables == "shared":
            shared = shared if shared is not None else dev.upload(r, b)
            h = shared
        else:
            h = dev.upload(r, b)
        p = dataclasses.replace(f.params, max_iter=mi)
        jobs.append(make_job(pl, tier, p, h, nuc, _flags(p.needs_derivative(), b, extra_flags)))
        handles.append(h)
        windows.append((0, p.nx, 0, p.ny))
    refs = [r] if tables == "shared" else [r] * len(frames)
    return JobSet(jobs, handles, refs, blas if tables != "shared" else blas[:1], planes, tiers, windows,
                  orbit_s, bla_s)


def tiles(dev, frames: List[Frame], tile: Tuple[int, int], extra_flags: int = 0, max_iter: Optional[int] = None,
          locations_first: Optional[int] = None) -> JobSet:
    """One job per tile-sized window of every frame (orbits computed in parallel threads,
    one thread each: the host orbit releases the interpreter while it runs, and with many
    orbits, parallelism across orbits beats sharing each orbit's squarings)."""
    frames = frames[:locations_first] if locations_first else frames
    setups = []
    for f in frames:
        p = dataclasses.replace(f.params, max_iter=max_iter or f.params.max_iter)
        plane, tier = _setup(f.view, p)
        setups.append((f, p, plane, tier))

    def orbit(s):
        f, p, plane, tier = s
        r = Reference.from_fixed(f.view.center_re, f.view.center_im, max(plane.bits, 128), p.max_iter, threads=1)
        r.bits = max(plane.bits, 128)
        return r

    t = time.perf_counter()
    with ThreadPoolExecutor() as ex:
        refs = list(ex.map(orbit, setups))
    orbit_s = time.perf_counter() - t
    t = time.perf_counter()
    blas = []
    for (f, p, plane, tier), r in zip(setups, refs):
        b = None
        if f.bla_eps is not None:
            dc, e = bla_dc_bound(f.view, p)
            b = Bla.build_scaled(r, f.bla_eps, dc, e)
            if b.levels == 0:
                b = None
        blas.append(b)
    bla_s = time.perf_counter() - t
    jobs, handles, planes, tiers, windows = [], [], [], [], []
    tw, th = tile
    groups = []
    for loc, ((f, p, plane, tier), r, b) in enumerate(zip(setups, refs, blas)):
        h = dev.upload(r, b)
        nuc = r.nucleus_period()
        tier = max(tier, TIERS["fixed"])
        for y0 in range(0, p.ny, th):
            for x0 in range(0, p.nx, tw):
                j = make_job(plane, tier, p, h, nuc, _flags(p.needs_derivative(), b, extra_flags))
                j.first_col, j.cols = x0, min(tw, p.nx - x0)
                j.first_row, j.rows = y0, min(th, p.ny - y0)
                jobs.append(j)
                handles.append(h)
                planes.append(plane)
                tiers.append(tier)
                windows.append((x0, j.cols, y0, j.rows))
                groups.append(loc)
    return JobSet(jobs, handles, refs, blas, planes, tiers, windows, orbit_s, bla_s, groups=groups)


def jittered(dev, frame: Frame, seed: int = 3, extra_flags: int = 0, max_iter: Optional[int] = None) -> JobSet:
    p = dataclasses.replace(frame.params, max_iter=max_iter or frame.params.max_iter)
    plane, tier = _setup(frame.view, p)
    t = time.perf_counter()
    r = Reference.from_fixed(frame.view.center_re, frame.view.center_im, plane.bits, p.max_iter)
    r.bits = plane.bits
    orbit_s = time.perf_counter() - t
    offs = jitter_offsets(plane, p.nx, p.ny, seed)
    t = time.perf_counter()
    bla = None
    if frame.bla_eps is not None:
        # the jitter reaches at most half a sample beyond the grid: bound |dc| by the
        # offsets themselves, with a margin over the route's own hypot of them
        half = float(np.hypot(offs[:, 0], offs[:, 1]).max()) * (1.0 + 1e-12)
        dc, e = (plane.h_m * half, plane.h_e) if tier == TIERS["scaled"] else (plane.h() * half, 0)
        bla = Bla.build_scaled(r, frame.bla_eps, dc, e)
        if bla.levels == 0:
            bla = None
    bla_s = time.perf_counter() - t
    h = dev.upload(r, bla)
    j = make_job(plane, tier, p, h, r.nucleus_period(), _flags(p.needs_derivative(), bla, extra_flags))
    j.offsets = offs.ctypes.data
    return JobSet([j], [h], [r], [bla], [plane], [tier], [(0, p.nx, 0, p.ny)], orbit_s, bla_s, keep=[offs])
