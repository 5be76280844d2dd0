"""The `--gpu-perturb cuda` route: fractodactyl's sample API over the CUDA library.

Mirrors the names, argument meaning and refusals of junovhs/fractodactyl's host side for
this path: View / Params (crates/fd-samples/src/header.rs:14-27, crates/fd-kernel/src/
grid.rs:17-38), Plane (view.rs:42-128), Reference (reference.rs), Bla (bla.rs), and the
route entry points perturb_gpu::{enabled, render, render_bla} (crates/fd-cli/src/
perturb_gpu/frame.rs:62-84), whose CUDA counterpart keeps every sample the device
finishes (its results are the CPU kernel's) instead of admitting only guarded escapes.
Frames the route declines raise Declined: the caller restarts them on the CPU from n = 0
(frame.rs:357-368), as the reference's route does.
"""
import ctypes as C
import math
import dataclasses
import os
import sys
import time
from typing import Optional

import numpy as np

from . import _lib
from ._lib import lib

EPS = 2.0 ** -50          # exact-mode BLA tolerance (crates/fd-cli/src/orbit.rs:16)
EPS_MAX = 2.0 ** -41      # largest eps whose blocks never cover a judged iterate (bla.rs:17)
FILM_EPS = 2.0 ** -26     # film-mode tolerance (orbit.rs:22)
MAX_LEN = 1 << 20         # reference.rs:16
COLUMNS = ("class", "nu", "de", "normal")
TIERS = {"f64": 0, "fx": 1, "fixed": 1, "scaled": 2}
TIER_NAMES = {0: "F64", 1: "Fixed", 2: "Scaled"}


class Declined(RuntimeError):
    """The route does not take this frame; render it on the CPU from n = 0."""


class Incomplete(Declined):
    """A deadline ended the render with some samples unfinished (frame.rs:338-341): the
    finished samples are the CPU kernel's, and only the samples where `mask` is true
    need the CPU (render_with_masked from n = 0, grid.rs:175-182), then the two are
    overlaid. Carries what render_with returns (header, samples, stats, bla_stats; the
    unfinished samples hold zeroed columns and status 0, the counters cover the finished
    ones) and the mask, one bool per sample in row-major order. A caller that treats it
    as a plain Declined restarts the whole frame instead, which is also correct."""

    def __init__(self, message, header, samples, stats, bla_stats, mask):
        super().__init__(message)
        self.header, self.samples, self.stats, self.bla_stats, self.mask = header, samples, stats, bla_stats, mask

    def merge(self, cpu: "Samples", cpu_stats: "Stats"):
        """The whole frame after the caller's CPU restart: `cpu` is its masked render of
        the unfinished samples (every column the device wrote, the others unset); the
        finished samples keep the device's values and the iterations add up, as
        frame.rs:338-343 overlays and counts them. Returns (Samples, Stats)."""
        out = dataclasses.replace(self.samples)
        for name in ("cls", "nu", "de", "normal", "n", "z", "dz", "dexp", "bound", "ez", "ed", "stripe"):
            g, c = getattr(self.samples, name), getattr(cpu, name)
            if g is not None and c is not None:
                g = g.copy()
                g[self.mask] = c[self.mask]
                setattr(out, name, g)
        if out.status is not None:
            out.status = self.samples.status.copy()
            out.status[self.mask] = 1
        return out, Stats(self.stats.reference_len, self.stats.reference_seconds,
                          self.stats.iterations + cpu_stats.iterations)


class RouteError(RuntimeError):
    pass


def enabled(value: Optional[str]) -> bool:
    """perturb_gpu::enabled (frame.rs:62-68) with the `cuda` and `cuda-bla` routes added."""
    v = "off" if value is None else value
    if v == "off":
        return False
    if v in ("on", "bla", "cuda", "cuda-bla"):
        return True
    raise ValueError(f"--gpu-perturb: expected on, bla, cuda, cuda-bla or off, got {v!r}")


@dataclasses.dataclass
class View:
    center_re: str
    center_im: str
    width: str
    rotation: float = 0.0


@dataclasses.dataclass
class Params:
    nx: int
    ny: int
    ss: int = 1
    max_iter: int = 100_000
    escape_radius: float = 1e10
    columns: tuple = ("nu", "de", "normal")
    threads: int = 0
    tier: Optional[str] = None
    stripe_window: int = 16   # StripeParams (crates/fd-kernel/src/stripe.rs:20-36, grid.rs:36-37)
    stripe_freq: float = 5.0

    def needs_derivative(self):
        return "de" in self.columns or "normal" in self.columns


@dataclasses.dataclass
class Plane:
    c_re: float
    c_im: float
    h_m: float
    h_e: int
    tier: int
    bits: int
    cos_rot: float
    sin_rot: float

    @classmethod
    def new(cls, view: View, nx: int, ny: int) -> "Plane":
        p = _lib.Plane()
        if lib().fdh_plane_new(view.center_re.encode(), view.center_im.encode(), view.width.encode(),
                               float(view.rotation), nx, ny, C.byref(p)) != 0:
            raise ValueError(_lib.host_error())
        return cls(p.c_re, p.c_im, p.h_m, p.h_e, p.tier, p.bits, p.cos_rot, p.sin_rot)

    def kernel(self, tier: int) -> str:
        """view.rs:90-96."""
        return {0: "pert-f64/1", 1: f"pert-fx/1 bits={self.bits}", 2: f"pert-fx-scaled/1 bits={self.bits}"}[tier]

    def allows(self, tier: int) -> bool:
        return tier == 2 or (tier == 1 and self.tier != 2) or (tier == 0 and self.tier == 0)

    def h(self) -> float:
        return self.h_m * 2.0 ** self.h_e if self.h_e > -1074 else 0.0

    def _c(self):
        return _lib.Plane(self.c_re, self.c_im, self.h_m, self.h_e, self.tier, self.bits, self.cos_rot,
                          self.sin_rot)


@dataclasses.dataclass
class Reference:
    """Reference orbit Z_0..Z_{len-1} as f64 SoA, with its working precision in bits."""
    re: np.ndarray
    im: np.ndarray
    bits: int = 53

    def __len__(self):
        return len(self.re)

    @classmethod
    def from_fixed(cls, center_re: str, center_im: str, bits: int, max_iter: int, threads: int = 0) -> "Reference":
        """threads: 3 shares each step's squarings among three threads on orbits of ~1,700
        bits and more, 1 keeps the orbit on the calling thread, 0 picks 3 on hosts with 4
        or more hardware threads. The orbit is the same bit for bit."""
        cap = min(max_iter, MAX_LEN - 1) + 1
        re, im = np.empty(cap), np.empty(cap)
        n = lib().fdh_orbit_fixed_threads(center_re.encode(), center_im.encode(), bits, max_iter, re.ctypes.data,
                                          im.ctypes.data, cap, threads)
        if n < 0:
            raise ValueError(_lib.host_error())
        return cls(re[:n].copy(), im[:n].copy(), bits)

    def error_radius(self, bits: Optional[int], c_re: float, c_im: float) -> np.ndarray:
        """Reference::error_radius (reference.rs:122-148): q[m] >= |A_m - Z_m| for each
        point; bits None for an f64 orbit from the correctly rounded centre (c_re, c_im)."""
        re, im = np.ascontiguousarray(self.re), np.ascontiguousarray(self.im)
        q = np.empty(len(re))
        if lib().fdh_error_radius(re.ctypes.data, im.ctypes.data, len(re), -1 if bits is None else bits, c_re, c_im,
                                  q.ctypes.data) != 0:
            raise ValueError(_lib.host_error())
        return q

    @classmethod
    def new(cls, c_re: float, c_im: float, max_iter: int, escape_radius: float) -> "Reference":
        cap = min(max_iter, MAX_LEN - 1) + 1
        re, im = np.empty(cap), np.empty(cap)
        n = lib().fdh_orbit_f64(c_re, c_im, max_iter, escape_radius, re.ctypes.data, im.ctypes.data, cap)
        if n < 0:
            raise ValueError(_lib.host_error())
        return cls(re[:n].copy(), im[:n].copy(), 53)

    def nucleus_period(self) -> Optional[int]:
        re, im = np.ascontiguousarray(self.re), np.ascontiguousarray(self.im)
        p = lib().fdh_nucleus_period(re.ctypes.data, im.ctypes.data, len(re))
        return None if p < 0 else int(p)


@dataclasses.dataclass
class Bla:
    """A BLA table in its export form: level-major [f64; 7] blocks (bla.rs:52-57)."""
    blocks: np.ndarray  # (n, 7)
    level_offsets: np.ndarray  # levels + 1
    eps: float
    dc_max: float
    dc_exp: int
    points: int

    @property
    def levels(self):
        return len(self.level_offsets) - 1

    @classmethod
    def build_scaled(cls, r: Reference, eps: float, dc_max: float, dc_exp: int = 0, threads: int = 0) -> "Bla":
        re, im = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
        levels, blocks = C.c_uint32(), C.c_uint64()
        # one pass into buffers of the largest possible size: at most len - 2 blocks (the
        # levels halve from (len - 2) / 2) and 64 levels
        cap = max(len(re) - 2, 1)
        b = np.empty((cap, 7))
        offs = np.empty(65, np.uint64)
        if lib().fdh_bla_build_into(re.ctypes.data, im.ctypes.data, len(re), eps, dc_max, dc_exp, threads,
                                    b.ctypes.data, cap, offs.ctypes.data, 64, C.byref(levels),
                                    C.byref(blocks)) != 0:
            raise ValueError(_lib.host_error())
        n = blocks.value
        b = b[:n] if 4 * n >= 3 * cap else b[:n].copy()  # a table well below the bound lets the rest go
        return cls(b, offs[:levels.value + 1].copy(), eps, dc_max, dc_exp, len(re))


@dataclasses.dataclass
class DeviceTable:
    """The BLA table Bla.build_scaled(orbit, eps, dc_max, dc_exp) would build, built on the
    device over the uploaded orbit instead (fdc_build_bla): no host build, no table upload.
    render_with fills in levels and blocks (the kept level and block counts) after the build."""
    eps: float
    dc_max: float
    dc_exp: int
    points: int
    levels: int = 0
    blocks: int = 0


@dataclasses.dataclass
class Series:
    """A parameter-series start (crates/fd-kernel/src/series.rs:57-84): every sample with
    |dc| <= rho may start at iterate n from delta = sum_k b_k (dc / rho)^k. n = 0: none
    admitted (the plain kernel)."""
    n: int
    rho: float
    points: int
    b: np.ndarray  # (order, 2): b_1..b_order as (re, im)
    state_bound: float
    derivative_bound: float
    shift_px: float
    built_steps: int
    coefficient_pairs: int
    stop: str

    @classmethod
    def build(cls, r: Reference, rho: float, pixel: float, max_iter: int, stalled_steps: int = 32) -> "Series":
        """Series::build with SeriesConfig::default() over orbit r, for |dc| <= rho and
        output pixels of `pixel` in c."""
        re, im = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
        info = _lib.SeriesInfo()
        b = np.zeros((64, 2))
        if lib().fdh_series_build(re.ctypes.data, im.ctypes.data, len(re), rho, pixel, max_iter, stalled_steps,
                                  C.byref(info), b.ctypes.data, 64) != 0:
            raise ValueError(_lib.host_error())
        return cls(info.n, info.rho, info.points, b[:info.order].copy(), info.state_bound, info.derivative_bound,
                   info.shift_px, info.built_steps, info.coefficient_pairs, info.stop.decode())


@dataclasses.dataclass
class Header:
    """crates/fd-samples/src/header.rs:29-45."""
    columns: tuple
    nx: int
    ny: int
    ss: int
    max_iter: int
    escape_radius: float
    view: View
    kernel: str
    minor: int = 1


@dataclasses.dataclass
class Samples:
    cls: np.ndarray
    nu: Optional[np.ndarray] = None
    de: Optional[np.ndarray] = None
    normal: Optional[np.ndarray] = None
    n: Optional[np.ndarray] = None
    z: Optional[np.ndarray] = None
    dz: Optional[np.ndarray] = None
    dexp: Optional[np.ndarray] = None
    status: Optional[np.ndarray] = None
    bound: Optional[np.ndarray] = None  # Bound column (f32 nu error bound; bounded renders)
    stripe: Optional[np.ndarray] = None  # Stripe column (f32 stripe average of escaped samples)
    ez: Optional[np.ndarray] = None     # raw error radii of escaped samples (bounded renders)
    ed: Optional[np.ndarray] = None


@dataclasses.dataclass
class Stats:
    reference_len: int = 0
    reference_seconds: float = 0.0
    iterations: int = 0


@dataclasses.dataclass
class BlaStats:
    blocks: int = 0
    skipped: int = 0
    fallback_samples: int = 0
    closed_form_samples: int = 0
    shift_px: Optional[float] = None


@dataclasses.dataclass
class RouteReport:
    """The counters frame.rs:350-353 prints, plus device time and launch count."""
    device: str = ""
    accepted: int = 0
    fallback: int = 0
    gpu_seconds: float = 0.0
    kernel_ms: float = 0.0
    launches: int = 0
    table_seconds: float = 0.0
    table_blocks: int = 0
    total_seconds: float = 0.0

    def line(self, st: Stats, bs: Optional[BlaStats]):
        eff = st.iterations - (bs.blocks - bs.skipped if bs else 0)
        extra = f" gpu_blocks={bs.blocks} gpu_skipped={bs.skipped}" if bs else ""
        return (f"fd gpu-perturb: device={self.device!r} accepted={self.accepted} fallback={self.fallback} "
                f"guard=0 unfinished={self.fallback} invalid=0 gpu_seconds={self.gpu_seconds:.6f} "
                f"kernel_ms={self.kernel_ms:.3f} total_seconds={self.total_seconds:.6f} restart=zero"
                f"{extra} effective_iterations={eff}")


def _check(status, dev, what):
    if status == _lib.DECLINED:
        raise Declined(f"{what}: {lib().fdc_last_error(dev.h).decode()}")
    if status != _lib.OK and status != _lib.TIMEOUT:
        raise RouteError(f"{what}: {_lib.STATUS_NAMES.get(status, status)}: {lib().fdc_last_error(dev.h).decode()}")


class Device:
    """One fdc_ctx on one GPU (a context per thread; it owns one CUDA stream)."""

    def __init__(self, index: int = 0):
        self.h = C.c_void_p()
        st = lib().fdc_open(index, C.byref(self.h))
        if st != _lib.OK:
            raise RouteError(f"fdc_open({index}): {_lib.STATUS_NAMES.get(st, st)}")
        self.index = index
        self._orbit_len = {}  # handle -> points, for build_bla's export size

    def close(self):
        if self.h:
            lib().fdc_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, r: Reference, bla: Optional[Bla] = None) -> int:
        re, im = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
        h = C.c_int32()
        _check(lib().fdc_upload_orbit(self.h, re.ctypes.data, im.ctypes.data, len(re), r.bits, C.byref(h)), self,
               "upload orbit")
        self._orbit_len[h.value] = len(re)
        if bla is not None:
            b = np.ascontiguousarray(bla.blocks)
            offs = np.ascontiguousarray(bla.level_offsets)
            _check(lib().fdc_upload_bla(self.h, h.value, b.ctypes.data if len(b) else None,
                                        offs.ctypes.data, bla.levels, bla.eps, bla.dc_max, bla.dc_exp), self,
                   "upload BLA")
        return h.value

    def build_bla(self, orbit: int, eps: float, dc_max: float, dc_exp: int = 0, export: bool = False):
        """fdc_build_bla: the BLA table of Bla.build_scaled(orbit, eps, dc_max, dc_exp) built on
        the device over the uploaded orbit, in place of an uploaded one. Returns the kept level
        count, and with export the blocks in the export form ([f64; 7] rows, level-major)."""
        levels = C.c_uint32()
        out = None
        if export:
            cap = max(self._orbit_len[orbit] - 3, 0)
            out = np.empty((max(cap, 1), 7))
        _check(lib().fdc_build_bla(self.h, orbit, eps, dc_max, dc_exp, C.byref(levels),
                                   out.ctypes.data if out is not None else None), self, "build BLA")
        if not export:
            return levels.value
        steps = max(self._orbit_len[orbit] - 2, 0)
        total = sum(steps >> (i + 1) for i in range(levels.value))
        return levels.value, out[:total].copy()

    def upload_series(self, orbit: int, series: "Series"):
        """fdc_upload_series: the series start for jobs on `orbit` with the SERIES flag."""
        b = np.ascontiguousarray(series.b, dtype=np.float64)
        _check(lib().fdc_upload_series(self.h, orbit, series.points, series.n, series.rho,
                                       b.ctypes.data if len(b) else None, len(b)), self, "upload series")

    def free(self, orbit: int):
        """fdc_free_orbit; refused (RouteError) while a live batch reads the orbit."""
        _check(lib().fdc_free_orbit(self.h, orbit), self, "free orbit")
        self._orbit_len.pop(orbit, None)

    def upload_error_radius(self, orbit: int, q: np.ndarray):
        """fdc_upload_error_radius: the orbit's error radii for bounded renders."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        _check(lib().fdc_upload_error_radius(self.h, orbit, q.ctypes.data, len(q)), self, "upload error radii")

    def render_job(self, job: _lib.Job, raw=False, columns=COLUMNS, device_out=None, host_out=None, bounded=False,
                   stripe=None):
        """fdc_render into fresh host arrays, into the caller's host arrays (host_out: the
        dict an earlier call returned, reused frame after frame) or into caller device
        buffers (device_out). bounded: fdc_render_bounded, adding the host arrays
        "bound", "ez" and "ed". stripe: (window, freq) for fdc_render_stripe, adding the
        array "stripe" (a device pointer under device_out["stripe"])."""
        n = job.nx * job.ny
        out = _lib.Out()
        arrays = {}
        if device_out is not None:
            for k, v in device_out.items():
                setattr(out, k, v)
        elif host_out is not None:
            arrays = host_out
            for k, a in arrays.items():
                setattr(out, k, a.ctypes.data)
        else:
            want = {"cls": np.uint8, "status": np.uint8, "n": np.uint32}
            if "nu" in columns:
                want["nu"] = np.float64
            if "de" in columns:
                want["de"] = np.float32
            if "normal" in columns:
                want["normal"] = np.uint16
            for k, dt in want.items():
                arrays[k] = np.zeros(n, dt)
            if raw:
                arrays["z"] = np.zeros((n, 2))
                arrays["dz"] = np.zeros((n, 2))
                arrays["dexp"] = np.zeros(n, np.int64)
            for k, a in arrays.items():
                setattr(out, k, a.ctypes.data)
        cnt = _lib.Counters()
        if stripe is not None:
            if device_out is not None:
                sp = device_out["stripe"]
            else:
                if "stripe" not in arrays:
                    arrays["stripe"] = np.zeros(n, np.float32)
                sp = arrays["stripe"].ctypes.data
            st = lib().fdc_render_stripe(self.h, C.byref(job), C.byref(out),
                                         C.byref(_lib.Stripe(int(stripe[0]), float(stripe[1]))), sp, C.byref(cnt))
        elif bounded:
            for k, dt in (("bound", np.float32), ("ez", np.float64), ("ed", np.float64)):
                if k not in arrays:
                    arrays[k] = np.zeros(n, dt)
            bout = _lib.BoundOut(arrays["bound"].ctypes.data, arrays["ez"].ctypes.data, arrays["ed"].ctypes.data)
            st = lib().fdc_render_bounded(self.h, C.byref(job), C.byref(out), C.byref(bout), C.byref(cnt))
        else:
            st = lib().fdc_render(self.h, C.byref(job), C.byref(out), C.byref(cnt))
        _check(st, self, "render")
        return arrays, cnt, st

    @property
    def tuning(self) -> _lib.Tuning:
        t = _lib.Tuning()
        lib().fdc_get_tuning(self.h, C.byref(t))
        return t

    def tune(self, defer: Optional[int] = None, blocks_per_sm: Optional[int] = None, tile_w: Optional[int] = None,
             order: Optional[int] = None):
        """fdc_set_tuning: change the given launch settings, keep the others."""
        t = self.tuning
        if order is not None:
            t.order = order
        if defer is not None:
            t.defer = defer
        if blocks_per_sm is not None:
            t.blocks_per_sm = blocks_per_sm
        if tile_w is not None:
            t.tile_w = tile_w
        _check(lib().fdc_set_tuning(self.h, C.byref(t)), self, "tuning")

    def batch(self, jobs, columns=COLUMNS, raw=False, groups=None) -> "Batch":
        """fdc_batch_create over `jobs` (uploaded orbits; FDC_DEVICE_OUT is set here) with
        fresh device columns per frame (torch tensors on this GPU; see Batch for groups)."""
        return Batch(self, jobs, columns, raw, groups)


_BATCH_DTYPES = {"cls": "uint8", "status": "uint8", "n": "int32", "nu": "float64", "de": "float32",
                 "normal": "int16", "z": "float64", "dz": "float64", "dexp": "int64"}
_HOST_DTYPES = {"cls": np.uint8, "status": np.uint8, "n": np.uint32, "nu": np.float64, "de": np.float32,
                "normal": np.uint16, "z": np.float64, "dz": np.float64, "dexp": np.int64}


class Batch:
    """Many jobs rendered by one graph replay (fdc_batch_run): one persistent launch per
    kernel variant over all jobs' tiles. Outputs stay on the device between runs, one
    tensor per column holding every frame's samples; `columns(k)` copies job k's frame
    back, `all_columns` every frame's with one copy per column. groups (optional, one
    key per job): jobs with the same key are windows of one frame (same view, grid and
    orbit) and write into one frame buffer; by default every job has a frame of its own."""

    def __init__(self, dev: Device, jobs, columns=COLUMNS, raw=False, groups=None):
        import torch
        self.dev, self.jobs, self.h = dev, list(jobs), C.c_void_p()
        self.names = ["cls", "status", "n"] + [c for c in ("nu", "de", "normal") if c in columns]
        if raw:
            self.names += ["z", "dz", "dexp"]
        keys = list(range(len(self.jobs))) if groups is None else list(groups)
        if len(keys) != len(self.jobs):
            raise ValueError("one group key per job")
        frame_of, sizes = {}, []
        self.frame = []  # frame index per job
        for j, key in zip(self.jobs, keys):
            if key not in frame_of:
                frame_of[key] = len(sizes)
                sizes.append(j.nx * j.ny)
            elif sizes[frame_of[key]] != j.nx * j.ny:
                raise ValueError("jobs of one group must share their grid")
            self.frame.append(frame_of[key])
        self.starts = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        total = int(self.starts[-1])
        self.cols = {}
        for name in self.names:
            shape = (total, 2) if name in ("z", "dz") else (total,)
            self.cols[name] = torch.zeros(shape, dtype=getattr(torch, _BATCH_DTYPES[name]), device=f"cuda:{dev.index}")
        outs = (_lib.Out * len(self.jobs))()
        cjobs = (_lib.Job * len(self.jobs))()
        for k, j in enumerate(self.jobs):
            a = int(self.starts[self.frame[k]])
            for name, t in self.cols.items():
                setattr(outs[k], name, t[a:].data_ptr())  # job k's frame starts here
            C.memmove(C.byref(cjobs[k]), C.byref(j), C.sizeof(_lib.Job))
            cjobs[k].flags |= _lib.DEVICE_OUT
        _check(lib().fdc_batch_create(dev.h, cjobs, outs, len(self.jobs), C.byref(self.h)), dev, "batch create")

    def run(self):
        """Replay the batch; returns (total counters, per-job counters)."""
        total = _lib.Counters()
        per = (_lib.Counters * len(self.jobs))()
        _check(lib().fdc_batch_run(self.dev.h, self.h, C.byref(total), per), self.dev, "batch run")
        return total, list(per)

    def columns(self, k: int):
        f = self.frame[k]
        a, b = int(self.starts[f]), int(self.starts[f + 1])
        return {name: t[a:b].cpu().numpy().view(_HOST_DTYPES[name]) for name, t in self.cols.items()}

    def host_arrays(self):
        """Host arrays for all_columns, allocated once by the caller and reused."""
        return {name: np.empty(tuple(t.shape), _HOST_DTYPES[name]) for name, t in self.cols.items()}

    def all_columns(self, host_out=None):
        """Every job's columns with one device-to-host copy per column: a list of per-job
        dicts of views into one host array per column, host_out's when given (a dict an
        earlier call returned as its second value, reused frame after frame)."""
        import torch
        host = host_out if host_out is not None else self.host_arrays()
        for name, t in self.cols.items():
            torch.from_numpy(host[name].view(_BATCH_DTYPES[name])).copy_(t)
        per = [{name: a[int(self.starts[f]):int(self.starts[f + 1])] for name, a in host.items()}
               for f in self.frame]
        return per, host

    def free(self):
        if self.h:
            lib().fdc_batch_free(self.dev.h, self.h)
            self.h = C.c_void_p()


def _rust_f64(x: float) -> str:
    """f64's Display in Rust for the values a refusal message prints."""
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return str(int(x)) if x == int(x) and abs(x) < 1e16 else repr(x)


def _check_bla_escape_radius(radius: float):
    """grid.rs:393-398: a BLA table needs an escape radius of at least 4 (NaN refused)."""
    if math.isnan(radius) or radius < 4.0:
        raise ValueError(f"escape radius {_rust_f64(radius)} is below 4: BLA blocks may only skip iterates with "
                         "|z| <= 2 (1 + 2 eps), which needs escape radius >= 4")


def _setup(view: View, p: Params):
    """grid.rs:779-799."""
    if p.ss == 0 or p.nx % p.ss or p.ny % p.ss:
        raise ValueError("grid must be a whole number of pixels")
    plane = Plane.new(view, p.nx, p.ny)
    tier = plane.tier if p.tier in (None, "auto") else TIERS[p.tier]
    if not plane.allows(tier):
        raise ValueError(f"{TIER_NAMES[tier]} tier is not valid at this depth (cheapest valid: "
                         f"{TIER_NAMES[plane.tier]})")
    return plane, tier


def reference(view: View, p: Params):
    """grid::reference (grid.rs:87-90, compute :802-815): the orbit and its precision."""
    plane, tier = _setup(view, p)
    if tier == 0:
        return Reference.new(plane.c_re, plane.c_im, p.max_iter, p.escape_radius), 53
    return Reference.from_fixed(view.center_re, view.center_im, plane.bits, p.max_iter), plane.bits


def bla_dc_bound(view: View, p: Params):
    """grid.rs:418-427."""
    plane, tier = _setup(view, p)
    dc, e = C.c_double(), C.c_int64()
    lib().fdh_dc_bound(C.byref(plane._c()), tier, p.nx, p.ny, C.byref(dc), C.byref(e))
    return dc.value, e.value


_devices = {}


def device(index: int = 0) -> Device:
    d = _devices.get(index)
    if d is None:
        d = _devices[index] = Device(index)
    return d


def make_job(plane: Plane, tier: int, p: Params, orbit: int, nucleus: Optional[int], flags: int) -> _lib.Job:
    j = _lib.Job()
    j.orbit = orbit
    j.tier = tier
    j.nx, j.ny, j.ss = p.nx, p.ny, p.ss
    j.flags = flags
    j.c_re, j.c_im = plane.c_re, plane.c_im
    j.h_m, j.h_e = plane.h_m, plane.h_e
    j.cos_rot, j.sin_rot = plane.cos_rot, plane.sin_rot
    j.max_iter = p.max_iter
    j.escape_radius = p.escape_radius
    j.nucleus_period = -1 if nucleus is None else nucleus
    return j


def encode_host(plane: Plane, ss: int, s: "Samples", columns=("nu", "de", "normal"), threads: int = 0):
    """Columns of the escaped samples from the device's raw state, on the host with the
    host's libm (fdh_encode = Store::put, store.rs:66-112): the CPU route's bytes."""
    n = len(s.cls)
    s.nu = np.zeros(n) if "nu" in columns else None
    s.de = np.zeros(n, np.float32) if "de" in columns else None
    s.normal = np.zeros(n, np.uint16) if "normal" in columns else None
    ptr = lambda a: None if a is None else np.ascontiguousarray(a).ctypes.data
    lib().fdh_encode(C.byref(plane._c()), ss, n, ptr(s.cls), ptr(s.n), ptr(s.z), ptr(s.dz), ptr(s.dexp),
                     ptr(s.nu), ptr(s.de), ptr(s.normal), threads)
    return s


def render_with(view: View, p: Params, orbit=None, bla: Optional[Bla] = None, dev: Optional[Device] = None,
                raw=False, shift=True, report: Optional[RouteReport] = None, quiet=True, host_encode=False,
                series: Optional["Series"] = None, deadline_ms: Optional[float] = None):
    """fd_kernel::render_with / render_bla (grid.rs:106-208) on the CUDA route; with
    `series`, every sample starts from it (Series::render_masked, grid.rs:341-373).

    Returns (Header, Samples, Stats, BlaStats or None). Refusals are the reference's
    (grid.rs:350-366, :378-413, :461-475, :783-788); the Bound column renders through
    fdc_render_bounded on the F64 / Fixed tiers, the Stripe column through
    fdc_render_stripe (declined, for a CPU restart, with the Bound column or a series start).
    deadline_ms: the device stops taking samples once it has passed; if any sample is
    left, Incomplete carries the finished ones and the mask of those the CPU must render.
    """
    started = time.perf_counter()
    striped = "stripe" in p.columns
    if striped and not (1 <= p.stripe_window <= 64 and math.isfinite(p.stripe_freq)):  # grid.rs:783-788
        raise ValueError("stripe window must be 1..=64 and the frequency finite")
    bound = "bound" in p.columns
    if striped and (bound or series is not None):
        raise Declined("frame declined (stripe with bound or a series start); CPU restart from zero")
    if bound and bla is not None:  # grid.rs:379-384
        raise ValueError("--columns bound certifies every step; BLA remainders are not certified (ACC-02)")
    if bound and series is not None:  # grid.rs:354
        raise ValueError("a series start needs f64 deltas and no Bound column")
    if bound and host_encode:
        raise ValueError("the host encoder writes heuristic columns only: render the Bound column on the device")
    plane, tier = _setup(view, p)
    need = 53 if tier == 0 else plane.bits
    t = time.perf_counter()
    if orbit is None:
        r, bits = reference(view, p)
    else:
        r, bits = orbit
        if bits != need and (tier == 0 or bits < need):
            at_least = "" if tier == 0 else "at least "
            raise ValueError(f"supplied reference has {bits} bits; this view needs {at_least}{need}")
        if len(r) == 0 or len(r.re) != len(r.im) or r.re[0] != 0.0 or r.im[0] != 0.0:
            raise ValueError("supplied reference orbit must start at Z_0 = 0 with equal re/im lengths")
        plane.bits = bits
    r.bits = bits
    reference_seconds = time.perf_counter() - t
    if bla is not None and bla.points != len(r):
        raise ValueError(f"BLA table covers a {bla.points}-point orbit, not this {len(r)}-point one")
    on_device = isinstance(bla, DeviceTable)
    if on_device and (bound or series is not None):
        raise ValueError("a device-built table serves the BLA kernel only (no Bound column, no series start)")
    # A table without levels skips nothing: its samples are the plain kernel's, so it is not
    # uploaded; the header and BlaStats stay render_bla's (grid.rs:526-529), and its
    # refusals (grid.rs:392-411), which the device checks for uploaded tables, are checked here.
    table = bla if bla is not None and (on_device or bla.levels > 0) else None
    if bla is not None and table is None:
        _check_bla_escape_radius(p.escape_radius)
        dc, e = bla_dc_bound(view, p)
        over = dc > bla.dc_max if e == bla.dc_exp else \
            math.log2(dc) + e > math.log2(bla.dc_max) + bla.dc_exp
        if math.isnan(dc) or over:
            raise ValueError("view reaches |dc| beyond the BLA table's dc_max")
    if series is not None:
        if tier == 2:
            raise ValueError("a series start needs f64 deltas and no Bound column")
        if series.points != len(r):
            raise ValueError("series built over another orbit")
        dc = plane.h() * math.hypot(p.nx / 2.0, p.ny / 2.0)
        if math.isnan(dc) or dc > series.rho:
            raise ValueError(f"view reaches |dc| = {dc:e}, beyond the series radius {series.rho:e}")
    dev = dev or device(0)
    h = dev.upload(r, None if on_device else table)
    try:
        if on_device:  # built over the uploaded orbit; without levels it skips nothing, as above
            bla.levels = dev.build_bla(h, bla.eps, bla.dc_max, bla.dc_exp)
            steps = max(len(r) - 2, 0)
            bla.blocks = sum(steps >> (i + 1) for i in range(bla.levels))
            table = bla if bla.levels > 0 else None
        flags = (_lib.DERIVATIVE if p.needs_derivative() or (bound and tier != 2) else 0) | \
            (_lib.BLA if table is not None else 0)
        if series is not None:
            dev.upload_series(h, series)
            flags |= _lib.SERIES
        if bound and tier != 2:  # grid.rs:588-593: the ordinary tiers' error radii
            dev.upload_error_radius(h, r.error_radius(None if tier == 0 else bits, plane.c_re, plane.c_im))
        if table is not None and shift and p.needs_derivative():
            flags |= _lib.SHIFT
        job = make_job(plane, tier, p, h, r.nucleus_period(), flags)
        if deadline_ms:
            job.deadline_ms = float(deadline_ms)
        g = time.perf_counter()
        arrays, cnt, status = dev.render_job(job, raw=raw or host_encode,
                                             columns=() if host_encode else p.columns, bounded=bound,
                                             stripe=(p.stripe_window, p.stripe_freq) if striped else None)
        gpu_seconds = time.perf_counter() - g
    finally:
        dev.free(h)
    rep = report if report is not None else RouteReport()
    rep.device = f"cuda:{dev.index}"
    rep.gpu_seconds = gpu_seconds
    rep.table_blocks = 0 if bla is None else (bla.blocks if on_device else len(bla.blocks))
    return assemble(view, p, plane, tier, bla, table, series, flags, shift, host_encode, arrays, cnt, status,
                    len(r), reference_seconds, rep, started, quiet)


def _f64_div(a: float, b: float) -> float:
    """a / b as binary64 divides (grid.rs:532-533 in Rust): +-inf or NaN for b == 0, where
    h underflows on the deepest views, instead of Python's ZeroDivisionError."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return float(np.float64(a) / np.float64(b))


def assemble(view: View, p: Params, plane: Plane, tier: int, bla: Optional[Bla], table: Optional[Bla],
             series: Optional["Series"], flags: int, shift: bool, host_encode: bool, arrays: dict,
             cnt: "_lib.Counters", status: int, reference_len: int, reference_seconds: float, rep: RouteReport,
             started: float, quiet: bool = True):
    """The route's result from one fdc_render (its arrays, counters and status): header,
    samples, Stats and BlaStats as render_with returns them, the report's counters, and on
    FDC_TIMEOUT the Incomplete restart contract (frame.rs:338-341)."""
    bound = "bound" in p.columns
    kernel = plane.kernel(tier) + (" bla/1" if bla is not None else "") + (" series/0" if series is not None else "") \
        + " gpu-perturb-cuda/1"
    cols = ("class",) + tuple(c for c in ("nu", "de", "normal") if c in p.columns) + \
        (("bound",) if bound else ()) + (("stripe",) if "stripe" in p.columns else ())
    header = Header(cols, p.nx, p.ny, p.ss, p.max_iter, p.escape_radius, view, kernel)
    s = Samples(cls=arrays["cls"], nu=arrays.get("nu"), de=arrays.get("de"), normal=arrays.get("normal"),
                n=arrays.get("n"), z=arrays.get("z"), dz=arrays.get("dz"), dexp=arrays.get("dexp"),
                status=arrays.get("status"), bound=arrays.get("bound"), ez=arrays.get("ez"), ed=arrays.get("ed"),
                stripe=arrays.get("stripe"))
    if host_encode:
        encode_host(plane, p.ss, s, p.columns, p.threads)
    unfinished = None
    if status == _lib.TIMEOUT:
        unfinished = arrays["status"] == 0
        for col in (s.nu, s.de, s.normal):  # the host encoder's values of unwritten samples
            if col is not None:
                col[unfinished] = 0
    stats = Stats(reference_len, reference_seconds, int(cnt.iterations))
    bstats = None
    if table is not None:
        bstats = BlaStats(int(cnt.blocks), int(cnt.skipped), int(cnt.fallback_samples),
                          int(cnt.closed_form_samples),
                          _f64_div(cnt.shift, plane.h() * p.ss) if (flags & _lib.SHIFT) else None)
    elif bla is not None:  # no block anywhere: closed-form interiors, every other sample a fallback
        closed = int((((arrays["cls"] & 3) == 1) & (arrays["n"] == 0) & (arrays["status"] != 0)).sum())
        bstats = BlaStats(0, 0, int(cnt.samples) - closed, closed,
                          0.0 if (shift and p.needs_derivative()) else None)
    rep.accepted = int(cnt.samples)
    rep.fallback = p.nx * p.ny - int(cnt.samples)
    rep.kernel_ms = cnt.kernel_ms
    rep.launches = cnt.launches
    rep.total_seconds = time.perf_counter() - started
    if not quiet:
        print(rep.line(stats, bstats), file=sys.stderr)
    if unfinished is not None:
        raise Incomplete(f"deadline passed with {rep.fallback} samples unfinished; CPU restart of those from zero",
                         header, s, stats, bstats, unfinished)
    return header, s, stats, bstats


def render(view: View, p: Params, orbit=None, **kw):
    """perturb_gpu::render (frame.rs:70-76) on the CUDA route: plain perturbation."""
    h, s, st, _ = render_with(view, p, orbit, None, **kw)
    return h, s, st


def render_series(view: View, p: Params, orbit, series: "Series", bla: Optional[Bla] = None, **kw):
    """fd_kernel::render_series (grid.rs:213-226) on the CUDA route: every sample starts at
    the series' admitted iterate, and a sample that ends unresolved from there retries from
    zero. Returns (Header, Samples, Stats, BlaStats or None)."""
    return render_with(view, p, orbit, bla, series=series, **kw)


def render_bla(view: View, p: Params, orbit=None, eps: float = EPS, device_table: bool = False, **kw):
    """perturb_gpu::render_bla (frame.rs:78-84) on the CUDA route: the reference orbit
    (computed unless supplied) and a BLA table built over it for the view's largest |dc|
    (control.rs:344-360), then the BLA kernel. The table is the CPU builder's, or with
    device_table the same table built on the GPU over the uploaded orbit (fdc_build_bla)."""
    if orbit is None:
        orbit = reference(view, p)
    _check_bla_escape_radius(p.escape_radius)
    dc, e = bla_dc_bound(view, p)
    if device_table:
        if not (0.0 < eps <= 2.0 ** -24 and 0.0 < dc < math.inf):  # bla.rs:26-33, the host builder's refusal
            raise ValueError("BLA needs 0 < eps <= 2^-24 and a finite dc_max > 0")
        return render_with(view, p, orbit, DeviceTable(eps, dc, e, len(orbit[0])), **kw)
    t = time.perf_counter()
    table = Bla.build_scaled(orbit[0], eps, dc, e, p.threads)
    report = kw.pop("report", None) or RouteReport()
    report.table_seconds = time.perf_counter() - t
    return render_with(view, p, orbit, table, report=report, **kw)
