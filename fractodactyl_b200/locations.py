"""Seeded synthetic benchmark locations (no public dataset is involved).

Frames of the five benchmark configurations: view, grid, iteration cap, escape radius,
columns, tier and BLA tolerance. Deep centres come from fdh_location (include/fdhost.h):
a Misiurewicz point near the seeded start -0.743643887 + 0.131825904i + U(-1e-9, 1e-9)^2,
then the ladder nucleus next to it whose size is about width/30, found by the ball
period and Newton in fixed point at the stated precision.

The recipe takes minutes per centre beyond ~1e-300 (about 5 at 1e-1000), so the centres
of configurations 2-5 are computed once by `python -m fractodactyl_b200.locations
--write` (all cores) into locations.json beside this file and read from there; the same
command with --check recomputes and compares them.
"""
import ctypes as C
import dataclasses
import json
import math
import os
from typing import Dict, List, Optional

import numpy as np

from . import _lib
from .route import EPS, Params, View

SEAHORSE = (-0.743643887, 0.131825904)


@dataclasses.dataclass
class Frame:
    name: str
    view: View
    params: Params
    bla_eps: Optional[float]
    period: Optional[int] = None
    log10_size_over_width: Optional[float] = None


def seeded_start(seed: int):
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1e-9, 1e-9, size=2)
    theta = float(rng.uniform(0.0, 2.0 * math.pi))
    return "%.22f" % (SEAHORSE[0] + u[0]), "%.22f" % (SEAHORSE[1] + u[1]), theta


def nucleus(seed: int, log10_width: float, bits: int, max_period: int = 2_000_000):
    """(re, im, period, log10(size/width)) of the seeded ladder nucleus for this width."""
    re_, im_, theta = seeded_start(seed)
    ro, io = C.create_string_buffer(1 << 16), C.create_string_buffer(1 << 16)
    per, rel = C.c_uint64(), C.c_double()
    if _lib.lib().fdh_location(re_.encode(), im_.encode(), theta, float(log10_width), bits, max_period, ro, io,
                               1 << 16, C.byref(per), C.byref(rel)) != 0:
        raise RuntimeError("location recipe failed: " + _lib.host_error())
    return ro.value.decode(), io.value.decode(), int(per.value), float(rel.value)


def config1() -> Frame:
    """Plain perturbation, FP64 deltas, no BLA: 480x270, 1e-12 wide, 20,000 iterations,
    bailout 2^8; escape count, smooth iteration and class."""
    return Frame("c1-480x270-1e-12", View("-0.7436438870371587", "0.1318259042053120", "1e-12"),
                 Params(480, 270, max_iter=20_000, escape_radius=256.0, columns=("nu",)), None)


def config2(seed: int = 2, nx: int = 1920, ny: int = 1080, tier: Optional[str] = "scaled") -> Frame:
    """Plain perturbation + BLA with floatexp deltas: 1920x1080 at the seeded 400-bit ladder
    nucleus, 1e-100 wide, 1,000,000 iterations, BLA table from the CPU builder (eps 2^-50).
    The benchmark seed's centre is read from locations.json; other seeds are computed."""
    hit = [d for d in cached("c2") if d["seed"] == seed] if os.path.exists(CACHE) else []
    if hit:
        re_, im_, p, rel = hit[0]["re"], hit[0]["im"], hit[0]["period"], hit[0]["log10_size_over_width"]
    else:
        re_, im_, p, rel = nucleus(seed, -100.0, C2_BITS)
    return Frame(f"c2-{nx}x{ny}-1e-100-seed{seed}", View(re_, im_, "1e-100"),
                 Params(nx, ny, max_iter=1_000_000, escape_radius=1e10, columns=("nu", "de", "normal"), tier=tier),
                 EPS, p, rel)


CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "locations.json")
C2_BITS = 400  # configuration 2's stated precision for its nucleus


def centre_bits(log10_width: float) -> int:
    """Fixed-point precision of a nucleus for a view this wide: 128 bits above the width
    plus 64 of margin."""
    return 128 + int(math.ceil(-log10_width * math.log2(10.0))) + 64


def specs() -> Dict[str, List[dict]]:
    """The seeded centres the configurations need: C2 the 1e-100 nucleus at 400 bits (seed
    2); C3 one nucleus 1e-300 wide (seed 3); C4 one nucleus for the deepest film frame,
    1e-500 (seed 4); C5 32 nuclei with widths log-uniform on [1e-1000, 1e-20] (seeds
    5000 + k). Configuration 1's centre is given as a decimal and needs no recipe."""
    rng = np.random.default_rng(5)
    c5 = [dict(seed=5000 + k, log10_width=float(w)) for k, w in enumerate(rng.uniform(-1000.0, -20.0, 32))]
    out = {"c3": [dict(seed=3, log10_width=-300.0)], "c4": [dict(seed=4, log10_width=-500.0)], "c5": c5}
    for v in out.values():
        for d in v:
            d["bits"] = centre_bits(d["log10_width"])
    return {"c2": [dict(seed=2, log10_width=-100.0, bits=C2_BITS)], **out}


def _compute(d):
    re_, im_, per, rel = nucleus(d["seed"], d["log10_width"], d["bits"])
    return dict(d, re=re_, im=im_, period=per, log10_size_over_width=rel)


def generate(processes: int = 0) -> Dict[str, List[dict]]:
    import multiprocessing as mp
    sp = specs()
    flat = [(k, d) for k, v in sp.items() for d in v]
    flat.sort(key=lambda kd: kd[1]["log10_width"])  # deepest (slowest) first
    with mp.get_context("spawn").Pool(processes or os.cpu_count() or 1) as pool:
        done = pool.map(_compute, [d for _, d in flat], chunksize=1)
    out: Dict[str, List[dict]] = {k: [] for k in sp}
    for (k, _), d in zip(flat, done):
        out[k].append(d)
    for k in out:
        out[k].sort(key=lambda d: d["seed"])
    return out


def cached(name: str) -> List[dict]:
    if not os.path.exists(CACHE):
        raise FileNotFoundError(f"{CACHE} is missing: run python -m fractodactyl_b200.locations --write")
    with open(CACHE) as f:
        return json.load(f)[name]


def film_widths(frames: int = 60, first: float = -10.0, last: float = -500.0) -> List[str]:
    """Geometric widths from 10^first to 10^last, as decimal strings."""
    return [_decimal(first + (last - first) * k / (frames - 1)) for k in range(frames)]


def _decimal(log10_value: float) -> str:
    """10^log10_value as a decimal string with 7 significant digits."""
    e = math.floor(log10_value)
    return "%.6fe%d" % (10 ** (log10_value - e), e)


def config3(nx: int = 3840, ny: int = 2160, spp: int = 4) -> Frame:
    """Precision form: 3840x2160 pixels with `spp` seeded jittered samples each (a 2x2 grid
    of samples per pixel, each moved by U[-1/2, 1/2)^2 of a sample spacing; jitter_offsets
    gives them), at the seed-3 nucleus, 1e-300 wide, 5,000,000 iterations, BLA and the
    distance-estimate derivative on."""
    d = cached("c3")[0]
    ss = int(round(math.sqrt(spp)))
    return Frame(f"c3-{nx}x{ny}x{spp}-1e-300", View(d["re"], d["im"], "1e-300"),
                 Params(nx * ss, ny * ss, ss=ss, max_iter=5_000_000, escape_radius=1e10,
                        columns=("nu", "de", "normal"), tier="scaled"),
                 EPS, d["period"], d["log10_size_over_width"])


def jitter_offsets(plane, nx: int, ny: int, seed: int = 3) -> np.ndarray:
    """Per-sample (ux, uy) of a jittered sample grid: the grid offset of view.rs:118-122
    with x, y moved by seeded U[-1/2, 1/2) each (the reference has no jitter; its grid is
    the zero-jitter case)."""
    rng = np.random.default_rng(seed)
    i = np.arange(nx, dtype=np.float64)
    j = np.arange(ny, dtype=np.float64)
    x = (i[None, :] + 0.5 - nx / 2.0) + rng.uniform(-0.5, 0.5, (ny, nx))
    y = (j[:, None] + 0.5 - ny / 2.0) + rng.uniform(-0.5, 0.5, (ny, nx))
    out = np.empty((ny * nx, 2))
    out[:, 0] = (plane.cos_rot * x + plane.sin_rot * y).ravel()
    out[:, 1] = (plane.sin_rot * x - plane.cos_rot * y).ravel()
    return out


def config4(frames: int = 60, nx: int = 1280, ny: int = 720) -> List[Frame]:
    """Film: `frames` frames of nx x ny with widths geometric from 1e-10 to 1e-500 toward
    the seed-4 nucleus, 10,000,000 iterations; all frames share one reference orbit (at
    the deepest frame's precision) and one BLA table."""
    d = cached("c4")[0]
    return [Frame(f"c4-{k:02d}-{nx}x{ny}-{w}", View(d["re"], d["im"], w),
                  Params(nx, ny, max_iter=10_000_000, escape_radius=1e10, columns=("nu", "de", "normal")),
                  EPS, d["period"], None)
            for k, w in enumerate(film_widths(frames))]


def config5(tiles_per_location: int = 8, tile: int = 256, max_iter: int = 10_000_000) -> List[Frame]:
    """Mixed locations: 32 seeded nuclei, widths log-uniform on [1e-1000, 1e-20]; each
    location's frame is a (4 tile) x (2 tile) grid cut into 8 tiles of 256x256 (column and
    row windows of one frame, sharing its orbit and BLA table)."""
    out = []
    for d in cached("c5"):
        w = _decimal(d["log10_width"])
        out.append(Frame(f"c5-{d['seed']}-{w}", View(d["re"], d["im"], w),
                         Params(4 * tile, 2 * tile, max_iter=max_iter, escape_radius=1e10,
                                columns=("nu", "de", "normal")),
                         EPS, d["period"], d["log10_size_over_width"]))
    return out


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="compute the seeded centres of configurations 3-5")
    ap.add_argument("--write", action="store_true", help=f"write {CACHE}")
    ap.add_argument("--check", action="store_true", help="recompute and compare with the cached file")
    ap.add_argument("--processes", type=int, default=0)
    a = ap.parse_args()
    got = generate(a.processes)
    if a.write:
        with open(CACHE, "w") as f:
            json.dump(got, f, indent=1)
        print("wrote", CACHE)
    if a.check:
        with open(CACHE) as f:
            want = json.load(f)
        assert got == want, "cached centres differ from the recipe's"
        print("cached centres reproduced")
