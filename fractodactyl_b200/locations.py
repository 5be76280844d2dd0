"""Seeded synthetic benchmark locations (no public dataset is involved).

Frames of the five benchmark configurations: view, grid, iteration cap, escape radius,
columns, tier and BLA tolerance. Deep centres come from fdh_location (include/fdhost.h):
a Misiurewicz point near the seeded start -0.743643887 + 0.131825904i + U(-1e-9, 1e-9)^2,
then the ladder nucleus next to it whose size is about width/30, found by the ball
period and Newton in fixed point at the stated precision.
"""
import ctypes as C
import dataclasses
import math
from typing import Optional

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
    nucleus, 1e-100 wide, 1,000,000 iterations, BLA table from the CPU builder (eps 2^-50)."""
    re_, im_, p, rel = nucleus(seed, -100.0, 400)
    return Frame(f"c2-{nx}x{ny}-1e-100-seed{seed}", View(re_, im_, "1e-100"),
                 Params(nx, ny, max_iter=1_000_000, escape_radius=1e10, columns=("nu", "de", "normal"), tier=tier),
                 EPS, p, rel)
