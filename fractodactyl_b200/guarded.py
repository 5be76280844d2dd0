"""The reference's admission pieces for approximate GPU results, on the host: the guarded
BLA table (crates/fd-kernel/src/bla/guarded.rs:1-134), the escaped-state guard
(external_escape_ok, store.rs:152-198) and the overlay of admitted escaped states onto a
CPU render (overlay_escaped, grid.rs:120-171).

The CUDA route iterates the reference's algorithm exactly, so it admits every finished
sample without them; they serve callers that keep the reference's guarded route, whose
GPU states carry error radii, and the overlay is the merge step of that route's CPU
restart.
"""
import ctypes as C
import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import lib
from .route import Params, Reference, Samples, View, _setup


@dataclasses.dataclass
class GuardedBla:
    """GuardedBla (guarded.rs:102-109): level-major [f64; 9] blocks (a.re, a.im, b.re, b.im,
    r, alpha, beta, derivative alpha, derivative beta) and the level offsets."""
    blocks: np.ndarray  # (n, 9)
    level_offsets: np.ndarray  # levels + 1
    dc_max: float

    @property
    def levels(self) -> int:
        return len(self.level_offsets) - 1

    def level(self, i: int) -> np.ndarray:
        return self.blocks[self.level_offsets[i]:self.level_offsets[i + 1]]

    @classmethod
    def build(cls, r: Reference, q: Sequence[float], eps: float, dc_max: float) -> "GuardedBla":
        """GuardedBla::build (guarded.rs:110-134) over the orbit with its reference radii q
        (one per point, finite and nonnegative)."""
        re, im = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
        qa = np.ascontiguousarray(q, dtype=np.float64)
        if len(qa) != len(re):
            raise ValueError("guarded BLA needs one finite nonnegative reference radius per point")
        cap = max(len(re) - 2, 1)
        out = np.empty((cap, 9))
        offs = np.empty(65, np.uint64)
        levels, blocks = C.c_uint32(), C.c_uint64()
        if lib().fdh_guarded_bla_build(re.ctypes.data, im.ctypes.data, qa.ctypes.data, len(re), eps, dc_max,
                                       out.ctypes.data, cap, offs.ctypes.data, 65, C.byref(levels),
                                       C.byref(blocks)) != 0:
            raise ValueError(_lib.host_error())
        return cls(out[:blocks.value].copy(), offs[:levels.value + 1].copy(), dc_max)


@dataclasses.dataclass
class EscapedState:
    """EscapedState (grid.rs:110-118): an externally computed escaped sample."""
    n: int
    z: Tuple[float, float]
    derivative: Tuple[float, float]
    derivative_exponent: int


def external_escape_ok(s: EscapedState, ez: float, ed: float, pixel: Tuple[float, int]) -> bool:
    """external_escape_ok (store.rs:152-198): whether the state, with error radii ez on z
    and ed on the derivative mantissa, encodes within half the comparison budget for the
    output pixel (mantissa, exponent)."""
    return bool(lib().fdh_external_escape_ok(int(s.n), float(s.z[0]), float(s.z[1]), float(s.derivative[0]),
                                             float(s.derivative[1]), int(s.derivative_exponent), float(ez),
                                             float(ed), float(pixel[0]), int(pixel[1])))


def overlay_escaped(view: View, p: Params, samples: Samples, states: List[Optional[EscapedState]]) -> None:
    """overlay_escaped (grid.rs:120-171): the admitted escaped states encoded through the
    CPU renderer's column encoder (here fdh_encode, the host's libm) into `samples`; every
    other sample keeps what it holds. Refused for the Bound and Stripe columns, a grid
    that does not match, and a state that is not a valid escape."""
    n = p.nx * p.ny
    if "bound" in p.columns or "stripe" in p.columns or len(states) != len(samples.cls) or len(states) != n:
        raise ValueError("escaped overlay needs a matching sample grid without bound or stripe columns")
    plane, _ = _setup(view, p)
    idx = [k for k, s in enumerate(states) if s is not None]
    for k in idx:
        s = states[k]
        zr, zi = s.z
        dr, di = s.derivative
        if (s.n > p.max_iter or not math.isfinite(zr) or not math.isfinite(zi)
                or np.hypot(zr, zi) <= p.escape_radius or not math.isfinite(dr) or not math.isfinite(di)
                or np.hypot(dr, di) == 0.0):
            raise ValueError("escaped overlay received an invalid state")
    if not idx:
        return
    m = len(idx)
    cls = np.zeros(m, np.uint8)  # Escaped with heuristic evidence (infinite radii prove nothing)
    nn = np.array([states[k].n for k in idx], np.uint32)
    z = np.array([states[k].z for k in idx], np.float64)
    dz = np.array([states[k].derivative for k in idx], np.float64)
    dexp = np.array([states[k].derivative_exponent for k in idx], np.int64)
    nu = np.zeros(m) if samples.nu is not None else None
    de = np.zeros(m, np.float32) if samples.de is not None else None
    normal = np.zeros(m, np.uint16) if samples.normal is not None else None
    ptr = lambda a: None if a is None else a.ctypes.data
    lib().fdh_encode(C.byref(plane._c()), p.ss, m, ptr(cls), ptr(nn), ptr(z), ptr(dz), ptr(dexp), ptr(nu), ptr(de),
                     ptr(normal), 1)
    sel = np.array(idx)
    samples.cls[sel] = cls
    for col, vals in ((samples.nu, nu), (samples.de, de), (samples.normal, normal)):
        if col is not None:
            col[sel] = vals
