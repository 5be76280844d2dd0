"""The reference's admission pieces on the host (fractodactyl_b200/guarded.py), on the CPU:

- GuardedBla::build (crates/fd-kernel/src/bla/guarded.rs:110-134) equals a plain-Python
  restatement of guarded.rs:8-134 bit for bit, on the reference test's three views with
  both of its eps values;
- the reference's own envelope test restated (guarded.rs:139-210): for every 17th valid block
  of every level, direct binary64 iteration over the block from delta = (0.9 r, 0.05 r),
  dc = (0.3 c, -0.2 c) and dz/dc = (0.7, -0.3) stays within the block's state and
  derivative envelopes plus the direct recurrence's own rounding; more than 500 blocks are
  checked and the state envelope alone misses derivative cases; the refusals;
- external_escape_ok (store.rs:152-198): a well-escaped state with small radii passes, and
  large, negative or non-finite radii and an unproven escape fail;
- overlay_escaped (grid.rs:120-171): the escaped states of an oracle render overlaid onto a
  zeroed frame give the oracle's class, nu, de and normal bytes; its refusals.
"""
import ctypes as C
import math
import sys

import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import guarded

EPS64 = sys.float_info.epsilon
_libm = C.CDLL("libm.so.6")
_libm.hypot.restype = C.c_double
_libm.hypot.argtypes = [C.c_double, C.c_double]
hypot = _libm.hypot  # the platform hypot, as Rust's f64::hypot
VIEWS = [(-0.743643887037158, 0.131825904205312, 1e-28), (-0.7453, 0.1127, 1e-24), (0.25, 0.0, 1e-24)]
EPS_VALUES = [fd.EPS_MAX, 2.0 ** -50]


# ---- plain-Python restatement of guarded.rs (test oracle) ----
def norm(z):
    return abs(z[0]) + abs(z[1])


def up(x):
    return x * (1.0 + 64.0 * EPS64) + sys.float_info.min


def affine(x, a, b):  # bla.rs:124-129
    return (a[0] * x[0] - a[1] * x[1] + b[0] + 0.0, a[0] * x[1] + a[1] * x[0] + b[1] + 0.0)


ZERO = ((0.0, 0.0), (0.0, 0.0), 0.0, 0.0, 0.0, 0.0, 0.0)  # a, b, r, alpha, beta, da, db


def single(z, q, eps):  # Block::single (bla.rs:72-85), GuardedBlock::single (guarded.rs:35-50)
    az = hypot(z[0], z[1])
    r = 2.0 * eps * az
    if not (r > 0.0 and az <= 2.0):
        return ZERO
    if not math.isfinite(q) or q < 0.0 or norm(z) + q > 2.0:
        return ZERO
    return ((2.0 * z[0] + 0.0, 2.0 * z[1] + 0.0), (1.0, 0.0), r, up(r + 2.0 * q), 0.0, up(2.0 * r + 2.0 * q), 0.0)


def rmin(a, b):  # f64::min ignores a NaN operand
    return b if math.isnan(a) else (a if math.isnan(b) else min(a, b))


def remainder(ay, ax, bx, xa, xb, ya, yb):  # guarded.rs:14-19
    return up(ay * xa + ya * (ax + xa)), up(ay * xb + ya * (bx + xb) + yb)


def merge(x, y, c):  # guarded.rs:51-98
    (xa_, xb_, xr, xal, xbe, xda, xdb), (ya_, yb_, yr, yal, ybe, yda, ydb) = x, y
    if xr == 0.0 or yr == 0.0:
        return ZERO
    ax, ay, bx = norm(xa_), norm(ya_), norm(xb_)
    r = rmin(xr, (yr - up((bx + xbe) * c)) / up(ax + xal)) * (1.0 - 64.0 * EPS64)
    a, b = affine(xa_, ya_, (0.0, 0.0)), affine(xb_, ya_, yb_)
    ra = up(32.0 * EPS64 * ay * ax)
    rb = up(32.0 * EPS64 * (ay * bx + norm(yb_)))
    alpha, beta = remainder(ay, ax, bx, xal, xbe, yal, ybe)
    da, db = remainder(ay, ax, bx, xda, xdb, yda, ydb)
    z = (a, b, r, up(alpha + ra), up(beta + rb), up(da + ra), up(db + rb))
    vals = [*a, *b, r, z[3], z[4], z[5], z[6]]
    return z if r > 0.0 and all(math.isfinite(v) for v in vals) else ZERO


def build(r, q, eps, c):  # guarded.rs:110-134
    nxt = [single((r.re[k], r.im[k]), q[k], eps) for k in range(1, len(r.re) - 1)]
    levels = []
    while True:
        nxt = [merge(nxt[2 * t], nxt[2 * t + 1], c) for t in range(len(nxt) // 2)]
        if not any(b[2] > 0.0 for b in nxt):
            return levels
        levels.append(nxt)


def as9(b):
    a, bb, r, alpha, beta, da, db = b
    return [a[0], a[1], bb[0], bb[1], r, alpha, beta, da, db]


@pytest.mark.parametrize("view", VIEWS, ids=lambda v: f"{v[2]:g}")
@pytest.mark.parametrize("eps", EPS_VALUES, ids=["eps-max", "eps-2^-50"])
def test_guarded_table_equals_restatement(view, eps):
    cr, ci, c = view
    r = fd.Reference.new(cr, ci, 10000, 1e10)
    q = r.error_radius(None, cr, ci)  # the orbit's own radii, which diverge near its escape
    q = np.where(np.isfinite(q), q, 1.0)
    got = guarded.GuardedBla.build(r, q, eps, c)
    want = build(r, q, eps, c)
    assert got.levels == len(want) and got.levels > 0
    for i, level in enumerate(want):
        mine = got.level(i)
        assert mine.shape == (len(level), 9)
        assert np.array_equal(mine.view(np.uint64), np.array([as9(b) for b in level]).view(np.uint64)), i


def test_guarded_envelopes_bound_direct_iteration():
    """guarded.rs:139-210 restated: zero reference radii, both eps, three views."""
    checked = naive_misses = 0
    worst = 0.0
    for cr, ci, c in VIEWS:
        r = fd.Reference.new(cr, ci, 10000, 1e10)
        q = np.zeros(len(r.re))
        for eps in EPS_VALUES:
            t = guarded.GuardedBla.build(r, q, eps, c)
            for j in range(t.levels):
                level = t.level(j)
                for i in range(0, len(level), 17):
                    ar, ai, br, bi, rr, alpha, beta, dalpha, dbeta = level[i]
                    if not rr > 0.0:
                        continue
                    m, length = 1 + (i << (j + 1)), 2 << j
                    delta, dc, initial_d = (0.9 * rr, 0.05 * rr), (0.3 * c, -0.2 * c), (0.7, -0.3)
                    d, derivative = delta, initial_d
                    for k in range(m, m + length):
                        z = (r.re[k] + d[0], r.im[k] + d[1])
                        derivative = affine(derivative, (2.0 * z[0], 2.0 * z[1]), (1.0, 0.0))
                        d = affine(d, (2.0 * r.re[k] + d[0], 2.0 * r.im[k] + d[1]), dc)
                    approximate = affine(initial_d, (ar, ai), (br, bi))
                    err = hypot(derivative[0] - approximate[0], derivative[1] - approximate[1])
                    bound = dalpha * norm(initial_d) + dbeta
                    rnd = 64.0 * EPS64 * length * (norm(derivative) + norm(approximate))
                    assert err <= bound + rnd, (m, length, err, bound, rnd)
                    state = affine(delta, (ar, ai), (br * dc[0] - bi * dc[1], br * dc[1] + bi * dc[0]))
                    serr = hypot(d[0] - state[0], d[1] - state[1])
                    sb = alpha * norm(delta) + beta * norm(dc)
                    assert serr <= sb + 64.0 * EPS64 * length * (norm(d) + norm(state))
                    naive_misses += err > alpha * norm(initial_d) + beta
                    worst = max(worst, err / (bound + rnd))
                    checked += 1
    assert checked > 500, checked
    assert naive_misses > 0, "the state-only envelope must miss derivative cases"
    r = fd.Reference.new(0.25, 0.0, 20, 1e10)
    with pytest.raises(ValueError, match="radius per point"):
        guarded.GuardedBla.build(r, [], 2.0 ** -50, 1e-20)
    with pytest.raises(ValueError, match="radius per point"):
        guarded.GuardedBla.build(r, np.full(len(r.re), np.nan), 2.0 ** -50, 1e-20)
    with pytest.raises(ValueError, match="eps"):
        guarded.GuardedBla.build(r, np.zeros(len(r.re)), 2.0 ** -20, 1e-20)


def test_external_escape_guard():
    s = guarded.EscapedState(n=120, z=(3.0e5, -1.0e5), derivative=(2.0e40, 1.0e40), derivative_exponent=0)
    pixel = (1.25, -60)
    assert guarded.external_escape_ok(s, 1e-12, 1e28, pixel)
    assert not guarded.external_escape_ok(s, 1e3, 1e28, pixel)          # |z| radius too large for nu
    assert not guarded.external_escape_ok(s, 1e-12, 5e39, pixel)         # derivative radius too large
    for ez, ed in ((-1.0, 0.0), (0.0, -1.0), (math.nan, 0.0), (0.0, math.inf)):
        assert not guarded.external_escape_ok(s, ez, ed, pixel)
    small = guarded.EscapedState(n=5, z=(1.5, 0.5), derivative=(3.0, 1.0), derivative_exponent=0)
    assert not guarded.external_escape_ok(small, 0.0, 0.0, pixel)       # |z| - ez <= 2 proves no escape
    assert guarded.external_escape_ok(s, 0.0, 0.0, pixel)


def test_overlay_escaped_gives_the_cpu_columns():
    view3 = ("-0.7453", "0.1127", "0.0065")
    v = fd.View(*view3)
    p = fd.Params(40, 24, max_iter=3000, columns=("nu", "de", "normal"))
    plane, tier = fd.route._setup(v, p)
    job = fdref.make_job(*view3, p.nx, p.ny, p.max_iter, escape_radius=p.escape_radius,
                         columns=fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL, tier=tier, threads=1)
    ref = fdref.Ref.for_job(job)
    want = fdref.render(job, ref, None, raw=True)
    n = p.nx * p.ny
    esc = (want["cls"] & 3) == 0
    assert esc.any() and not esc.all()
    states = [guarded.EscapedState(int(want["n"][k]), tuple(want["z"][k]), tuple(want["dz"][k]), int(want["dexp"][k]))
              if esc[k] else None for k in range(n)]
    s = fd.Samples(cls=np.full(n, 7, np.uint8), nu=np.zeros(n), de=np.zeros(n, np.float32),
                   normal=np.zeros(n, np.uint16))
    guarded.overlay_escaped(v, p, s, states)
    assert np.array_equal(s.cls[esc], want["cls"][esc]) and np.all(s.cls[~esc] == 7)
    assert np.array_equal(s.nu[esc].view(np.uint64), want["nu"][esc].view(np.uint64))
    assert np.array_equal(s.de[esc].view(np.uint32), want["de"][esc].view(np.uint32))
    assert np.array_equal(s.normal[esc], want["normal"][esc])
    assert not s.nu[~esc].any()
    with pytest.raises(ValueError, match="matching sample grid"):
        guarded.overlay_escaped(v, p, s, states[:-1])
    pb = fd.Params(40, 24, max_iter=3000, columns=("nu", "bound"))
    with pytest.raises(ValueError, match="matching sample grid"):
        guarded.overlay_escaped(v, pb, s, states)
    bad = list(states)
    k = int(np.flatnonzero(esc)[0])
    bad[k] = guarded.EscapedState(states[k].n, (1.0, 0.0), states[k].derivative, states[k].derivative_exponent)
    with pytest.raises(ValueError, match="invalid state"):
        guarded.overlay_escaped(v, p, s, bad)
