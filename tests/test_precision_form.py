"""The precision form (FP32-mantissa floatexp deltas, FP64 for the rebase test, the
bailout, the BLA radii and the derivative) against the plain FP64 route and against the
fd-fixed direct-iteration oracle on a seeded subset of samples.

FP32 mantissas (24 bits) cannot follow chaotic orbits as far as FP64 does: an error of
one FP32 rounding in a delta grows by the orbit's Lyapunov factor (1e-14 -> 1e-3 within
~1,100 iterations on the 1e-12 view) and can change the escape count. The ceiling is the
arithmetic's: the oracle with its deltas and its copy of the orbit point rounded to 24
bits (an ideal FP32 recurrence, everything else binary64) agrees with itself on no more
samples, and the GPU form must come within 3% of that ceiling on every view. So the bar is set per view and the rates
are reported: on views whose samples escape before that
amplification (the 1e-300 Misiurewicz view) escape counts equal the plain route's on
>= 99.9% of samples and differ by at most one iteration elsewhere; on chaotic views at
least 75% equal and 99% agree on escaping or not. Where the counts agree, smooth
iteration agrees within 1e-6 relative on 99% of them (1e-3 on every one) on the
non-chaotic view and within 1e-5 relative on the median sample elsewhere (the same amplification moves the escaping z). Against fd-fixed
direct iteration (which the plain form follows except where FP64 perturbation itself
loses the chaotic orbit: at most 2 of 96 samples) the precision form's mismatch rate is
reported and bounded.
"""
import math

import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

pytestmark = pytest.mark.gpu
COUNT_MATCH = 0.999
NU_REL_P99 = 1e-6      # non-chaotic view, 99% of the samples whose count agrees
NU_REL_MAX = 1e-3      # non-chaotic view, every sample whose count agrees
NU_REL_MEDIAN = 1e-5   # chaotic views, median over samples whose count agrees


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def both_forms(dev, view, p, bla_eps=None):
    r, bits = fd.reference(view, p)
    r.bits = bits
    plane, tier = fd.route._setup(view, p)
    bla = None
    if bla_eps is not None:
        dc, e = fd.bla_dc_bound(view, p)
        bla = fd.Bla.build_scaled(r, bla_eps, dc, e)
        if bla.levels == 0:
            bla = None
    h = dev.upload(r, bla)
    try:
        flags = (_lib.DERIVATIVE if p.needs_derivative() else 0) | (_lib.BLA if bla is not None else 0)
        j = fd.route.make_job(plane, tier, p, h, r.nucleus_period(), flags)
        plain, cp, _ = dev.render_job(j, columns=p.columns, raw=True)
        j.flags = flags | _lib.F32
        prec, cq, _ = dev.render_job(j, columns=p.columns, raw=True)
    finally:
        dev.free(h)
    return plane, tier, plain, prec, cp, cq


def agreement(a, b):
    """Fractions of samples whose escape counts agree (both non-escaping counts as agreeing)
    and agree within one iteration."""
    n = len(a["cls"])
    ea, eb = a["cls"] == 0, b["cls"] == 0
    dn = np.abs(a["n"].astype(np.int64) - b["n"].astype(np.int64))
    same = (ea == eb) & (~ea | (dn == 0))
    off1 = (ea == eb) & (~ea | (dn <= 1))
    return same.sum() / n, off1.sum() / n


VIEWS = [
    # (re, im, width, nx, ny, max_iter, tier, chaotic)
    ("-0.7453", "0.1127", "0.0065", 256, 144, 20_000, None, True),
    ("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28", 256, 144, 50_000,
     None, True),
    ("0", "1", "1e-300", 256, 144, 20_000, None, False),
    ("-0.7436438870371587", "0.1318259042053120", "1e-12", 240, 135, 20_000, None, True),
]


def ideal_fp32(v, p, tier, bla_eps):
    """Escape-count agreement of the oracle with 24-bit deltas and a 24-bit copy of the
    orbit point each step multiplies them by (everything else binary64) with the oracle
    itself on the same frame: the ceiling of an FP32 delta recurrence there."""
    job = fdref.make_job(v.center_re, v.center_im, v.width, p.nx, p.ny, p.max_iter,
                         escape_radius=p.escape_radius, columns=fdref.COL_NU, tier=tier)
    ref = fdref.Ref.for_job(job)
    t = None
    if bla_eps is not None:
        dc, e = fdref.bla_dc_bound(job)
        t = fdref.Bla(ref, bla_eps, dc, e)
        t = t if t.levels else None
    base = fdref.render(job, ref, t)
    try:
        fdref.set_delta_bits(24, round_orbit=True)
        rounded = fdref.render(job, ref, t)
    finally:
        fdref.set_delta_bits(0)
    return agreement(base, rounded)[0]


@pytest.mark.parametrize("view", VIEWS, ids=lambda v: v[2])
@pytest.mark.parametrize("bla", [None, 2.0 ** -50])
def test_precision_form_agrees_with_plain(dev, view, bla):
    re_, im_, w, nx, ny, it, tier, chaotic = view
    v = fd.View(re_, im_, w)
    p = fd.Params(nx, ny, max_iter=it, columns=("nu", "de", "normal"), tier=tier)
    plane, tier, a, b, cp, cq = both_forms(dev, v, p, bla)
    same, off1 = agreement(a, b)
    escaping = float(((a["cls"] == 0) == (b["cls"] == 0)).mean())
    ceiling = ideal_fp32(v, p, tier, bla)
    print(f"{w} bla={bla}: counts equal {same:.6f} (ideal FP32 deltas {ceiling:.6f}), within one {off1:.6f}, "
          f"escape agreement {escaping:.6f}")
    # the kernel loses no more than sampling noise beyond the arithmetic's own ceiling
    assert same >= ceiling - 0.03, (same, ceiling)
    if chaotic:
        assert same >= 0.75 and escaping >= 0.99, (same, escaping)
    else:
        assert same >= COUNT_MATCH and off1 == 1.0, (same, off1)
    esc = (a["cls"] == 0) & (b["cls"] == 0) & (a["n"] == b["n"])
    rel = np.abs(a["nu"][esc] - b["nu"][esc]) / np.abs(a["nu"][esc])
    if rel.size:
        print(f"  nu relative error where counts agree: median {np.median(rel):.3e}, "
              f"p99 {np.quantile(rel, 0.99):.3e}, max {rel.max():.3e}")
        if chaotic:
            assert np.median(rel) <= NU_REL_MEDIAN, np.median(rel)
        else:
            assert np.quantile(rel, 0.99) <= NU_REL_P99 and rel.max() <= NU_REL_MAX, rel.max()


def test_precision_form_against_direct_iteration(dev):
    """Seeded subset of a 1e-28 frame: both forms against fd-fixed direct iteration."""
    re_, im_ = "-0.743643887037158704752191506114774", "0.131825904205311970493132056385139"
    v = fd.View(re_, im_, "1e-28")
    p = fd.Params(128, 72, max_iter=50_000, columns=("nu",))
    plane, tier, a, b, _, _ = both_forms(dev, v, p)
    rng = np.random.default_rng(7)
    idx = rng.choice(p.nx * p.ny, 96, replace=False)
    h = plane.h_m * 2.0 ** plane.h_e
    miss_a = miss_b = 0
    worst = 0.0
    for k in idx:
        i, j = int(k % p.nx), int(k // p.nx)
        x, y = i + 0.5 - p.nx / 2.0, j + 0.5 - p.ny / 2.0
        ux, uy = plane.cos_rot * x + plane.sin_rot * y, plane.sin_rot * x - plane.cos_rot * y
        n, zr, zi = fdref.direct(re_, im_, ux * h, uy * h, 0, plane.bits + 64, p.max_iter, p.escape_radius)
        for arr, which in ((a, "a"), (b, "b")):
            esc = int(arr["cls"][k]) == 0
            ok = (n is None and not esc) or (n is not None and esc and abs(int(arr["n"][k]) - n) <= 1)
            if not ok:
                if which == "a":
                    miss_a += 1
                else:
                    miss_b += 1
        if n is not None and int(b["cls"][k]) == 0 and int(b["n"][k]) == n:
            nu = n + 1 - math.log2(math.log2(math.hypot(zr, zi)))
            worst = max(worst, abs(b["nu"][k] - nu) / nu)
    print(f"direct iteration, {len(idx)} samples: plain misses {miss_a}, precision misses {miss_b}, "
          f"precision nu error {worst:.3e}")
    assert miss_a <= 2, miss_a
    assert miss_b <= 0.25 * len(idx) and worst <= 1e-4, (miss_b, worst)


def test_precision_form_on_a_deep_fixed_tier_view(dev):
    """Ordinary-tier views far below f32's range (1e-200 wide): the precision form keeps
    dc as mantissa and exponent on every tier, so its deltas grow from dc as the plain
    form's do. A dc held as one f32-scaled value would vanish here and leave samples on
    the reference orbit until max_iter."""
    from fractodactyl_b200 import locations
    c = locations.cached("c4")[0]
    v = fd.View(c["re"], c["im"], "1e-200")
    p = fd.Params(96, 54, max_iter=100_000, columns=("nu", "de"), tier="fixed")
    plane, tier, a, b, cp, cq = both_forms(dev, v, p, 2.0 ** -50)
    assert tier == 1
    same, off1 = agreement(a, b)
    escaping = float(((a["cls"] == 0) == (b["cls"] == 0)).mean())
    print(f"deep fixed tier: counts equal {same:.4f}, escape agreement {escaping:.4f}, "
          f"iterations {cp.iterations} vs {cq.iterations}")
    assert escaping >= 0.99 and same >= 0.5
    assert cq.iterations <= 2 * cp.iterations


def test_precision_form_below_f64_range(dev):
    """Scaled-tier views so deep that every delta stays below f64's range for thousands
    of iterations (1e-999, the deepest seeded mixed location): the precision form
    advances its save points as the extended tier does, its blocks stop there, and its
    samples escape with the plain form's instead of being rebased onto the reference
    orbit at its last point."""
    from fractodactyl_b200 import locations
    c = min(locations.cached("c5"), key=lambda d: d["log10_width"])
    v = fd.View(c["re"], c["im"], "1.5e-999")
    p = fd.Params(64, 32, max_iter=10_000_000, columns=("nu",), tier="scaled")
    plane, tier, a, b, cp, cq = both_forms(dev, v, p, 2.0 ** -50)
    escaping = float(((a["cls"] == 0) == (b["cls"] == 0)).mean())
    same, _ = agreement(a, b)
    print(f"1e-999: counts equal {same:.4f}, escape agreement {escaping:.4f}, "
          f"iterations {cp.iterations} vs {cq.iterations}")
    assert escaping >= 0.99
    assert cq.iterations <= 2 * cp.iterations
