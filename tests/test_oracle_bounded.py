"""The oracle's bounded variant (B: error radii on z and dz/dc, the Bound column and
Bounded evidence; crates/fd-kernel/src/sample.rs:221-229, 338-350, 373-377, 419-421,
reference.rs:122-148, store.rs:66-151) against the reference's own test
(error_radius_covers_the_exact_orbit, sample.rs:1041-1087: the radius covers the exact
orbit, computed here by fd-fixed direct iteration), and frame properties: the bounded
render keeps every class kind and count of the plain render, certifies most escaped
samples, and encodes de and the Bound column from the radii."""
import ctypes as C
import math

import numpy as np
import pytest

import fdref

U = 2.0 ** -53


@pytest.mark.parametrize("case", [
    ((0.375, 0.28125), (0.03125, 0.015625), ("0.40625", "0.296875")),
    ((-0.7421875, 0.0546875), (-0.0078125, 0.0078125), ("-0.75", "0.0625")),
    ((0.25, 0.0), (0.03125, 0.0078125), ("0.28125", "0.0078125")),
])
def test_error_radius_covers_the_exact_orbit(case):
    # dyadic reference and offset, so the sample point is exact; the exact orbit is the
    # 256-bit fixed-point direct iteration at that point (f64 and fixed references)
    (c0r, c0i), (ar, ai), (er, ei) = case
    r2 = 4294967296.0
    f64_ref = fdref.Ref.f64(c0r, c0i, 10_000, math.sqrt(r2))
    fx_ref = fdref.Ref.fixed(repr(c0r), repr(c0i), 256, 10_000)
    for ref, bits in ((f64_ref, None), (fx_ref, 256)):
        o = fdref.iterate_bounded(ref, bits, c0r, c0i, c=(c0r + ar, c0i + ai), ar=ar, ai=ai, max_iter=10_000, r2=r2)
        assert o["kind"] == "escaped", (case, bits)
        xr, xi = C.c_double(), C.c_double()
        n = fdref.lib().fdref_direct(er.encode(), ei.encode(), 0.0, 0.0, 0, 256, 10_000, math.sqrt(r2), C.byref(xr),
                                     C.byref(xi))
        assert n == o["n"]
        d, az = math.hypot(o["zr"] - xr.value, o["zi"] - xi.value), math.hypot(o["zr"], o["zi"])
        assert d <= o["ez"] + 4.0 * U * az, (case, bits, d, o["ez"])
        assert o["ez"] < 1e-9 * az and math.isfinite(o["ed"]), (case, bits)


def test_error_radius_recurrence():
    """reference.rs:122-148 restated in numpy for an f64 orbit: q[m] = a_m (round 0),
    a' = (a (2 s + a) + defect) (1 + 8U)."""
    ref = fdref.Ref.f64(-0.7453, 0.1127, 2_000, 1e10)
    re_, im_ = ref.arrays_()
    c_re, c_im = -0.7453, 0.1127
    q = fdref.error_radius(ref, None, c_re, c_im)
    c1 = abs(c_re) + abs(c_im)
    mp = 2.2250738585072014e-308
    a, want = 0.0, []
    for m in range(len(re_)):
        s = math.sqrt(re_[m] * re_[m] + im_[m] * im_[m]) * (1.0 + 4.0 * U)
        defect = 8.0 * U * (s * s + c1) + 2.0 * U * c1 + mp
        want.append(a)
        a = (a * (2.0 * (s + 0.0) + a) + defect) * (1.0 + 8.0 * U)
    assert np.array_equal(q, np.array(want))
    assert np.all(q >= 0) and q[-1] > q[1]  # it contracts where |Z| < 1/2 but grows overall


@pytest.mark.parametrize("view,max_iter", [(("-0.7453", "0.1127", "0.0065"), 4_000),  # F64 tier
                                           (("-0.743643887037158", "0.131825904205312", "1e-14"), 20_000)])  # Fixed
def test_bounded_frame(view, max_iter):
    cols = fdref.COL_NU | fdref.COL_DE | fdref.COL_BOUND
    job = fdref.make_job(*view, 40, 24, max_iter, columns=cols, threads=2)
    ref = fdref.Ref.for_job(job)
    assert fdref.plane(job)["tier"] in (0, 1)
    got = fdref.render_columns(job, ref)
    plain = fdref.render_columns(fdref.make_job(*view, 40, 24, max_iter, columns=fdref.COL_NU | fdref.COL_DE,
                                                threads=2), ref)
    kind = got["cls"] & 3
    if ref.nucleus_period() is None:  # the bounded variant declines only the nucleus gate
        assert np.array_equal(kind, plain["cls"] & 3)
        assert np.array_equal(got["n"], plain["n"])
    esc = kind == 0
    assert esc.sum() > 100
    bounded = got["cls"] == 4
    assert bounded.sum() > 0.5 * esc.sum()
    assert np.all((got["bound"] > 0) == bounded)
    # z, dz and nu are the plain render's; de is the plain de scaled by the lower factor
    assert np.array_equal(got["z"][esc], plain["z"][esc])
    assert np.array_equal(got["nu"][esc], plain["nu"][esc])
    assert np.all(got["de"][bounded] <= plain["de"][bounded])
    assert np.array_equal(got["de"][esc & ~bounded], plain["de"][esc & ~bounded])
    assert np.all(np.isinf(plain["ez"][esc]))
    # the radii grow with the orbit's instability and may overflow on long samples, which
    # then stay heuristic; every bounded sample has finite radii
    assert np.all(np.isfinite(got["ez"][bounded]) & np.isfinite(got["ed"][bounded]))


def test_bound_column_refuses_bla():
    job = fdref.make_job("-0.7453", "0.1127", "0.0065", 16, 8, 2_000, columns=fdref.COL_NU | fdref.COL_BOUND)
    ref = fdref.Ref.for_job(job)
    dc, e = fdref.bla_dc_bound(job)
    bla = fdref.Bla(ref, 2.0 ** -50, dc, e)
    with pytest.raises(ValueError, match="not certified"):
        fdref.render_columns(job, ref, bla)
