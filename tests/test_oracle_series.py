"""The oracle's parameter-series start (crates/fd-kernel/src/series.rs) against the
reference's own series tests (series.rs:606-753), restated on the oracle: the evaluated
start stays within its carried bounds of direct f64 perturbation; a frame started from
the series keeps every class and moves nu by less than 1e-3 px; a masked render reuses
the same start; no admitted prefix is the plain render; and an unresolved series start
retries from zero, so a nucleus-centred frame keeps its interior samples."""
import json
import math
import os

import numpy as np

import fdref

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kats.json")))


def test_start_is_within_its_bounds_of_direct_iteration():
    # series.rs:606-642
    r = fdref.Ref.f64(-0.743643887037158, 0.131825904205312, 20_000, 1e10)
    rho, pixel = 1e-11, 1e-13
    s = fdref.Series(r, rho, pixel, 20_000)
    info = s.info()
    assert info["n"] > 100, info
    assert info["shift_px"] <= 1e-8
    re_, im_ = r.arrays_()
    for ar, ai in [(rho, 0.0), (0.0, -rho), (0.6 * rho, 0.7 * rho), (1e-3 * rho, 0.0)]:
        xr = xi = dr = di = 0.0
        for m in range(info["n"]):
            zr, zi = re_[m] + xr, im_[m] + xi
            dr, di = 2.0 * (zr * dr - zi * di) + 1.0, 2.0 * (zr * di + zi * dr)
            wr, wi = re_[m], im_[m]
            xr, xi = (2.0 * (wr * xr - wi * xi) + xr * xr - xi * xi + ar,
                      2.0 * (wr * xi + wi * xr) + 2.0 * xr * xi + ai)
        sr, si, sdr, sdi = s.eval(ar, ai)
        assert math.hypot(sr - xr, si - xi) <= info["state_bound"] + 1e-9 * math.hypot(xr, xi), (ar, ai)
        assert math.hypot(sdr - dr, sdi - di) <= info["derivative_bound"] / rho + 1e-9 * math.hypot(dr, di), (ar, ai)


def _job(re_, im_, width, nx, ny, max_iter, columns):
    return fdref.make_job(re_, im_, width, nx, ny, max_iter, escape_radius=1e10, columns=columns, threads=2)


def test_series_frame_keeps_classes():
    # series.rs:695-753
    job = _job("-0.743643887037158", "0.131825904205312", "1e-10", 48, 27, 20_000, fdref.COL_NU | fdref.COL_DE)
    ref = fdref.Ref.for_job(job)
    plain = fdref.render(job, ref)
    rho, e = fdref.bla_dc_bound(job)
    assert e == 0
    s = fdref.Series(ref, rho, 1e-10 / 48.0, job.max_iter)
    assert s.info()["n"] > 0
    got = fdref.render_series(job, ref, s)
    assert got["kernel"].endswith(" series/0"), got["kernel"]
    assert np.array_equal(plain["cls"], got["cls"])
    # fd compare's displacement |dnu| / |grad nu|, |grad nu| = 2 / (de ln 2) per pixel,
    # where the plain de exceeds 1e-3 px
    a, b, de = plain["nu"], got["nu"], plain["de"].astype(np.float64)
    sel = de > 1e-3
    worst = np.max(np.abs(a[sel] - b[sel]) * de[sel] * math.log(2) / 2.0)
    assert worst < 1e-3, worst
    assert got["stats"]["iterations"] < 48 * 27 * 20_000
    assert got["stats"]["iterations"] < plain["stats"]["iterations"]
    # a masked pass reuses the exact start and matches the full render
    mask = (np.arange(48 * 27) % 2 == 0).astype(np.uint8)
    part = fdref.render_series(job, ref, s, mask=mask)
    on = mask.astype(bool)
    assert np.array_equal(part["cls"][on], got["cls"][on])
    assert np.array_equal(part["nu"][on], got["nu"][on])
    assert not part["n"][~on].any()
    # no admitted prefix: the plain render, bit for bit
    none = fdref.render_series(job, ref, s.with_n(0))
    assert np.array_equal(none["cls"], plain["cls"])
    assert np.array_equal(none["nu"], plain["nu"])


def test_unresolved_series_start_preserves_nucleus_interior():
    # series.rs:644-693: an odd grid holds the exact centre, whose zero perturbation cannot
    # pass the resolvability guard; the retry from zero keeps the nucleus contraction
    v = KATS["series_frames"][-1]
    job = _job(v["re"], v["im"], v["width"], 33, 19, 10_000, fdref.COL_NU | fdref.COL_DE)
    ref = fdref.Ref.for_job(job)
    assert ref.nucleus_period() is not None
    plain = fdref.render(job, ref)
    centre = (19 // 2) * 33 + 33 // 2
    assert plain["cls"][centre] & 3 == 1  # interior
    rho, e = fdref.bla_dc_bound(job)
    s = fdref.Series(ref, rho, float(v["width"]) / 33.0, job.max_iter)
    assert s.info()["n"] > 0
    got = fdref.render_series(job, ref, s)
    assert np.array_equal(plain["cls"], got["cls"])


def test_series_refusals():
    """Series::render_masked's refusals (grid.rs:350-366): another orbit, a view beyond the
    series radius."""
    job = _job("-0.743643887037158", "0.131825904205312", "1e-10", 48, 27, 20_000, fdref.COL_NU)
    ref = fdref.Ref.for_job(job)
    rho, _ = fdref.bla_dc_bound(job)
    small = fdref.Series(ref, rho / 2, 1e-10 / 48.0, job.max_iter)
    try:
        fdref.render_series(job, ref, small)
        raise AssertionError("a view beyond the series radius must be refused")
    except ValueError as err:
        assert "radius" in str(err)
    other = fdref.Ref.f64(-0.743643887037158, 0.131825904205312, 1_000, 1e10)
    s_other = fdref.Series(other, rho, 1e-10 / 48.0, 1_000)
    try:
        fdref.render_series(job, ref, s_other)
        raise AssertionError("a series over another orbit must be refused")
    except ValueError as err:
        assert "orbit" in str(err)
