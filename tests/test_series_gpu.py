"""The parameter-series start on the CUDA route (fdc_upload_series + FDC_SERIES) against
the oracle's render_series (crates/fd-kernel/src/grid.rs:213-226, 341-373): class, escape
count and z at escape bit for bit, and the work counters equal, on the reference's own
series views. The seahorse frame runs plain and through a sample mask, a 7.9e-26 series
frame with BLA blocks; the nucleus frame admits 9,999 of 10,000 iterations, so nearly
every sample's series start ends unresolved and retries from zero. Refusals follow
Series::render_masked."""
import json
import os

import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

pytestmark = pytest.mark.gpu

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kats.json")))
SEAHORSE = ("-0.743643887037158", "0.131825904205312", "1e-10")


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def _setup(view3, nx, ny, max_iter, bla=False):
    v = fd.View(*view3)
    p = fd.Params(nx, ny, max_iter=max_iter, columns=("nu", "de"))
    plane, tier = fd.route._setup(v, p)
    r, bits = fd.reference(v, p)
    r.bits = bits
    rho, e = fd.bla_dc_bound(v, p)
    assert e == 0 and tier in (0, 1)
    series = fd.Series.build(r, rho, float(view3[2]) / nx, max_iter)
    table = fd.Bla.build_scaled(r, fd.route.EPS, rho, 0) if bla else None
    # the oracle's own series and table over the same orbit
    ref = fdref.Ref.arrays(r.re, r.im, bits)
    o_series = fdref.Series(ref, rho, float(view3[2]) / nx, max_iter)
    assert o_series.info()["n"] == series.n > 0
    o_bla = fdref.Bla(ref, fd.route.EPS, rho, 0) if bla else None
    job = fdref.make_job(*view3, nx, ny, max_iter, escape_radius=p.escape_radius, columns=fdref.COL_NU | fdref.COL_DE,
                         tier=tier)
    return v, p, (r, bits), series, table, ref, o_series, o_bla, job


def _check(got, want, stats, bstats, mask=None):
    sel = np.ones(len(want["cls"]), bool) if mask is None else mask.astype(bool)
    assert np.array_equal(got.cls[sel], want["cls"][sel])
    assert np.array_equal(got.n[sel], want["n"][sel].astype(np.uint32))
    esc = sel & (want["cls"] == 0)
    assert np.array_equal(got.z[esc], want["z"][esc])
    assert stats.iterations == want["stats"]["iterations"]
    if bstats is not None:
        assert (bstats.blocks, bstats.skipped) == (want["stats"]["blocks"], want["stats"]["skipped"])
        assert bstats.fallback_samples == want["stats"]["fallback_samples"]
        assert bstats.closed_form_samples == want["stats"]["closed_form_samples"]


@pytest.mark.parametrize("use_bla", [False, True])
def test_series_frame_equals_oracle(dev, use_bla):
    """The seahorse frame at 1e-10 (F64 tier; no BLA level is valid there), and with BLA
    the series frame at 7.9e-26 (Fixed tier: 9 levels, blocks applied, a few samples
    unresolved from the series start)."""
    if use_bla:
        f = KATS["series_frames"][18]
        view3, nx, ny, max_iter = (f["re"], f["im"], f["width"]), 33, 19, 10_000
    else:
        view3, nx, ny, max_iter = SEAHORSE, 48, 27, 20_000
    v, p, orbit, series, table, ref, o_series, o_bla, job = _setup(view3, nx, ny, max_iter, use_bla)
    h, s, st, bst = fd.render_series(v, p, orbit, series, table, dev=dev, raw=True)
    assert " series/0" in h.kernel
    want = fdref.render_series(job, ref, o_series, bla=o_bla, raw=True)
    _check(s, want, st, bst)
    if use_bla:
        assert table.levels > 0 and bst.blocks > 0
    # the series skipped work: fewer counted iterations than the plain render
    plain = fdref.render(job, ref, o_bla, raw=True)
    assert np.array_equal(s.cls, plain["cls"])
    assert st.iterations < plain["stats"]["iterations"]


def test_series_masked_render_equals_oracle(dev):
    v, p, orbit, series, table, ref, o_series, o_bla, job = _setup(SEAHORSE, 48, 27, 20_000)
    r, bits = orbit
    plane, tier = fd.route._setup(v, p)
    mask = (np.arange(48 * 27) % 3 != 1).astype(np.uint8)
    hnd = dev.upload(r, None)
    try:
        dev.upload_series(hnd, series)
        j = fd.route.make_job(plane, tier, p, hnd, r.nucleus_period(), _lib.DERIVATIVE | _lib.SERIES)
        j.mask = mask.ctypes.data
        got, cnt, _ = dev.render_job(j, raw=True)
    finally:
        dev.free(hnd)
    want = fdref.render_series(job, ref, o_series, mask=mask, raw=True)
    on = mask.astype(bool)
    assert np.array_equal(got["status"], mask)
    assert np.array_equal(got["cls"][on], want["cls"][on])
    assert np.array_equal(got["n"][on], want["n"][on].astype(np.uint32))
    esc = on & (want["cls"] == 0)
    assert np.array_equal(got["z"][esc], want["z"][esc])
    assert cnt.iterations == want["stats"]["iterations"]


def test_unresolved_series_start_retries_from_zero(dev):
    f = KATS["series_frames"][-1]
    v, p, orbit, series, table, ref, o_series, o_bla, job = _setup((f["re"], f["im"], f["width"]), 33, 19, 10_000)
    assert series.n == 9_999
    h, s, st, _ = fd.render_series(v, p, orbit, series, dev=dev, raw=True)
    want = fdref.render_series(job, ref, o_series, raw=True)
    _check(s, want, st, None)
    plain = fdref.render(job, ref, raw=True)
    assert np.array_equal(s.cls, plain["cls"])  # the nucleus interior survives (series.rs:644-693)
    assert s.cls[(19 // 2) * 33 + 33 // 2] & 3 == 1


def test_series_refusals(dev):
    v, p, orbit, series, table, ref, o_series, o_bla, job = _setup(SEAHORSE, 48, 27, 20_000)
    small = fd.Series(**{**series.__dict__, "rho": series.rho / 2})
    with pytest.raises(ValueError, match="radius"):
        fd.render_series(v, p, orbit, small, dev=dev)
    other = fd.Series(**{**series.__dict__, "points": series.points + 1})
    with pytest.raises(ValueError, match="another orbit"):
        fd.render_series(v, p, orbit, other, dev=dev)
    r, bits = orbit
    plane, tier = fd.route._setup(v, p)
    hnd = dev.upload(r, None)
    try:
        with pytest.raises(fd.route.RouteError, match="another orbit"):
            dev.upload_series(hnd, other)
        j = fd.route.make_job(plane, tier, p, hnd, r.nucleus_period(), _lib.DERIVATIVE | _lib.SERIES)
        with pytest.raises(fd.route.RouteError, match="without an uploaded series"):
            dev.render_job(j)
        dev.upload_series(hnd, series)
        j.flags |= _lib.F32
        with pytest.raises(fd.route.RouteError, match="plain form"):
            dev.render_job(j)
        j.flags = _lib.SERIES | _lib.DEVICE_OUT
        with pytest.raises(fd.route.RouteError, match="FDC_SERIES"):
            dev.batch([j])
    finally:
        dev.free(hnd)
