"""Bounded renders on the CUDA route (fdc_upload_error_radius + fdc_render_bounded: the
Bound column, Bounded evidence; sample.rs's B variant, store.rs:88-106) against the
oracle's bounded render over the same orbit, on the F64 and Fixed tiers: class kind,
count, z at escape and the raw error radii ez / ed bit for bit, the Bounded evidence bit
equal, and the Bound and de columns within CUDA libm's ulps of the host's (log, log1p,
exp, exp2, hypot). The scaled tier has no radii and renders as fdc_render. Refusals
follow grid.rs:379-384."""
import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

pytestmark = pytest.mark.gpu

VIEWS = [(("-0.7453", "0.1127", "0.0065"), 4_000),                       # F64 tier
         (("-0.743643887037158", "0.131825904205312", "1e-14"), 20_000)]  # Fixed tier


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def _close(a, b, rel):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)))


@pytest.mark.parametrize("view,max_iter", VIEWS)
def test_bounded_render_equals_oracle(dev, view, max_iter):
    v = fd.View(*view)
    p = fd.Params(40, 24, max_iter=max_iter, columns=("nu", "de", "bound"))
    plane, tier = fd.route._setup(v, p)
    assert tier in (0, 1)
    r, bits = fd.reference(v, p)
    h, s, st, _ = fd.render_with(v, p, (r, bits), dev=dev, raw=True)
    assert h.columns[-1] == "bound"
    ref = fdref.Ref.arrays(r.re, r.im, bits)
    job = fdref.make_job(*view, 40, 24, max_iter, escape_radius=p.escape_radius,
                         columns=fdref.COL_NU | fdref.COL_DE | fdref.COL_BOUND, tier=tier)
    want = fdref.render_columns(job, ref)
    assert np.array_equal(s.cls & 3, want["cls"] & 3)
    assert np.array_equal(s.n, want["n"].astype(np.uint32))
    esc = (want["cls"] & 3) == 0
    assert esc.sum() > 100
    assert np.array_equal(s.z[esc], want["z"][esc])
    assert np.array_equal(s.ez[esc], want["ez"][esc])
    assert np.array_equal(s.ed[esc], want["ed"][esc])
    assert np.array_equal(s.cls, want["cls"])  # the Bounded evidence bit
    bounded = want["cls"] == 4
    assert bounded.sum() > 0.5 * esc.sum()
    assert _close(s.bound[bounded], want["bound"][bounded], 1e-6)
    assert not s.bound[~bounded].any()
    assert _close(s.de[esc], want["de"][esc], 1e-6)
    assert _close(s.nu[esc], want["nu"][esc], 1e-12)
    assert st.iterations == want["stats"]["iterations"]


def test_bounded_render_on_the_scaled_tier_is_plain(dev):
    v = fd.View("0", "1", "1e-300")
    p = fd.Params(24, 16, max_iter=5_000, columns=("nu", "de", "bound"))
    plane, tier = fd.route._setup(v, p)
    assert tier == 2
    orbit = fd.reference(v, p)
    _, s, _, _ = fd.render_with(v, p, orbit, dev=dev)
    _, plain, _, _ = fd.render_with(v, fd.Params(24, 16, max_iter=5_000, columns=("nu", "de")), orbit, dev=dev)
    assert np.array_equal(s.cls, plain.cls) and not (s.cls & 4).any()
    assert np.array_equal(s.de, plain.de) and not s.bound.any()


def test_bounded_refusals(dev):
    v = fd.View("-0.7453", "0.1127", "0.0065")
    p = fd.Params(16, 8, max_iter=2_000, columns=("nu", "bound"))
    plane, tier = fd.route._setup(v, p)
    r, bits = fd.reference(v, p)
    r.bits = bits
    dc, e = fd.bla_dc_bound(v, p)
    table = fd.Bla.build_scaled(r, 2.0 ** -50, dc, e)
    with pytest.raises(ValueError, match="not certified"):
        fd.render_with(v, p, (r, bits), table, dev=dev)
    hnd = dev.upload(r, table)
    try:
        j = fd.route.make_job(plane, tier, p, hnd, r.nucleus_period(), _lib.DERIVATIVE)
        with pytest.raises(fd.route.RouteError, match="without uploaded error radii"):
            dev.render_job(j, bounded=True)
        with pytest.raises(fd.route.RouteError, match="cover the orbit"):
            dev.upload_error_radius(hnd, np.zeros(len(r) - 1))
        dev.upload_error_radius(hnd, r.error_radius(None, plane.c_re, plane.c_im))
        j.flags |= _lib.BLA
        with pytest.raises(fd.route.RouteError, match="not certified"):
            dev.render_job(j, bounded=True)
        j.flags = _lib.DERIVATIVE | _lib.F32
        with pytest.raises(fd.route.RouteError, match="plain form"):
            dev.render_job(j, bounded=True)
    finally:
        dev.free(hnd)
