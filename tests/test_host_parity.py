"""CPU tests of the route's C++ host side against the oracle, and of the C ABI's surface.

The host set-up (decimal centres, fixed-point orbit, plane, BLA builder, nucleus gate)
must equal the reference's bit for bit; the oracle stands in for the reference here.
No test in this file touches a GPU.
"""
import ctypes as C
import json
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KATS = json.load(open(os.path.join(ROOT, "tests", "golden", "kats.json")))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"\b(fd[ch]_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(line.split()[-1] for line in out.stdout.splitlines())
    want = declared("fdcuda.h") + declared("fdhost.h")
    assert want and set(want) <= exported, set(want) - exported
    assert set(want) == set(_lib.FDC_SYMBOLS + _lib.FDH_SYMBOLS)


def test_library_loads_and_reports_no_device_without_a_gpu():
    L = _lib.lib()
    assert L.fdc_abi_version() == 1
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert L.fdc_open(0, C.byref(h)) == _lib.NO_DEVICE and not h


VIEWS = [("-0.7453", "0.1127", "0.0065", 0.3), ("0", "1", "1e-20", 0.0), ("0", "1", "1e-300", 0.5),
         ("0", "1", "1e-1000", 0.0), ("0.25", "0", "1e-3", 0.0), ("-2", "0", "1e-200", 0.0),
         ("3e-298", "1." + "0" * 300 + "7", "1e-300", 0.0), ("-0.7436438870371587", "0.1318259042053120", "1e-12", 0.0)]


@pytest.mark.parametrize("re_,im_,width,rot", VIEWS)
def test_plane_equals_reference(re_, im_, width, rot):
    a = fdref.plane(fdref.make_job(re_, im_, width, 480, 270, 100, rotation=rot))
    b = fd.Plane.new(fd.View(re_, im_, width, rot), 480, 270)
    assert (a["h_m"], a["h_e"], a["tier"], a["bits"], a["c_re"], a["c_im"]) == \
        (b.h_m, b.h_e, b.tier, b.bits, b.c_re, b.c_im)


@pytest.mark.parametrize("bad", ["", ".", "1e", "--1", "1.2.3", "0x10", "abc"])
def test_plane_refuses_malformed_decimals(bad):
    with pytest.raises(ValueError):
        fd.Plane.new(fd.View(bad, "0", "1"), 8, 8)
    with pytest.raises(ValueError):
        fd.Plane.new(fd.View("0", "0", bad), 8, 8)


@pytest.mark.parametrize("bits", [128, 177, 218, 471, 1130, 3456])
def test_fixed_orbit_bit_exact(bits):
    re_, im_ = KATS["v0"]["re"], KATS["v0"]["im"]
    a = fdref.Ref.fixed(re_, im_, bits, 3000)
    b = fd.Reference.from_fixed(re_, im_, bits, 3000)
    ar, ai = a.arrays_()
    assert len(b) == len(a)
    assert np.array_equal(ar.view(np.uint64), b.re.view(np.uint64))
    assert np.array_equal(ai.view(np.uint64), b.im.view(np.uint64))


def test_fixed_orbit_escaping_and_rung():
    rung = KATS["rung_7676"]
    for (re_, im_, bits, n) in [("1", "1", 128, 100), ("-0.75", "0.1", 256, 5000),
                                (rung["re"], rung["im"], 3456, 4000)]:
        a = fdref.Ref.fixed(re_, im_, bits, n)
        b = fd.Reference.from_fixed(re_, im_, bits, n)
        ar, ai = a.arrays_()
        assert np.array_equal(ar, b.re) and np.array_equal(ai, b.im)
        assert a.nucleus_period() == b.nucleus_period()


@pytest.mark.parametrize("threads", [1, 3])
def test_fixed_orbit_reaches_the_mpmath_nucleus_return(threads):
    """The period-764 nucleus orbit of crates/fd-fixed/tests/fixtures/v0_orbit.txt at
    1,400 bits: the host orbit equals the oracle's bit for bit, lands within one ulp of
    mpmath's 400-digit z_764 (~6e-54) and the nucleus gate finds the period."""
    f = KATS["v0_orbit"]
    period = int(f["period"])
    a = fdref.Ref.fixed(f["c"][0], f["c"][1], 1400, 2 * period + 10)
    b = fd.Reference.from_fixed(f["c"][0], f["c"][1], 1400, 2 * period + 10, threads=threads)
    ar, ai = a.arrays_()
    assert np.array_equal(ar.view(np.uint64), b.re.view(np.uint64))
    assert np.array_equal(ai.view(np.uint64), b.im.view(np.uint64))
    want = np.array([float(f["z"][0]), float(f["z"][1])])
    got = np.array([b.re[period], b.im[period]])
    assert np.all(np.abs(got - want) <= np.spacing(np.abs(want)))
    assert b.nucleus_period() == a.nucleus_period() == period


@pytest.mark.parametrize("threads", [1, 3])
def test_fixed_orbit_shared_squarings_bit_exact(threads):
    """A wide orbit (3,456 bits, 55 limbs) whose step squarings run on three threads equals
    the serial one and the oracle's, bit for bit; so does one below the threshold."""
    rung = KATS["rung_7676"]
    for bits, n in ((3456, 4000), (1130, 3000)):
        a = fdref.Ref.fixed(rung["re"], rung["im"], bits, n)
        b = fd.Reference.from_fixed(rung["re"], rung["im"], bits, n, threads=threads)
        ar, ai = a.arrays_()
        assert len(b) == len(a) == n + 1
        assert np.array_equal(ar.view(np.uint64), b.re.view(np.uint64))
        assert np.array_equal(ai.view(np.uint64), b.im.view(np.uint64))


def test_f64_orbit_and_nucleus_gate():
    for c in [(-0.7487, 0.0789), (0.2501, 0.0), (-1.7548776662466927, 0.0), (0.0, 1.0)]:
        a = fdref.Ref.f64(c[0], c[1], 100_000, 1e10)
        b = fd.Reference.new(c[0], c[1], 100_000, 1e10)
        ar, ai = a.arrays_()
        assert np.array_equal(ar, b.re) and np.array_equal(ai, b.im)
        assert a.nucleus_period() == b.nucleus_period()


@pytest.mark.parametrize("eps,dc,e", [(2.0 ** -50, 1e-25, 0), (2.0 ** -41, 2e-17, 0), (2.0 ** -50, 1.3, -1000),
                                      (2.0 ** -26, 1e-30, 0)])
def test_bla_table_bit_exact(eps, dc, e):
    a = fdref.Ref.f64(-0.743643887037158, 0.131825904205312, 20_000, 1e10)
    re_, im_ = a.arrays_()
    ta = fdref.Bla(a, eps, dc, e)
    tb = fd.Bla.build_scaled(fd.Reference(re_, im_, 53), eps, dc, e, threads=4)
    ba, oa = ta.export()
    assert np.array_equal(oa, tb.level_offsets)
    assert np.array_equal(ba.view(np.uint64), tb.blocks.view(np.uint64))


def test_bla_one_pass_build_equals_two_call_build():
    """fdh_bla_build_into (one pass into bounded buffers, as Bla.build_scaled uses it)
    gives the table of the two-call fdh_bla_build, and refuses buffers that are too small."""
    import ctypes as C
    from fractodactyl_b200._lib import lib
    a = fdref.Ref.f64(-0.743643887037158, 0.131825904205312, 20_000, 1e10)
    re_, im_ = a.arrays_()
    re_, im_ = np.ascontiguousarray(re_), np.ascontiguousarray(im_)
    tb = fd.Bla.build_scaled(fd.Reference(re_, im_, 53), 2.0 ** -50, 1e-25, 0)
    L = lib()
    lv, bl = C.c_uint32(), C.c_uint64()
    args = (re_.ctypes.data, im_.ctypes.data, len(re_), 2.0 ** -50, 1e-25, 0, 2)
    assert L.fdh_bla_build(*args, None, None, C.byref(lv), C.byref(bl)) == 0
    b = np.zeros((bl.value, 7))
    o = np.zeros(lv.value + 1, np.uint64)
    assert L.fdh_bla_build(*args, b.ctypes.data, o.ctypes.data, C.byref(lv), C.byref(bl)) == 0
    assert tb.levels == lv.value > 5 and len(tb.blocks) == bl.value
    assert np.array_equal(b.view(np.uint64), tb.blocks.view(np.uint64))
    assert np.array_equal(o, tb.level_offsets)
    small = np.zeros((bl.value - 1, 7))
    offs = np.zeros(65, np.uint64)
    assert L.fdh_bla_build_into(*args, small.ctypes.data, bl.value - 1, offs.ctypes.data, 64, C.byref(lv),
                                C.byref(bl)) == -1
    assert not small.any() and not offs.any()
    assert L.fdh_bla_build_into(*args, b.ctypes.data, len(b), offs.ctypes.data, tb.levels - 1, C.byref(lv),
                                C.byref(bl)) == -1


def test_bla_refuses_bad_eps():
    r = fd.Reference.new(-0.7453, 0.1127, 2000, 1e10)
    with pytest.raises(ValueError):
        fd.Bla.build_scaled(r, 2.0 * 2.0 ** -24, 1e-20)
    with pytest.raises(ValueError):
        fd.Bla.build_scaled(r, 2.0 ** -50, float("inf"))


def test_dc_bound_equals_reference():
    for (re_, im_, width) in [("-0.7453", "0.1127", "0.0065"), ("0", "1", "1e-300")]:
        job = fdref.make_job(re_, im_, width, 32, 32, 100)
        assert fdref.bla_dc_bound(job) == fd.bla_dc_bound(fd.View(re_, im_, width), fd.Params(32, 32))


def test_route_flag_and_declines():
    assert fd.enabled(None) is False and fd.enabled("cuda") and fd.enabled("cuda-bla") and fd.enabled("bla")
    with pytest.raises(ValueError):
        fd.enabled("fast")
    # the Stripe column: the reference's refusal (grid.rs:783-788), and the combinations the
    # route leaves to the CPU (with the Bound column or a series start)
    with pytest.raises(ValueError, match="stripe window"):
        fd.render(fd.View("0", "1", "1e-3"), fd.Params(8, 8, columns=("nu", "stripe"), stripe_window=65))
    with pytest.raises(ValueError, match="stripe window"):
        fd.render(fd.View("0", "1", "1e-3"), fd.Params(8, 8, columns=("nu", "stripe"), stripe_freq=float("inf")))
    with pytest.raises(fd.Declined):
        fd.render(fd.View("0", "1", "1e-3"), fd.Params(8, 8, columns=("nu", "stripe", "bound")))
    # the Bound column certifies every step: no BLA (grid.rs:379-384), no series start
    r = fd.Reference.new(-0.7453, 0.1127, 2_000, 1e10)
    table = fd.Bla.build_scaled(r, 2.0 ** -50, 1e-5)
    with pytest.raises(ValueError, match="not certified"):
        fd.render_with(fd.View("-0.7453", "0.1127", "1e-3"), fd.Params(8, 8, columns=("nu", "bound")), None, table)
    with pytest.raises(ValueError):
        fd.route._setup(fd.View("0", "1", "1e-300"), fd.Params(8, 8, tier="f64"))


@pytest.mark.parametrize("radius,shown", [(float("nan"), "NaN"), (3.5, "3.5"), (2.0, "2")])
def test_bla_escape_radius_refusals(radius, shown):
    """A BLA table needs an escape radius of at least 4, NaN refused (grid.rs:393-398),
    with the reference's message: for a table without levels the route checks this on the
    host, and render_bla before it builds the table. Nothing reaches a device."""
    msg = f"escape radius {shown} is below 4: BLA blocks may only skip iterates with |z| <= 2 (1 + 2 eps), " \
          "which needs escape radius >= 4"
    view = fd.View("-0.7453", "0.1127", "1e-3")
    p = fd.Params(8, 8, max_iter=200, escape_radius=radius)
    r = fd.Reference.new(-0.7453, 0.1127, 200, 1e10)
    empty = fd.Bla(np.zeros((0, 7)), np.zeros(1, np.uint64), 2.0 ** -50, 1e-5, 0, len(r))
    with pytest.raises(ValueError) as e:
        fd.render_with(view, p, (r, 53), empty)
    assert str(e.value) == msg
    with pytest.raises(ValueError) as e:
        fd.render_bla(view, p, (r, 53))
    assert str(e.value) == msg


@pytest.mark.parametrize("case", KATS["fnv_views"], ids=lambda c: c["width"])
def test_fds_writer_and_host_encoder_bytes(case):
    """fds.encode over the oracle's raw outcomes encoded by fdh_encode equals the oracle's
    own .fds bytes (header.rs:62-81, write.rs:8-53, store.rs:66-112)."""
    from fractodactyl_b200 import fds
    job = fdref.make_job(case["re"], case["im"], case["width"], 8, 4, 5000, rotation=0.3, threads=1)
    want = fdref.render_fds(job)
    o = fdref.render(job, raw=True)
    view = fd.View(case["re"], case["im"], case["width"], 0.3)
    plane, tier = fd.route._setup(view, fd.Params(8, 4, max_iter=5000))
    s = fd.Samples(cls=o["cls"], n=o["n"].astype(np.uint32), z=o["z"], dz=o["dz"], dexp=o["dexp"])
    fd.route.encode_host(plane, 1, s)
    h = fd.Header(("class", "nu", "de", "normal"), 8, 4, 1, 5000, 1e10, view, o["kernel"])
    assert fds.encode(h, s) == want


@pytest.mark.parametrize("case", ["seahorse", "frame_first", "frame_last", "unbounded", "tight"])
def test_series_build_bit_exact(case):
    """fdh_series_build (Series::build, series.rs:86-245) equals the oracle's series bit for
    bit: admitted prefix, coefficients, bounds and the work counters."""
    frames = KATS["series_frames"]
    stalled = 32
    if case in ("seahorse", "unbounded", "tight"):
        a = fdref.Ref.f64(-0.743643887037158, 0.131825904205312, 20_000, 1e10)
        rho, pixel, max_iter = {"seahorse": (1e-11, 1e-13, 20_000), "unbounded": (1e-11, 1e-13, 20_000),
                                "tight": (1e-6, 1e-9, 5_000)}[case]
        stalled = 0 if case == "unbounded" else 32
    else:
        v = frames[0] if case == "frame_first" else frames[-1]
        job = fdref.make_job(v["re"], v["im"], v["width"], 33, 19, 10_000)
        a = fdref.Ref.for_job(job)
        rho, _ = fdref.bla_dc_bound(job)
        pixel, max_iter = float(v["width"]) / 33.0, 10_000
    want = fdref.Series(a, rho, pixel, max_iter, stalled_steps=stalled)
    re_, im_ = a.arrays_()
    got = fd.Series.build(fd.Reference(np.ascontiguousarray(re_), np.ascontiguousarray(im_), a.bits), rho, pixel,
                          max_iter, stalled_steps=stalled)
    w = want.info()
    assert (got.n, got.points, got.built_steps, got.coefficient_pairs, got.stop) == \
        (w["n"], w["points"], w["built_steps"], w["coefficient_pairs"], w["stop"])
    assert len(got.b) == w["order"]
    assert np.array_equal(got.b.view(np.uint64), want.coefficients().view(np.uint64))
    for k in ("rho", "state_bound", "derivative_bound", "shift_px"):
        assert np.float64(getattr(got, k)).view(np.uint64) == np.float64(w[k]).view(np.uint64), k
    if case != "tight":
        assert got.n > 0


@pytest.mark.parametrize("case", ["f64", "fixed", "deep"])
def test_error_radius_bit_exact(case):
    """fdh_error_radius (Reference::error_radius, reference.rs:122-148) equals the
    oracle's bit for bit, for f64 and fixed-point orbits (bits beyond the subnormal range
    clamp the unit to the smallest normal)."""
    if case == "f64":
        a = fdref.Ref.f64(-0.7453, 0.1127, 5_000, 1e10)
        bits, c = None, (-0.7453, 0.1127)
    else:
        rung = KATS["rung_7676"]
        bits = 256 if case == "fixed" else 3456
        a = fdref.Ref.fixed(rung["re"], rung["im"], bits, 4_000)
        c = (float(rung["re"]), float(rung["im"]))
    re_, im_ = a.arrays_()
    want = fdref.error_radius(a, bits, *c)
    got = fd.Reference(np.ascontiguousarray(re_), np.ascontiguousarray(im_), a.bits).error_radius(bits, *c)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    assert np.all(got >= 0)


def test_fds_writer_bound_column():
    """A bounded render's .fds file (the Bound column, bit 16, f32, after normal:
    crates/fd-samples/src/column.rs:18-19, 42) written by fds.encode from the oracle's
    bounded columns equals the oracle's own .fds bytes, on the F64 and Fixed tiers."""
    from fractodactyl_b200 import fds
    for view3, max_iter in ((("-0.7453", "0.1127", "0.0065"), 4000),
                            (("-0.743643887037158", "0.131825904205312", "1e-14"), 20000)):
        cols = fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL | fdref.COL_BOUND
        job = fdref.make_job(*view3, 9, 5, max_iter, rotation=0.2, columns=cols, threads=1)
        ref = fdref.Ref.for_job(job)
        want = fdref.render_fds(job, ref)
        o = fdref.render_columns(job, ref)
        assert (o["cls"] == 4).any() and (o["bound"] > 0).any()
        view = fd.View(*view3, 0.2)
        s = fd.Samples(cls=o["cls"], nu=o["nu"], de=o["de"], normal=o["normal"], bound=o["bound"])
        h = fd.Header(("class", "nu", "de", "normal", "bound"), 9, 5, 1, max_iter, 1e10, view, o["kernel"])
        b = fds.encode(h, s)
        assert struct.unpack_from("<I", b, 12)[0] == 1 | 2 | 4 | 8 | 16
        assert b == want
