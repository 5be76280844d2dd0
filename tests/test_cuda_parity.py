"""Parity of the CUDA route (through the C ABI) with the CPU oracle.

Bar for the plain (FP64) form: class, escape count, z and dz/dc (mantissa and exponent)
bit-exact; nu within 1e-12 relative, de within 1e-6 relative and the normal within one
u16 step (these three go through CUDA's log2/hypot/atan2 instead of glibc's).
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
import truthpack
from fractodactyl_b200 import _lib

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KATS = json.load(open(os.path.join(ROOT, "tests", "golden", "kats.json")))
NU_REL, DE_REL = 1e-12, 1e-6


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def oracle_ref(job_o):
    r = fdref.Ref.for_job(job_o)
    re_, im_ = r.arrays_()
    return r, fd.Reference(re_, im_, r.bits)


def assert_same(o, s, columns=("nu", "de", "normal")):
    """CUDA samples s against oracle render o (raw=True)."""
    assert np.array_equal(o["cls"], s.cls), np.nonzero(o["cls"] != s.cls)[0][:10]
    n_o = o["n"].astype(np.uint64)
    assert np.array_equal(n_o, s.n.astype(np.uint64)), np.nonzero(n_o != s.n)[0][:10]
    esc = o["cls"] == 0
    assert np.array_equal(o["z"][esc].view(np.uint64), s.z[esc].view(np.uint64))
    assert np.array_equal(o["dz"][esc].view(np.uint64), s.dz[esc].view(np.uint64))
    assert np.array_equal(o["dexp"][esc], s.dexp[esc])
    if "nu" in columns:
        rel = np.abs(o["nu"][esc] - s.nu[esc]) / np.maximum(np.abs(o["nu"][esc]), 1e-300)
        assert rel.size == 0 or rel.max() <= NU_REL
    if "de" in columns:
        d_o, d_s = o["de"][esc].astype(np.float64), s.de[esc].astype(np.float64)
        fin = np.isfinite(d_o) & (d_o != 0)
        assert np.array_equal(np.isfinite(d_o), np.isfinite(d_s))
        assert not fin.any() or (np.abs(d_o[fin] - d_s[fin]) / np.abs(d_o[fin])).max() <= DE_REL
    if "normal" in columns:
        dn = (o["normal"][esc].astype(np.int64) - s.normal[esc].astype(np.int64)) % 65536
        assert np.all((dn <= 1) | (dn >= 65535))


def frame(dev, re_, im_, width, nx, ny, max_iter, rot=0.0, tier=None, bla_eps=None, escape_radius=1e10,
          columns=("nu", "de", "normal")):
    cols = fdref.COL_NU * ("nu" in columns) | fdref.COL_DE * ("de" in columns) | fdref.COL_NORMAL * (
        "normal" in columns)
    jo = fdref.make_job(re_, im_, width, nx, ny, max_iter, rotation=rot, tier=tier, escape_radius=escape_radius,
                        columns=cols)
    r_o, r_c = oracle_ref(jo)
    bla_o = bla_c = None
    if bla_eps is not None:
        dc, e = fdref.bla_dc_bound(jo)
        bla_o = fdref.Bla(r_o, bla_eps, dc, e)
        blocks, offs = bla_o.export()
        bla_c = fd.Bla(blocks, offs, bla_eps, dc, e, len(r_c))
    o = fdref.render(jo, r_o, bla_o, raw=True)
    view = fd.View(re_, im_, width, rot)
    p = fd.Params(nx, ny, max_iter=max_iter, escape_radius=escape_radius, columns=columns, tier=tier)
    h, s, st, bs = fd.render_with(view, p, (r_c, r_c.bits), bla_c, dev=dev, raw=True)
    return o, h, s, st, bs


@pytest.mark.parametrize("case", KATS["fnv_views"], ids=lambda c: c["width"])
def test_fnv_views(dev, case):
    o, h, s, st, _ = frame(dev, case["re"], case["im"], case["width"], 8, 4, 5000, rot=0.3)
    assert_same(o, s)
    assert st.iterations == o["stats"]["iterations"]
    assert h.kernel.startswith(o["kernel"]) and h.kernel.endswith("gpu-perturb-cuda/1")


@pytest.mark.parametrize("name", truthpack.CASES)
def test_truth_pack_views(dev, name):
    c = truthpack.load(name)
    edges = truthpack.load_edges()
    for bla_eps in (None, 2.0 ** -41):
        o, h, s, st, bs = frame(dev, c["re"], c["im"], c["width"], c["nx"], c["ny"], c["max_iter"],
                                rot=c["rotation"], bla_eps=bla_eps)
        assert_same(o, s)
        assert st.iterations == o["stats"]["iterations"]
        if bs is not None:
            assert (bs.blocks, bs.skipped, bs.fallback_samples, bs.closed_form_samples) == (
                o["stats"]["blocks"], o["stats"]["skipped"], o["stats"]["fallback_samples"],
                o["stats"]["closed_form_samples"])
            if bs.shift_px is not None:
                assert math.isclose(bs.shift_px, o["stats"]["shift_px"], rel_tol=1e-9)
        sc = truthpack.compare(c, s.cls, s.nu, s.de, s.normal, edges)
        expect = len([e for e in edges if e["case"] == name])
        assert sc["scalar_failures"] == 0 and sc["class_mismatches"] == sc["known_edges"] == expect


BIG = [
    # (re, im, width, nx, ny, max_iter, rot, tier): every tier, interior-heavy and deep views
    ("-0.7436438870371587", "0.1318259042053120", "1e-12", 120, 68, 20_000, 0.0, None),
    ("-0.7453", "0.1127", "0.0065", 96, 54, 20_000, 0.0, "scaled"),
    ("0.25", "0", "1e-8", 96, 54, 200_000, 0.0, None),
    ("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28", 64, 36, 50_000, 0.0,
     None),
    ("0", "1", "1e-300", 96, 54, 20_000, 0.0, None),
    ("-2", "0", "1e-200", 96, 54, 20_000, 0.0, None),
]


@pytest.mark.parametrize("view", BIG, ids=lambda v: v[2] + (v[7] or ""))
@pytest.mark.parametrize("bla", [False, True])
def test_frames_bit_exact(dev, view, bla):
    re_, im_, width, nx, ny, it, rot, tier = view
    o, h, s, st, bs = frame(dev, re_, im_, width, nx, ny, it, rot=rot, tier=tier,
                            bla_eps=2.0 ** -50 if bla else None)
    assert_same(o, s)
    assert st.iterations == o["stats"]["iterations"]
    assert np.all(s.status == 1)


def test_c1_view_without_derivative(dev):
    """Config 1's view (480x270 crop of it): n, nu, class only, escape radius 2^8."""
    o, h, s, st, _ = frame(dev, "-0.7436438870371587", "0.1318259042053120", "1e-12", 160, 90, 20_000,
                           escape_radius=256.0, columns=("nu",))
    assert_same(o, s, columns=("nu",))


def single(dev, ref_c, ar, ai, max_iter, r2, offset_exp=None, bla=None, nucleus=-2, deriv=True):
    """One sample with an explicit offset through a 1x1 job (tier Fixed, or Scaled when
    offset_exp is given: dc = (ar, ai) 2^offset_exp)."""
    h = dev.upload(ref_c, bla)
    try:
        j = _lib.Job()
        j.orbit = h
        j.tier = 2 if offset_exp is not None else 1
        j.nx = j.ny = j.ss = 1
        j.flags = (_lib.DERIVATIVE if deriv else 0) | (_lib.BLA if bla is not None else 0)
        j.h_m, j.h_e = 1.0, offset_exp or 0
        j.cos_rot, j.sin_rot = 1.0, 0.0
        j.max_iter = max_iter
        j.escape_radius = math.sqrt(r2)
        if nucleus == -2:
            nucleus = ref_c.nucleus_period()
        j.nucleus_period = -1 if nucleus is None else nucleus
        off = np.array([ar, ai])
        j.offsets = off.ctypes.data
        arrays, cnt, _ = dev.render_job(j, raw=True)
    finally:
        dev.free(h)
    kind = {0: "escaped", 1: "interior", 2: "unresolved"}[int(arrays["cls"][0]) & 3]
    return dict(kind=kind, n=int(arrays["n"][0]), zr=arrays["z"][0, 0], zi=arrays["z"][0, 1],
                dr=arrays["dz"][0, 0], di=arrays["dz"][0, 1], dexp=int(arrays["dexp"][0]), blocks=cnt.blocks,
                skipped=cnt.skipped)


def as_c(r_o):
    re_, im_ = r_o.arrays_()
    return fd.Reference(re_, im_, r_o.bits)


def test_kat_near_return_that_expands(dev):
    r = fdref.Ref.fixed(KATS["v0"]["re"], KATS["v0"]["im"], 218, 2000)
    h = 8.29151e-25 / 960.0
    o = single(dev, as_c(r), h * (287 + 0.5 - 480.0), -h * (212 + 0.5 - 270.0), 2000, 1e20)
    assert o["kind"] == "escaped" and o["n"] == 788


def test_kat_bla_frame_749(dev):
    r = fdref.Ref.fixed(KATS["v0"]["re"], KATS["v0"]["im"], 300, 20_000)
    t = fdref.Bla(r, 2.0 ** -50, 2e-49 * 1.15)
    b, offs = t.export()
    h = 2e-49 / 960.0
    rc = as_c(r)
    o = single(dev, rc, h * (324 + 0.5 - 480.0), -h * (10 + 0.5 - 270.0), 20_000, 1e20,
               bla=fd.Bla(b, offs, 2.0 ** -50, 2e-49 * 1.15, 0, len(rc)))
    assert o["kind"] == "escaped" and o["n"] == 7412 and o["skipped"] > 4096


@pytest.mark.parametrize("cr,ci,n", [(0.0, 1.0, 887), (0.250001, 0.0, 3145), (-0.75, 0.01, 320)])
def test_kat_deep_exteriors(dev, cr, ci, n):
    r = fdref.Ref.f64(cr, ci, 20_000, 65536.0)
    o = single(dev, as_c(r), 1.0, 0.5, 20_000, 1e20, offset_exp=-1100)
    assert o["kind"] == "escaped" and o["n"] == n


def test_kat_rung_7676(dev):
    rung = KATS["rung_7676"]
    r = fdref.Ref.fixed(rung["re"], rung["im"], 3456, 150_000)
    rc = as_c(r)
    o = single(dev, rc, -0.5737130423454617, 0.290231303774763, 140_000, 1e20, offset_exp=-3310)
    assert o["kind"] == "escaped" and o["n"] == 133_115
    assert abs(o["zr"] / -27519423631.080235 - 1.0) < 1e-6
    assert abs(math.log2(math.hypot(o["dr"], o["di"])) + o["dexp"] - 3359.4391791173814) < 1e-6
    o = single(dev, rc, 0.006749565204064256, 0.10124347806096384, 140_000, 1e20, offset_exp=-3310)
    assert o["kind"] == "escaped" and o["n"] == 139_850
    p = fdref.plane(fdref.make_job(rung["re"], rung["im"], "5.050000000000E-998", 480, 270, 644_640))
    o = single(dev, rc, (184 + 0.5 - 240.0) * p["h_m"], -(201 + 0.5 - 135.0) * p["h_m"], 644_640, 1e20,
               offset_exp=p["h_e"])
    assert o["kind"] == "escaped" and o["n"] == 145_079


def test_kat_period3_interior_with_and_without_bla(dev):
    cr, ci = -1.7548776662466927, 0.0
    r = fdref.Ref.f64(cr, ci, 100_000, 1e10)
    rc = as_c(r)
    for e in (1e-16, 1e-18):
        t = fdref.Bla(r, 2.0 ** -50, 2.0 * e)
        b, offs = t.export()
        bla = fd.Bla(b, offs, 2.0 ** -50, 2.0 * e, 0, len(rc))
        for k in range(8):
            a = math.pi / 4 * k
            ar, ai = e * math.cos(a), e * math.sin(a)
            want = fdref.iterate(r, t, False, True, None, ar, ai, 0, 100_000, 1e20)
            got = single(dev, rc, ar, ai, 100_000, 1e20, bla=bla)
            plain = single(dev, rc, ar, ai, 100_000, 1e20)
            assert (got["kind"], got["n"]) == (want["kind"], want["n"]) == (plain["kind"], plain["n"])
            assert got["kind"] == "interior" and got["skipped"] > 0


def test_mask_rows_and_status(dev):
    view = fd.View("-0.7453", "0.1127", "0.0065")
    p = fd.Params(64, 32, max_iter=2000)
    r, bits = fd.reference(view, p)
    plane = fd.Plane.new(view, 64, 32)
    h = dev.upload(r)
    try:
        mask = (np.arange(64 * 32) % 3 == 0).astype(np.uint8)
        j = fd.route.make_job(plane, plane.tier, p, h, r.nucleus_period(), _lib.DERIVATIVE)
        j.mask = mask.ctypes.data
        j.first_row, j.rows = 5, 20
        a, cnt, _ = dev.render_job(j)
        full, _, _ = dev.render_job(fd.route.make_job(plane, plane.tier, p, h, r.nucleus_period(), _lib.DERIVATIVE))
    finally:
        dev.free(h)
    rows = np.zeros(64 * 32, bool)
    rows[5 * 64:25 * 64] = True
    sel = rows & (mask == 1)
    assert np.all(a["status"][sel] == 1) and np.all(a["status"][~sel] == 0)
    assert np.array_equal(a["cls"][sel], full["cls"][sel]) and np.array_equal(a["n"][sel], full["n"][sel])
    assert cnt.samples == sel.sum()


def test_column_window_host_and_device_outputs(dev):
    """A window of columns and rows (first_col/cols, first_row/rows) renders exactly the
    samples of the full frame inside it, with host outputs (staged as the window, with a
    mask and per-sample offsets) and with device outputs of whole rows; nothing outside it
    is written."""
    import torch
    view = fd.View("-0.7453", "0.1127", "0.0065")
    nx, ny = 72, 40
    p = fd.Params(nx, ny, max_iter=3000)
    r, bits = fd.reference(view, p)
    plane = fd.Plane.new(view, nx, ny)
    h = dev.upload(r)
    win = np.zeros((ny, nx), bool)
    win[7:30, 13:50] = True
    win = win.ravel()
    try:
        job = lambda: fd.route.make_job(plane, plane.tier, p, h, r.nucleus_period(), _lib.DERIVATIVE)
        full, _, _ = dev.render_job(job(), raw=True)
        j = job()
        j.first_row, j.rows, j.first_col, j.cols = 7, 23, 13, 37
        a, cnt, _ = dev.render_job(j, raw=True)
        assert cnt.samples == win.sum()
        assert np.all(a["status"][win] == 1) and np.all(a["status"][~win] == 0)
        for k in ("cls", "n", "nu", "de", "normal", "z", "dz", "dexp"):
            assert np.array_equal(a[k][win], full[k][win]), k
            assert not np.any(a[k][~win]), k
        # mask and offsets inside a window: the offsets of the grid reproduce the grid
        mask = (np.arange(nx * ny) % 4 != 1).astype(np.uint8)
        ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
        x, y = ii.ravel() + 0.5 - nx / 2.0, jj.ravel() + 0.5 - ny / 2.0
        offs = np.ascontiguousarray(np.stack([plane.cos_rot * x + plane.sin_rot * y,
                                              plane.sin_rot * x - plane.cos_rot * y], axis=1))
        j = job()
        j.first_row, j.rows, j.first_col, j.cols = 7, 23, 13, 37
        j.mask, j.offsets = mask.ctypes.data, offs.ctypes.data
        b, cnt, _ = dev.render_job(j, raw=True)
        sel = win & (mask == 1)
        assert cnt.samples == sel.sum() and np.all(b["status"][~sel] == 0)
        for k in ("cls", "n", "z", "dz", "dexp"):
            assert np.array_equal(b[k][sel], full[k][sel]), k
        # device outputs of whole rows
        bufs = {k: torch.zeros(nx * ny * (2 if k in ("z",) else 1), dtype=t, device="cuda:0")
                for k, t in (("cls", torch.uint8), ("n", torch.int32), ("status", torch.uint8), ("z", torch.float64))}
        j = job()
        j.first_row, j.rows, j.first_col, j.cols = 7, 23, 13, 37
        j.flags |= _lib.DEVICE_OUT
        dev.render_job(j, device_out={k: v.data_ptr() for k, v in bufs.items()})
        got = {k: v.cpu().numpy() for k, v in bufs.items()}
        assert np.array_equal(got["status"].astype(bool), win)
        assert np.array_equal(got["cls"][win], full["cls"][win])
        assert np.array_equal(got["n"].view(np.uint32)[win], full["n"][win])
        assert np.array_equal(got["z"].reshape(-1, 2)[win], full["z"][win])
        j.first_col, j.cols = 60, 13  # past the last column
        with pytest.raises(fd.route.RouteError, match="column range"):
            dev.render_job(j, device_out={k: v.data_ptr() for k, v in bufs.items()})
    finally:
        dev.free(h)


def test_invalid_inputs_are_refused_not_crashed(dev):
    L = _lib.lib()
    h = C.c_int32()
    z = np.zeros(4)
    bad = np.array([1.0, 0.0])
    assert L.fdc_upload_orbit(dev.h, bad.ctypes.data, bad.ctypes.data, 2, 53, C.byref(h)) == _lib.INVALID
    assert L.fdc_upload_orbit(dev.h, z.ctypes.data, z.ctypes.data, 1, 53, C.byref(h)) == _lib.INVALID
    j = _lib.Job()
    j.orbit = 12345
    out, cnt = _lib.Out(), _lib.Counters()
    assert L.fdc_render(dev.h, C.byref(j), C.byref(out), C.byref(cnt)) == _lib.INVALID
    r = fd.Reference.new(-0.75, 0.1, 100, 1e10)
    oh = dev.upload(r)
    try:
        j.orbit = oh
        j.nx = j.ny = j.ss = 4
        j.h_m, j.max_iter, j.escape_radius = 1.0, 100, 1e10
        j.flags = _lib.BLA  # no table uploaded
        assert L.fdc_render(dev.h, C.byref(j), C.byref(out), C.byref(cnt)) == _lib.INVALID
        j.flags = 0
        j.max_iter = 1 << 40
        assert L.fdc_render(dev.h, C.byref(j), C.byref(out), C.byref(cnt)) == _lib.INVALID
    finally:
        dev.free(oh)


@pytest.mark.parametrize("case", KATS["fnv_views"], ids=lambda c: c["width"])
def test_route_reproduces_reference_fds_hashes(dev, case):
    """End to end on the product side only: host orbit (fdh_orbit_*), CUDA kernel, host
    encoder (fdh_encode) and .fds writer give the reference's FNV-1a hashes of these renders
    (sample.rs:715-752), once the route's own kernel-id suffix is taken off."""
    from fractodactyl_b200 import fds
    view = fd.View(case["re"], case["im"], case["width"], 0.3)
    p = fd.Params(8, 4, max_iter=5000, columns=("nu", "de", "normal"))
    h, s, st, _ = fd.render_with(view, p, dev=dev, host_encode=True)
    h.kernel = h.kernel.replace(" gpu-perturb-cuda/1", "")
    assert fdref.fnv1a64(fds.encode(h, s, minor=0)) == int(case["fnv"], 16)


MPMATH = json.load(open(os.path.join(ROOT, "tests", "golden", "mpmath_checks.json")))


@pytest.mark.parametrize("rec", MPMATH, ids=lambda r: r["name"])
def test_route_writes_the_renders_mpmath_passed(dev, rec):
    """The route end to end (host orbit, host BLA builder, CUDA kernel, host encoder, .fds
    writer) writes, once its kernel-id suffix is taken off, the very bytes the reference's
    independent mpmath checker (tools/oracle.py) passed (tests/golden/mpmath_checks.json),
    and render_bla's BlaStats equal the oracle's, also for the seahorse table that admits
    no level at eps 2^-50 (grid.rs:526-529: the header still says bla/1)."""
    from fractodactyl_b200 import fds
    view = fd.View(rec["re"], rec["im"], rec["width"], rec["rotation"])
    p = fd.Params(rec["nx"], rec["ny"], max_iter=rec["max_iter"], columns=("nu", "de", "normal"))
    if rec["bla_eps"] is None:
        h, s, _, _ = fd.render_with(view, p, dev=dev, host_encode=True)
    else:
        h, s, _, bs = fd.render_bla(view, p, eps=rec["bla_eps"], dev=dev, host_encode=True)
        job = fdref.make_job(rec["re"], rec["im"], rec["width"], rec["nx"], rec["ny"], rec["max_iter"],
                             rotation=rec["rotation"], columns=fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL,
                             threads=2)
        ref = fdref.Ref.for_job(job)
        dc, e = fdref.bla_dc_bound(job)
        want = fdref.render(job, ref, fdref.Bla(ref, rec["bla_eps"], dc, e))["stats"]
        assert (bs.blocks, bs.skipped, bs.fallback_samples, bs.closed_form_samples) == (
            want["blocks"], want["skipped"], want["fallback_samples"], want["closed_form_samples"])
        assert h.kernel.endswith(" bla/1 gpu-perturb-cuda/1")
    h.kernel = h.kernel.replace(" gpu-perturb-cuda/1", "")
    assert "0x%016x" % fdref.fnv1a64(fds.encode(h, s)) == rec["fnv"]


@pytest.mark.parametrize("tile_w", [1, 8, 32])
def test_ragged_windows_and_tile_shapes(dev, tile_w):
    """Windows of odd sizes at the grid's edges (one column, one row, a single sample,
    the last rows and columns) under narrow, default and wide tiles equal the full
    frame's samples there, and nothing else is written."""
    view = fd.View("-0.7453", "0.1127", "0.0065")
    nx, ny = 37, 23
    p = fd.Params(nx, ny, max_iter=2500)
    r, bits = fd.reference(view, p)
    plane = fd.Plane.new(view, nx, ny)
    h = dev.upload(r)
    try:
        dev.tune(tile_w=tile_w)
        job = lambda: fd.route.make_job(plane, plane.tier, p, h, r.nucleus_period(), _lib.DERIVATIVE)
        full, _, _ = dev.render_job(job(), raw=True)
        for (x0, cw, y0, rh) in ((nx - 1, 1, 0, ny), (0, nx, ny - 1, 1), (nx - 1, 1, ny - 1, 1), (5, 31, 3, 19),
                                 (0, 1, 0, 1)):
            j = job()
            j.first_col, j.cols, j.first_row, j.rows = x0, cw, y0, rh
            a, cnt, _ = dev.render_job(j, raw=True)
            win = np.zeros((ny, nx), bool)
            win[y0:y0 + rh, x0:x0 + cw] = True
            win = win.ravel()
            assert cnt.samples == win.sum() and np.all(a["status"][~win] == 0)
            for k in ("cls", "n", "z", "dz", "dexp", "nu"):
                assert np.array_equal(a[k][win], full[k][win]), (k, x0, cw, y0, rh)
    finally:
        dev.tune(tile_w=0)
        dev.free(h)
