"""The plain-form CUDA kernel's own source (fractodactyl_b200/csrc/perturb_f64.cuh) built
for the host (tests/emu: builtins shimmed, the persistent kernel run as a single-lane
warp) against the oracle, on the CPU: class, escape count, z, dz/dc and the work
counters bit for bit on the F64, Fixed and Scaled tiers with and without BLA and the
derivative, from a parameter-series start (with its retries from zero) and in the
bounded variant (error radii, Bounded evidence, Bound column), in windows with masks,
offsets and tile orders, and as batches. Host libm stands in for
CUDA's, so nu, de and the Bound column also equal the oracle's here. This checks the
kernel's state machine without a GPU; its arithmetic on the device is checked by the
GPU suite. The precision form (perturb_f32.cuh) runs here too, without the device's fused
multiply-adds, so it is held to its own agreement bars rather than to bit equality."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
KATS = json.load(open(os.path.join(HERE, "golden", "kats.json")))
LIB = os.path.join(HERE, "emu", "libemu.so")
SEAHORSE = ("-0.743643887037158", "0.131825904205312")


@pytest.fixture(scope="module")
def emu():
    src = [os.path.join(HERE, "emu", "emu.cpp"), os.path.join(HERE, "emu", "cuda_host_shim.hpp"),
           os.path.join(ROOT, "fractodactyl_b200", "csrc", "perturb_f64.cuh"),
           os.path.join(ROOT, "fractodactyl_b200", "csrc", "perturb_f32.cuh"),
           os.path.join(ROOT, "fractodactyl_b200", "csrc", "fd_device.cuh"),
           os.path.join(ROOT, "fractodactyl_b200", "csrc", "bla_build.cuh")]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(s) for s in src):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-Wno-unknown-pragmas",
                        "-I", os.path.join(HERE, "emu"), "-I", os.path.join(ROOT, "fractodactyl_b200", "csrc"),
                        src[0], "-o", LIB], check=True)
    L = C.CDLL(LIB)
    P, D, U32, U64, I32, I64 = C.c_void_p, C.c_double, C.c_uint32, C.c_uint64, C.c_int32, C.c_int64
    L.emu_render.restype = C.c_int
    L.emu_render.argtypes = [P, P, U64, P, P, U32, P, U32, U32, D, P, I32, U32, U32, U32, U32, D, D, D, I64, D, D,
                             U32, D, I64] + [P] * 12 + [P]
    L.emu_render_window.restype = C.c_int
    L.emu_render_window.argtypes = L.emu_render.argtypes + [C.POINTER(Window)]
    L.emu_render_batch.restype = C.c_int
    L.emu_render_batch.argtypes = [C.POINTER(Job), U32]
    L.emu_set_stripe.argtypes = [U32, D, P]
    L.emu_hypot_check.restype = U64
    L.emu_hypot_check.argtypes = [P, P, U64]
    L.emu_bla_build.restype = U32
    L.emu_bla_build.argtypes = [P, P, U64, D, D, I64, P]
    return L


class Window(C.Structure):
    """emu.cpp's EmuWindow: fdc_job's window, mask and offsets (whole-frame arrays), the
    tile width 2^tile_shift, the tile order (0 row-major, 1 reversed) and the deadline in
    ns of the emulated clock (1 us per read)."""
    _fields_ = [("first_row", C.c_uint32), ("rows", C.c_uint32), ("first_col", C.c_uint32), ("cols", C.c_uint32),
                ("tile_shift", C.c_uint32), ("tile_order", C.c_uint32), ("mask", C.c_void_p),
                ("offsets", C.c_void_p), ("deadline_ns", C.c_uint64)]


class Job(C.Structure):
    """emu.cpp's EmuJob: one batch job (orbit, BLA table, frame, window, outputs) and its
    returned counters."""
    _fields_ = [("re", C.c_void_p), ("im", C.c_void_p), ("len", C.c_uint64), ("blocks7", C.c_void_p),
                ("level_offsets", C.c_void_p), ("levels", C.c_uint32), ("tier", C.c_int32), ("flags", C.c_uint32),
                ("nx", C.c_uint32), ("ny", C.c_uint32), ("ss", C.c_uint32), ("max_iter", C.c_uint32),
                ("c_re", C.c_double), ("c_im", C.c_double), ("h_m", C.c_double), ("h_e", C.c_int64),
                ("cos_rot", C.c_double), ("sin_rot", C.c_double), ("escape_radius", C.c_double),
                ("nucleus", C.c_int64), ("first_row", C.c_uint32), ("rows", C.c_uint32), ("first_col", C.c_uint32),
                ("cols", C.c_uint32)] + [(k, C.c_void_p) for k in ("cls", "n", "nu", "de", "normal", "z", "dz", "dexp",
                                                                    "status")] + [("counters", C.c_uint64 * 6)]


def _ptr(a):
    return None if a is None else a.ctypes.data


def emulate(emu, r, plane, tier, p, flags, bla=None, series=None, q=None, nucleus=None, win=None, timed_out=False):
    n = p.nx * p.ny
    out = dict(cls=np.zeros(n, np.uint8), n=np.zeros(n, np.uint32), nu=np.zeros(n), de=np.zeros(n, np.float32),
               normal=np.zeros(n, np.uint16), z=np.zeros((n, 2)), dz=np.zeros((n, 2)), dexp=np.zeros(n, np.int64),
               status=np.zeros(n, np.uint8), bound=np.zeros(n, np.float32), ez=np.zeros(n), ed=np.zeros(n))
    cnt = np.zeros(6, np.uint64)
    re_, im_ = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
    blocks = offs = sb = None
    if bla is not None:
        blocks = np.ascontiguousarray(bla.blocks)
        offs = np.ascontiguousarray(bla.level_offsets, dtype=np.uint64)
    if series is not None:
        sb = np.ascontiguousarray(series.b, dtype=np.float64)
    nuc = r.nucleus_period() if nucleus is None else nucleus
    args = (_ptr(re_), _ptr(im_), len(re_), _ptr(blocks), _ptr(offs), bla.levels if bla else 0, _ptr(sb),
            len(sb) if sb is not None else 0, series.n if series else 0, series.rho if series else 0.0,
            _ptr(q), tier, flags, p.nx, p.ny, p.ss, plane.c_re, plane.c_im, plane.h_m, plane.h_e,
            plane.cos_rot, plane.sin_rot, p.max_iter, p.escape_radius, -1 if nuc is None else nuc,
            *[_ptr(out[k]) for k in ("cls", "n", "nu", "de", "normal", "z", "dz", "dexp", "status", "bound",
                                     "ez", "ed")], _ptr(cnt))
    rc = emu.emu_render(*args) if win is None else emu.emu_render_window(*args, C.byref(win))
    assert rc == (1 if timed_out else 0)
    out["counters"] = dict(zip(("samples", "iterations", "blocks", "skipped", "fallback_samples",
                                "closed_form_samples"), (int(c) for c in cnt)))
    return out


def _setup(view3, nx, ny, max_iter, tier=None, columns=("nu", "de", "normal")):
    v = fd.View(*view3)
    p = fd.Params(nx, ny, max_iter=max_iter, columns=columns, tier=tier)
    plane, t = fd.route._setup(v, p)
    r, bits = fd.reference(v, p)
    r.bits = bits
    plane.bits = bits
    return v, p, plane, t, r


def _oracle_job(view3, p, tier, columns):
    return fdref.make_job(*view3, p.nx, p.ny, p.max_iter, escape_radius=p.escape_radius, columns=columns, tier=tier,
                          threads=2)


def _check(got, want, counters=True, escaped=True):
    assert np.array_equal(got["cls"], want["cls"])
    assert np.array_equal(got["n"], want["n"].astype(np.uint32))
    esc = (want["cls"] & 3) == 0
    assert esc.any() or not escaped
    for k in ("z", "dz", "dexp"):
        if k in want:
            assert np.array_equal(got[k][esc], want[k][esc]), k
    assert np.array_equal(got["nu"][esc], want["nu"][esc])
    assert np.array_equal(got["de"][esc], want["de"][esc])
    assert np.all(np.abs(got["normal"][esc].astype(np.int64) - want["normal"][esc]) <= 1)
    assert got["status"].all()
    if counters:
        st = want["stats"]
        for k in ("iterations", "blocks", "skipped", "fallback_samples", "closed_form_samples"):
            assert got["counters"][k] == st[k], k


@pytest.mark.parametrize("case", ["f64", "f64-bla", "fixed-bla", "scaled-bla", "scaled-nod"])
def test_kernel_equals_oracle(emu, case):
    eps = fd.route.EPS
    if case == "f64":
        view3, nx, ny, it, tier = ("-0.7453", "0.1127", "0.0065"), 40, 24, 4_000, None
    elif case == "f64-bla":  # F64-tier depths admit no block at eps 2^-50: a looser table
        view3, nx, ny, it, tier, eps = (*SEAHORSE, "1e-10"), 40, 24, 20_000, None, 2.0 ** -30
    elif case == "fixed-bla":  # a series frame deep enough for eps 2^-50 blocks
        f = KATS["series_frames"][18]
        view3, nx, ny, it, tier = (f["re"], f["im"], f["width"]), 33, 19, 10_000, None
    else:
        view3, nx, ny, it, tier = ("0", "1", "1e-300"), 32, 16, 5_000, None
    bla = "bla" in case
    cols = ("nu",) if case == "scaled-nod" else ("nu", "de", "normal")
    v, p, plane, t, r = _setup(view3, nx, ny, it, tier, cols)
    table = None
    if bla:
        dc, e = fd.bla_dc_bound(v, p)
        table = fd.Bla.build_scaled(r, eps, dc, e)
        assert table.levels > 0
    flags = (1 if p.needs_derivative() else 0) | (2 if bla else 0)
    got = emulate(emu, r, plane, t, p, flags, bla=table)
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    ob = fdref.Bla(ref, eps, table.dc_max, table.dc_exp) if bla else None
    ocols = fdref.COL_NU | (fdref.COL_DE | fdref.COL_NORMAL if p.needs_derivative() else 0)
    want = fdref.render(_oracle_job(view3, p, t, ocols), ref, ob, raw=True)
    if not p.needs_derivative():  # the oracle's dz without the derivative is not a column
        want.pop("dz")
        want.pop("dexp")
        got["de"][:] = want["de"]
        got["normal"][:] = want["normal"]
    _check(got, want)
    if bla:
        assert got["counters"]["blocks"] > 0


@pytest.mark.parametrize("frame", [18, -1])
def test_kernel_series_start_equals_oracle(emu, frame):
    """Frame 18 (BLA blocks, a few unresolved starts) and the nucleus frame, whose series
    admits 9,999 of 10,000 iterations so nearly every sample retries from zero."""
    f = KATS["series_frames"][frame]
    view3 = (f["re"], f["im"], f["width"])
    v, p, plane, t, r = _setup(view3, 33, 19, 10_000)
    rho, e = fd.bla_dc_bound(v, p)
    series = fd.Series.build(r, rho, float(f["width"]) / 33, p.max_iter)
    assert series.n > 0
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    o_series = fdref.Series(ref, rho, float(f["width"]) / 33, p.max_iter)
    table = ob = None
    if frame == 18:
        table = fd.Bla.build_scaled(r, fd.route.EPS, rho, 0)
        ob = fdref.Bla(ref, fd.route.EPS, rho, 0)
    got = emulate(emu, r, plane, t, p, 1 | (2 if table else 0) | 4, bla=table, series=series)
    want = fdref.render_series(_oracle_job(view3, p, t, fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL), ref,
                               o_series, bla=ob, raw=True)
    _check(got, want, escaped=frame == 18)  # the nucleus frame has no escaping sample
    if frame == -1:
        assert (got["cls"] & 3 == 1).any()  # its interior survives the retries (series.rs:644-693)


@pytest.mark.parametrize("view3,max_iter", [(("-0.7453", "0.1127", "0.0065"), 4_000),
                                           ((*SEAHORSE, "1e-14"), 20_000)])
def test_kernel_bounded_equals_oracle(emu, view3, max_iter):
    v, p, plane, t, r = _setup(view3, 40, 24, max_iter, columns=("nu", "de", "bound"))
    q = r.error_radius(None if t == 0 else r.bits, plane.c_re, plane.c_im)
    got = emulate(emu, r, plane, t, p, 1 | 8, q=q)
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    want = fdref.render_columns(_oracle_job(view3, p, t, fdref.COL_NU | fdref.COL_DE | fdref.COL_BOUND), ref)
    esc = (want["cls"] & 3) == 0
    assert (want["cls"] == 4).sum() > 0.5 * esc.sum()
    for k in ("cls", "bound"):
        assert np.array_equal(got[k], want[k]), k
    assert np.array_equal(got["n"], want["n"].astype(np.uint32))
    for k in ("z", "ez", "ed", "nu", "de"):
        assert np.array_equal(got[k][esc], want[k][esc]), k
    assert got["counters"]["iterations"] == want["stats"]["iterations"]


def test_kernel_fuzz_equals_oracle(emu):
    """Seeded random frames on structure at every depth (the seeded nucleus locations of
    1e-20 .. 1e-1000 and the reference's series frames, each at a random multiple of its
    width, plus classic shallow views; every tier, derivative and BLA on or off): the
    emulated kernel equals the oracle on each."""
    from fractodactyl_b200 import locations
    rng = np.random.default_rng(20261203)
    views = [(d["re"], d["im"], float(d["log10_width"])) for d in locations.cached("c5")]
    views += [(f["re"], f["im"], float(np.log10(float(f["width"])))) for f in KATS["series_frames"]]
    views += [("-0.7453", "0.1127", np.log10(0.0065)), (*SEAHORSE, -10.0), ("-0.1011", "0.9563", -3.0)]
    kinds, tiers, blocks = set(), set(), 0
    for case in range(36):
        re_, im_, lw = views[int(rng.integers(0, len(views)))]
        width = f"{10 ** (lw % 1) * rng.uniform(0.5, 4):.4f}e{int(np.floor(lw))}"
        max_iter = int(rng.integers(2_000, 20_000))
        deriv, bla = bool(rng.integers(0, 2)), bool(rng.integers(0, 2))
        cols = ("nu", "de", "normal") if deriv else ("nu",)
        view3 = (re_, im_, width)
        v, p, plane, t, r = _setup(view3, 12, 8, max_iter, None, cols)
        table = ob = None
        if bla:
            dc, e = fd.bla_dc_bound(v, p)
            table = fd.Bla.build_scaled(r, fd.route.EPS if t else 2.0 ** -30, dc, e)
            if table.levels == 0:
                table = None
        got = emulate(emu, r, plane, t, p, (1 if deriv else 0) | (2 if table else 0), bla=table)
        ref = fdref.Ref.arrays(r.re, r.im, r.bits)
        if table is not None:
            ob = fdref.Bla(ref, table.eps, table.dc_max, table.dc_exp)
        ocols = fdref.COL_NU | (fdref.COL_DE | fdref.COL_NORMAL if deriv else 0)
        want = fdref.render(_oracle_job(view3, p, t, ocols), ref, ob, raw=True)
        assert np.array_equal(got["cls"], want["cls"]), (case, view3, max_iter, deriv, bla)
        assert np.array_equal(got["n"], want["n"].astype(np.uint32)), (case, view3)
        esc = (want["cls"] & 3) == 0
        assert np.array_equal(got["z"][esc], want["z"][esc]), (case, view3)
        if deriv:
            assert np.array_equal(got["dz"][esc], want["dz"][esc]) and np.array_equal(got["dexp"][esc],
                                                                                     want["dexp"][esc]), (case, view3)
        for k in ("iterations", "blocks", "skipped"):
            assert got["counters"][k] == want["stats"][k], (case, view3, k)
        kinds |= set(np.unique(want["cls"] & 3).tolist())
        tiers.add(t)
        blocks += want["stats"]["blocks"]
    assert kinds == {0, 1, 2} and tiers == {0, 1, 2} and blocks > 0  # the draw covers every path


def test_kernel_fuzz_series_and_bounded_equal_oracle(emu):
    """Seeded random ordinary-tier frames on the same locations, started from their
    parameter series (BLA on or off) or rendered bounded: the emulated kernel equals the
    oracle's render_series / bounded render on each."""
    from fractodactyl_b200 import locations
    rng = np.random.default_rng(20261204)
    views = [(d["re"], d["im"], float(d["log10_width"])) for d in locations.cached("c5")
             if float(d["log10_width"]) > -260]
    views += [(f["re"], f["im"], float(np.log10(float(f["width"])))) for f in KATS["series_frames"]]
    views += [(*SEAHORSE, -10.0), (*SEAHORSE, -14.0)]
    started, bounded_samples = 0, 0
    for case in range(24):
        re_, im_, lw = views[int(rng.integers(0, len(views)))]
        width = f"{10 ** (lw % 1) * rng.uniform(0.5, 4):.4f}e{int(np.floor(lw))}"
        max_iter = int(rng.integers(2_000, 20_000))
        view3 = (re_, im_, width)
        if case % 2 == 0:  # series start
            v, p, plane, t, r = _setup(view3, 11, 7, max_iter)
            if t == 2:
                continue
            rho, _ = fd.bla_dc_bound(v, p)
            pixel = float(width) / 11
            series = fd.Series.build(r, rho, pixel, max_iter)
            if series.n == 0:
                continue
            ref = fdref.Ref.arrays(r.re, r.im, r.bits)
            table = fd.Bla.build_scaled(r, fd.route.EPS, rho, 0) if rng.integers(0, 2) else None
            table = table if table is not None and table.levels else None
            ob = fdref.Bla(ref, fd.route.EPS, rho, 0) if table is not None else None
            got = emulate(emu, r, plane, t, p, 1 | (2 if table else 0) | 4, bla=table, series=series)
            want = fdref.render_series(_oracle_job(view3, p, t, fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL),
                                       ref, fdref.Series(ref, rho, pixel, max_iter), bla=ob, raw=True)
            _check(got, want, escaped=False)
            started += 1
        else:  # bounded
            v, p, plane, t, r = _setup(view3, 11, 7, max_iter, columns=("nu", "de", "bound"))
            if t == 2:
                continue
            q = r.error_radius(None if t == 0 else r.bits, plane.c_re, plane.c_im)
            got = emulate(emu, r, plane, t, p, 1 | 8, q=q)
            want = fdref.render_columns(_oracle_job(view3, p, t, fdref.COL_NU | fdref.COL_DE | fdref.COL_BOUND),
                                        fdref.Ref.arrays(r.re, r.im, r.bits))
            for k in ("cls", "bound"):
                assert np.array_equal(got[k], want[k]), (case, view3, k)
            assert np.array_equal(got["n"], want["n"].astype(np.uint32)), (case, view3)
            esc = (want["cls"] & 3) == 0
            for k in ("z", "ez", "ed", "de"):
                assert np.array_equal(got[k][esc], want[k][esc]), (case, view3, k)
            bounded_samples += int((want["cls"] == 4).sum())
    assert started >= 4 and bounded_samples > 0


def _grid_offsets(plane, nx, ny):
    """Every sample's unit offset from the centre, as the kernel derives it from the grid
    (view.rs:118-122), frame-major (nx*ny, 2)."""
    j, i = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    x = i + 0.5 - nx / 2.0
    y = j + 0.5 - ny / 2.0
    ux = plane.cos_rot * x + plane.sin_rot * y
    uy = plane.sin_rot * x - plane.cos_rot * y
    return np.ascontiguousarray(np.stack([ux.ravel(), uy.ravel()], axis=1))


@pytest.mark.parametrize("case", ["f64-bla", "fixed-bla", "scaled"])
def test_kernel_window_mask_offsets_equal_oracle(emu, case):
    """The job inputs the other emulation tests leave at their defaults: a window of rows and
    columns, a mask, 4x8 tiles handed out in reverse order, and per-sample offsets. The
    windowed, masked render writes exactly the selected samples, each equal to the oracle's
    masked render (columns and work counters), and nothing else; offsets equal to the grid's
    own positions reproduce the grid render bit for bit; jittered offsets equal the oracle's
    iteration of each sample at its own offset."""
    rng = np.random.default_rng(20261205)
    eps = fd.route.EPS
    if case == "f64-bla":
        view3, nx, ny, it, eps = (*SEAHORSE, "1e-10"), 40, 24, 20_000, 2.0 ** -30
    elif case == "fixed-bla":
        f = KATS["series_frames"][18]
        view3, nx, ny, it = (f["re"], f["im"], f["width"]), 33, 19, 10_000
    else:
        view3, nx, ny, it = ("0", "1", "1e-300"), 32, 16, 5_000
    v, p, plane, t, r = _setup(view3, nx, ny, it)
    table = ob = None
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    if "bla" in case:
        dc, e = fd.bla_dc_bound(v, p)
        table = fd.Bla.build_scaled(r, eps, dc, e)
        assert table.levels > 0
        ob = fdref.Bla(ref, eps, table.dc_max, table.dc_exp)
    flags = 1 | (2 if table else 0)
    full = emulate(emu, r, plane, t, p, flags, bla=table)
    r0, rows, c0, cols = 3, ny - 8, 5, nx - 11
    inwin = np.zeros((ny, nx), bool)
    inwin[r0:r0 + rows, c0:c0 + cols] = True
    inwin = inwin.ravel()
    mask = (rng.random(nx * ny) < 0.6).astype(np.uint8)
    sel = inwin & (mask != 0)
    win = Window(r0, rows, c0, cols, 2, 1, mask.ctypes.data, None)
    got = emulate(emu, r, plane, t, p, flags, bla=table, win=win)
    want = fdref.render_columns(_oracle_job(view3, p, t, fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL), ref, ob,
                                mask=sel.astype(np.uint8))
    assert sel.sum() > 0.3 * inwin.sum()
    assert np.array_equal(got["status"] != 0, sel)
    assert not got["cls"][~sel].any() and not got["n"][~sel].any() and not got["z"][~sel].any()
    assert np.array_equal(got["cls"][sel], want["cls"][sel])
    assert np.array_equal(got["n"][sel], want["n"][sel].astype(np.uint32))
    esc = sel & ((want["cls"] & 3) == 0)
    assert esc.any()
    for k in ("z", "dz", "dexp", "nu", "de"):
        assert np.array_equal(got[k][esc], want[k][esc]), k
        assert np.array_equal(got[k][sel], full[k][sel]), k
    for k in ("iterations", "blocks", "skipped", "fallback_samples", "closed_form_samples"):
        assert got["counters"][k] == want["stats"][k], k
    # offsets at the grid's own positions: the grid render, over the window
    grid = _grid_offsets(plane, nx, ny)
    got = emulate(emu, r, plane, t, p, flags, bla=table, win=Window(r0, rows, c0, cols, 3, 0, None, grid.ctypes.data))
    for k in ("cls", "n", "z", "dz", "dexp", "nu", "de", "normal"):
        assert np.array_equal(got[k][inwin], full[k][inwin]), k
    assert np.array_equal(got["status"] != 0, inwin)
    # jittered offsets: each sample is the oracle's iteration at its own offset
    jit = np.ascontiguousarray(grid + rng.uniform(-0.5, 0.5, grid.shape))
    got = emulate(emu, r, plane, t, p, flags, bla=table, win=Window(r0, rows, c0, cols, 5, 1, None, jit.ctypes.data))
    h = np.ldexp(plane.h_m, plane.h_e)
    kinds = {"escaped": 0, "interior": 1, "unresolved": 2}
    for k in np.flatnonzero(inwin):
        ux, uy = jit[k]
        if t == 2:
            o = fdref.iterate(ref, ob, extended=True, ar=ux * plane.h_m, ai=uy * plane.h_m, offset_exp=plane.h_e,
                              max_iter=it, r2=p.escape_radius ** 2)
        else:
            ar, ai = ux * h, uy * h
            o = fdref.iterate(ref, ob, c=(plane.c_re + ar, plane.c_im + ai) if t == 0 else None, ar=ar, ai=ai,
                              max_iter=it, r2=p.escape_radius ** 2)
        assert got["cls"][k] & 3 == kinds[o["kind"]], k
        assert got["n"][k] == (it if o["kind"] == "unresolved" else o["n"]), k
        if o["kind"] == "escaped":
            assert tuple(got["z"][k]) == (o["zr"], o["zi"]) and tuple(got["dz"][k]) == (o["dr"], o["di"]), k
            assert got["dexp"][k] == o["dexp"], k


def _outputs(n):
    return dict(cls=np.zeros(n, np.uint8), n=np.zeros(n, np.uint32), nu=np.zeros(n), de=np.zeros(n, np.float32),
                normal=np.zeros(n, np.uint16), z=np.zeros((n, 2)), dz=np.zeros((n, 2)), dexp=np.zeros(n, np.int64),
                status=np.zeros(n, np.uint8))


@pytest.mark.parametrize("raw", [True, False], ids=["raw-outputs", "columns-only"])
def test_batch_kernel_equals_oracle(emu, raw):
    """The batch kernel as fdc_batch_create groups a mixed batch (jobs of every tier, with and
    without BLA and the derivative, so several variant groups whose jobs are reordered deepest
    first; one frame split into three row tiles that write one shared output): every job's
    samples equal the oracle's frame, and every job's counters equal the oracle's render of
    just that job's samples (its window as a mask). Without raw outputs (no z, dz/dc or
    exponent columns) the BLA jobs' raw state goes to scratch and the encode pass still
    writes nu, de and normal."""
    frame18 = KATS["series_frames"][18]
    specs = [  # view, nx, ny, max_iter, BLA eps (None: no table), derivative, row tiles
        ((*SEAHORSE, "1e-10"), 24, 16, 20_000, 2.0 ** -30, True, 1),
        ((frame18["re"], frame18["im"], frame18["width"]), 33, 19, 10_000, fd.route.EPS, True, 3),
        (("0", "1", "1e-300"), 32, 16, 5_000, fd.route.EPS, False, 1),
        (("-0.7453", "0.1127", "0.0065"), 20, 12, 4_000, None, True, 1),
        ((frame18["re"], frame18["im"], frame18["width"]), 16, 8, 10_000, None, False, 1),
    ]
    keep, jobs, frames = [], [], []
    for view3, nx, ny, it, eps, deriv, tiles in specs:
        cols = ("nu", "de", "normal") if deriv else ("nu",)
        v, p, plane, t, r = _setup(view3, nx, ny, it, None, cols)
        table = ob = None
        ref = fdref.Ref.arrays(r.re, r.im, r.bits)
        if eps is not None:
            dc, e = fd.bla_dc_bound(v, p)
            table = fd.Bla.build_scaled(r, eps, dc, e)
            assert table.levels > 0
            ob = fdref.Bla(ref, eps, table.dc_max, table.dc_exp)
        out = _outputs(nx * ny)
        re_, im_ = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
        blocks = offs = None
        if table is not None:
            blocks = np.ascontiguousarray(table.blocks)
            offs = np.ascontiguousarray(table.level_offsets, dtype=np.uint64)
        keep += [re_, im_, blocks, offs]
        nuc = r.nucleus_period()
        edges = np.linspace(0, ny, tiles + 1).astype(int)
        windows = []
        for a, b in zip(edges[:-1], edges[1:]):
            j = Job(re=re_.ctypes.data, im=im_.ctypes.data, len=len(re_), blocks7=_ptr(blocks),
                    level_offsets=_ptr(offs), levels=table.levels if table else 0, tier=t,
                    flags=(1 if deriv else 0) | (2 if table else 0), nx=nx, ny=ny, ss=p.ss, max_iter=it,
                    c_re=plane.c_re, c_im=plane.c_im, h_m=plane.h_m, h_e=plane.h_e, cos_rot=plane.cos_rot,
                    sin_rot=plane.sin_rot, escape_radius=p.escape_radius, nucleus=-1 if nuc is None else nuc,
                    first_row=int(a), rows=int(b - a) if tiles > 1 else 0, first_col=0, cols=0,
                    **{k: out[k].ctypes.data for k in out if raw or k not in ("z", "dz", "dexp")})
            windows.append((len(jobs), int(a), int(b)))
            jobs.append(j)
        ocols = fdref.COL_NU | (fdref.COL_DE | fdref.COL_NORMAL if deriv else 0)
        frames.append((view3, p, t, ref, ob, ocols, deriv, out, windows))
    arr = (Job * len(jobs))(*jobs)
    assert emu.emu_render_batch(arr, len(jobs)) == 0
    tiers = set()
    for view3, p, t, ref, ob, ocols, deriv, out, windows in frames:
        want = fdref.render(_oracle_job(view3, p, t, ocols), ref, ob, raw=True)
        tiers.add(t)
        assert out["status"].all()
        assert np.array_equal(out["cls"], want["cls"]), view3
        assert np.array_equal(out["n"], want["n"].astype(np.uint32)), view3
        esc = (want["cls"] & 3) == 0
        assert np.array_equal(out["nu"][esc], want["nu"][esc])
        if raw:
            assert np.array_equal(out["z"][esc], want["z"][esc])
        if deriv:
            for k in (("dz", "dexp", "de") if raw else ("de", "normal")):
                assert np.array_equal(out[k][esc], want[k][esc]), (view3, k)
        for k, a, b in windows:
            m = np.zeros((p.ny, p.nx), np.uint8)
            m[a:b] = 1
            st = fdref.render_columns(_oracle_job(view3, p, t, ocols), ref, ob, mask=m.ravel())["stats"]
            got = dict(zip(("samples", "iterations", "blocks", "skipped", "fallback_samples", "closed_form_samples"),
                           (int(c) for c in arr[k].counters)))
            assert got["samples"] == (b - a) * p.nx, (view3, a, b)
            for key in ("iterations", "blocks", "skipped", "fallback_samples", "closed_form_samples"):
                assert got[key] == st[key], (view3, a, b, key)
    assert tiers == {0, 1, 2}


PRECISION_VIEWS = [  # view, nx, ny, max_iter, chaotic (the precision form's GPU bars per view)
    (("-0.7453", "0.1127", "0.0065"), 64, 36, 20_000, True),
    (("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28"), 64, 36, 50_000, True),
    (("0", "1", "1e-300"), 64, 36, 20_000, False),
    (("-0.7436438870371587", "0.1318259042053120", "1e-12"), 60, 34, 20_000, True),
]


@pytest.mark.parametrize("view,bla", [(v, False) for v in PRECISION_VIEWS] +
                         [(v, True) for v in PRECISION_VIEWS[1:3]],  # F64-tier views admit no block at 2^-50
                         ids=lambda x: x[0][2] if isinstance(x, tuple) else ("bla" if x else "plain"))
def test_precision_form_kernel_meets_its_bars(emu, view, bla):
    """The precision-form kernel (perturb_f32.cuh, host float arithmetic without fused
    multiply-adds, so not the device's roundings) against the oracle's FP64 render, held to
    the bars its GPU tests set: escape agreement >= 99% and equal counts >= 75% on chaotic
    views, equal counts >= 99.9% and none more than one apart on the non-chaotic view; smooth
    iteration within 1e-5 relative (median) or 1e-6 (p99) where the counts agree."""
    view3, nx, ny, it, chaotic = view
    v, p, plane, t, r = _setup(view3, nx, ny, it)
    table = ob = None
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    if bla:
        dc, e = fd.bla_dc_bound(v, p)
        table = fd.Bla.build_scaled(r, fd.route.EPS, dc, e)
        assert table.levels > 0
        ob = fdref.Bla(ref, fd.route.EPS, table.dc_max, table.dc_exp)
    got = emulate(emu, r, plane, t, p, 1 | (2 if table else 0) | 16, bla=table)
    want = fdref.render(_oracle_job(view3, p, t, fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL), ref, ob, raw=True)
    assert got["status"].all()
    ea, eb = (want["cls"] & 3) == 0, (got["cls"] & 3) == 0
    dn = np.abs(want["n"].astype(np.int64) - got["n"].astype(np.int64))
    same = ((ea == eb) & (~ea | (dn == 0))).mean()
    off1 = ((ea == eb) & (~ea | (dn <= 1))).mean()
    escaping = (ea == eb).mean()
    agree = ea & eb & (dn == 0)
    rel = np.abs(want["nu"][agree] - got["nu"][agree]) / np.abs(want["nu"][agree])
    assert agree.any()
    if chaotic:
        assert escaping >= 0.99 and same >= 0.75, (same, escaping)
        assert np.median(rel) <= 1e-5
    else:
        assert same >= 0.999 and off1 == 1.0, (same, off1)
        assert np.quantile(rel, 0.99) <= 1e-6 and rel.max() <= 1e-3
    if table is not None:
        assert got["counters"]["blocks"] > 0


def test_precision_form_batch_equals_single_frames(emu):
    """The precision form's batch kernel over a mixed batch (three tiers, BLA on and off, one
    frame in three row tiles) writes exactly what the precision form's frame kernel writes
    for each frame, with equal per-job counters."""
    specs = [(("-0.7453", "0.1127", "0.0065"), 24, 16, 4_000, False, 1),
             (("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28"), 33, 19,
              50_000, True, 3),
             (("0", "1", "1e-300"), 32, 16, 5_000, True, 1)]
    keep, jobs, frames = [], [], []
    for view3, nx, ny, it, bla, tiles in specs:
        v, p, plane, t, r = _setup(view3, nx, ny, it)
        table = None
        if bla:
            dc, e = fd.bla_dc_bound(v, p)
            table = fd.Bla.build_scaled(r, fd.route.EPS, dc, e)
            assert table.levels > 0
        single = emulate(emu, r, plane, t, p, 1 | (2 if table else 0) | 16, bla=table)
        out = _outputs(nx * ny)
        re_, im_ = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
        blocks = offs = None
        if table is not None:
            blocks = np.ascontiguousarray(table.blocks)
            offs = np.ascontiguousarray(table.level_offsets, dtype=np.uint64)
        keep += [re_, im_, blocks, offs]
        nuc = r.nucleus_period()
        edges = np.linspace(0, ny, tiles + 1).astype(int)
        ids = []
        for a, b in zip(edges[:-1], edges[1:]):
            ids.append(len(jobs))
            jobs.append(Job(re=re_.ctypes.data, im=im_.ctypes.data, len=len(re_), blocks7=_ptr(blocks),
                            level_offsets=_ptr(offs), levels=table.levels if table else 0, tier=t,
                            flags=1 | (2 if table else 0) | 4, nx=nx, ny=ny, ss=p.ss, max_iter=it, c_re=plane.c_re,
                            c_im=plane.c_im, h_m=plane.h_m, h_e=plane.h_e, cos_rot=plane.cos_rot,
                            sin_rot=plane.sin_rot, escape_radius=p.escape_radius,
                            nucleus=-1 if nuc is None else nuc, first_row=int(a),
                            rows=int(b - a) if tiles > 1 else 0, first_col=0, cols=0,
                            **{k: out[k].ctypes.data for k in out}))
        frames.append((single, out, ids, t))
    arr = (Job * len(jobs))(*jobs)
    assert emu.emu_render_batch(arr, len(jobs)) == 0
    assert {f[3] for f in frames} == {0, 1, 2}
    for single, out, ids, _ in frames:
        for k in ("cls", "n", "nu", "de", "normal", "z", "dz", "dexp", "status"):
            assert np.array_equal(out[k], single[k]), k
        total = np.sum([np.array(arr[i].counters, dtype=np.uint64) for i in ids], axis=0)
        assert [int(c) for c in total] == [single["counters"][k] for k in (
            "samples", "iterations", "blocks", "skipped", "fallback_samples", "closed_form_samples")]


@pytest.mark.parametrize("case", ["f64", "scaled-bla", "precision"])
def test_deadline_stops_taking_samples(emu, case):
    """A job's deadline (fdc_job.deadline_ms; here on the emulated clock, 1 us per read):
    once it has passed, warps take no new samples, finish the ones they hold and raise the
    timed-out flag (FDC_TIMEOUT). Exactly the samples taken are written (status 1, equal
    to the unlimited render's), the rest keep zeroed columns and status 0, and the counters
    cover the finished samples only."""
    if case == "f64":
        view3, nx, ny, it, flags = ("-0.7453", "0.1127", "0.0065"), 40, 24, 4_000, 1
    else:
        view3, nx, ny, it, flags = ("0", "1", "1e-300"), 32, 16, 5_000, 3 | (16 if case == "precision" else 0)
    v, p, plane, t, r = _setup(view3, nx, ny, it)
    table = None
    if flags & 2:
        dc, e = fd.bla_dc_bound(v, p)
        table = fd.Bla.build_scaled(r, fd.route.EPS, dc, e)
    full = emulate(emu, r, plane, t, p, flags, bla=table)
    took = 150  # the clock's first read is the kernel's start: a deadline of 1000 k ns admits k pickups
    got = emulate(emu, r, plane, t, p, flags, bla=table, win=Window(0, 0, 0, 0, 3, 0, None, None, 1000 * took),
                  timed_out=True)
    done = got["status"] != 0
    assert done.sum() == took == got["counters"]["samples"]
    # one lane takes queue slots in order: slot s is lane s % 32 of row-major 8x4 tile s // 32
    slots = np.arange(took)
    tile, lane = slots // 32, slots % 32
    tiles_x = (nx + 7) // 8
    i, j = (tile % tiles_x) * 8 + lane % 8, (tile // tiles_x) * 4 + lane // 8
    assert np.array_equal(np.flatnonzero(done), np.sort(j * nx + i))
    for k in ("cls", "n", "nu", "de", "normal", "z", "dz", "dexp"):
        assert np.array_equal(got[k][done], full[k][done]), k
        assert not got[k][~done].any(), k
    c = got["counters"]
    assert c["iterations"] == int(got["n"][done].astype(np.int64).sum()) - c["skipped"] + c["blocks"]
    # a deadline the frame does not reach changes nothing
    late = emulate(emu, r, plane, t, p, flags, bla=table, win=Window(0, 0, 0, 0, 3, 0, None, None, 1 << 40))
    for k in ("cls", "n", "nu", "z", "status"):
        assert np.array_equal(late[k], full[k]), k
    assert late["counters"] == full["counters"]


@pytest.mark.parametrize("case", ["f64", "scaled-bla"])
def test_route_restarts_only_unfinished_samples(emu, case):
    """The route's deadline contract (frame.rs:338-341 -> grid.rs:175-182): a render the
    deadline cut short raises Incomplete with the finished samples (the kernel's, here on
    the emulated clock) and the mask of the unfinished ones; the caller's CPU render of
    just those samples (the oracle's masked render standing in for fd_kernel's), merged in,
    gives the whole frame and its iteration count. The host encoder's columns of
    unfinished samples are zero, not values computed from unwritten state."""
    if case == "f64":
        view3, nx, ny, it, flags = ("-0.7453", "0.1127", "0.0065"), 40, 24, 4_000, 1
    else:
        view3, nx, ny, it, flags = ("0", "1", "1e-300"), 32, 16, 5_000, 3
    cols = ("nu", "de", "normal")
    v, p, plane, t, r = _setup(view3, nx, ny, it)
    table = None
    if flags & 2:
        dc, e = fd.bla_dc_bound(v, p)
        table = fd.Bla.build_scaled(r, fd.route.EPS, dc, e)
    got = emulate(emu, r, plane, t, p, flags, bla=table, win=Window(0, 0, 0, 0, 3, 0, None, None, 1000 * 200),
                  timed_out=True)
    c = got["counters"]
    cnt = _lib.Counters(samples=c["samples"], iterations=c["iterations"], blocks=c["blocks"], skipped=c["skipped"],
                        fallback_samples=c["fallback_samples"], closed_form_samples=c["closed_form_samples"])
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    ot = fdref.Bla(ref, fd.route.EPS, table.dc_max, table.dc_exp) if table is not None else None
    job = _oracle_job(view3, p, t, fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL)
    whole = fdref.render(job, ref, ot, raw=True)
    for host_encode in (False, True):
        arrays = {k: got[k].copy() for k in ("cls", "n", "z", "dz", "dexp", "status")}
        if not host_encode:
            arrays.update({k: got[k].copy() for k in cols})
        with pytest.raises(fd.Incomplete) as ex:
            fd.route.assemble(v, p, plane, t, table, table, None, flags, True, host_encode, arrays, cnt,
                              _lib.TIMEOUT, len(r), 0.0, fd.RouteReport(), 0.0)
        inc = ex.value
        assert isinstance(inc, fd.Declined)
        assert np.array_equal(inc.mask, got["status"] == 0) and 0 < inc.mask.sum() < nx * ny
        assert inc.stats.iterations == c["iterations"]
        if table is not None:
            assert (inc.bla_stats.blocks, inc.bla_stats.skipped) == (c["blocks"], c["skipped"])
        for k in cols:
            assert not getattr(inc.samples, k)[inc.mask].any(), k
        # the caller's CPU restart of the masked samples only, then the overlay
        part = fdref.render_columns(job, ref, ot, mask=inc.mask.astype(np.uint8))
        cpu = fd.Samples(cls=part["cls"], nu=part["nu"], de=part["de"], normal=part["normal"],
                         n=part["n"].astype(np.uint32), z=part["z"], dz=part["dz"], dexp=part["dexp"])
        merged, st = inc.merge(cpu, fd.Stats(len(r), 0.0, part["stats"]["iterations"]))
        assert np.array_equal(merged.cls, whole["cls"]) and np.array_equal(merged.n, whole["n"].astype(np.uint32))
        esc = whole["cls"] == 0
        assert np.array_equal(merged.z[esc], whole["z"][esc]) and merged.status.all()
        assert np.array_equal(merged.nu[esc], whole["nu"][esc])
        assert st.iterations == whole["stats"]["iterations"]


@pytest.mark.parametrize("view3,it", [(("-0.7436438870371587", "0.1318259042053120", "1e-12"), 20_000),
                                      (("-0.75", "0.1", "0.4"), 2_000)])
def test_bla_kernel_with_a_table_without_levels(emu, view3, it):
    """A table that admits no level (eps 2^-50 at these depths) uploaded as it is, as a
    caller of fdc_upload_bla may: the BLA kernel skips nothing, so every sample equals the
    plain kernel's, and its counters are the reference's for such a table (no block,
    closed-form interiors, every other sample a fallback: grid.rs:767-768)."""
    v, p, plane, t, r = _setup(view3, 48, 32, it)
    dc, e = fd.bla_dc_bound(v, p)
    table = fd.Bla.build_scaled(r, fd.route.EPS, dc, e)
    assert table.levels == 0
    plain = emulate(emu, r, plane, t, p, 1)
    got = emulate(emu, r, plane, t, p, 1 | 2, bla=table)
    for k in ("cls", "n", "z", "dz", "dexp", "nu", "de", "normal", "status"):
        assert np.array_equal(got[k], plain[k]), k
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    want = fdref.render(_oracle_job(view3, p, t, fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL), ref,
                        fdref.Bla(ref, fd.route.EPS, table.dc_max, table.dc_exp))["stats"]
    for k in ("iterations", "blocks", "skipped", "fallback_samples", "closed_form_samples"):
        assert got["counters"][k] == want[k], k


STRIPE_FRAMES = [
    # view, grid, iterations, BLA, tier
    (("-0.7453", "0.1127", "0.0065"), 40, 24, 3000, False, None),
    (("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28"), 40, 24, 30_000, True,
     None),
    (("0", "1", "1e-300"), 32, 24, 5000, True, None),
    (("0", "1", "1e-300"), 32, 24, 5000, True, "scaled"),
]


@pytest.mark.parametrize("frame", STRIPE_FRAMES, ids=lambda f: f"{f[0][2]}-{f[4]}-{f[5]}")
@pytest.mark.parametrize("window,freq,deriv", [(16, 5.0, True), (64, 2.5, False), (3, -7.0, True)])
def test_stripe_kernel_equals_oracle(emu, frame, window, freq, deriv):
    """The stripe variant of the kernel (perturb_kernel<..., T>: every iterate recorded in a
    128-entry ring, the last 8 block starts kept, a plain replay of an incomplete window
    from a kept block start, sample.rs:231-236, 387-403) equals the oracle's Stripe column
    bit for bit on the host (same libm), and its class, count and z are the untraced
    kernel's: on the F64 and Fixed tiers with and without BLA and on the Scaled tier."""
    view3, nx, ny, it, use_bla, tier = frame
    v, p, plane, t, r = _setup(view3, nx, ny, it, tier=tier, columns=("nu", "de") if deriv else ("nu",))
    table = None
    if use_bla:
        dc, e = fd.bla_dc_bound(v, p)
        table = fd.Bla.build_scaled(r, fd.route.EPS, dc, e)
        assert table.levels > 0
    flags = (1 if deriv else 0) | (2 if table is not None else 0)
    plain = emulate(emu, r, plane, t, p, flags, bla=table)
    stripe = np.zeros(nx * ny, np.float32)
    emu.emu_set_stripe(window, freq, stripe.ctypes.data)
    try:
        got = emulate(emu, r, plane, t, p, flags | 32, bla=table)
    finally:
        emu.emu_set_stripe(16, 5.0, None)
    for k in ("cls", "n", "z", "dz", "dexp", "status"):
        assert np.array_equal(got[k], plain[k]), k
    assert got["counters"] == plain["counters"]
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    job = fdref.make_job(*view3, nx, ny, it, columns=fdref.COL_NU | fdref.COL_STRIPE, tier=t, threads=2,
                         stripe_window=window, stripe_freq=freq)
    ot = fdref.Bla(ref, fd.route.EPS, table.dc_max, table.dc_exp) if table is not None else None
    want = fdref.render_columns(job, ref, ot)
    assert np.array_equal(got["cls"], want["cls"])
    esc = want["cls"] == 0
    assert esc.any() and np.array_equal(stripe, want["stripe"]), np.abs(stripe - want["stripe"]).max()


def hypot_pairs(n, seed):
    """Seeded pairs across the whole binary64 range (subnormals, overflowing squares and
    the infinities that ldexp makes at the top): independent exponents, exponents within 70
    of each other, near-equal pairs and pairs near a ratio of 2 (the two correction cases)."""
    g = np.random.default_rng(seed)
    with np.errstate(over="ignore"):
        x = np.ldexp(g.uniform(-1, 1, n), g.integers(-1080, 1031, n))
        kind = g.integers(0, 4, n)
        y = np.ldexp(g.uniform(-1, 1, n), g.integers(-1080, 1031, n))
        close = np.ldexp(g.uniform(-1, 1, n), np.frexp(x)[1] + g.integers(-70, 71, n))
        near = x * (1 + 1e-3 * g.uniform(-1, 1, n))
        half = x * (0.5 + 1e-2 * g.uniform(-1, 1, n))
    return x, np.where(kind == 1, close, np.where(kind == 2, near, np.where(kind == 3, half, y)))


def test_device_hypot_equals_host_libm(emu):
    """The device table builder's hypot (Borges' corrected square root with power-of-two
    scaling) returns the host C library's hypot bit for bit: 4M seeded pairs over the whole
    range and every pair of special values (zeros, subnormals, the largest finite value,
    infinities, NaN, the scaling thresholds)."""
    x, y = hypot_pairs(4_000_000, 5)
    assert emu.emu_hypot_check(x.ctypes.data, y.ctypes.data, len(x)) == 0
    sp = np.array([0.0, -0.0, 1.0, -3.0, 4.0, np.inf, -np.inf, np.nan, 5e-324, 2.2250738585072014e-308,
                   1.7976931348623157e308, 2.0 ** 1023, 2.0 ** -537, 2.0 ** 511, 2.0 ** 500, 2.0 ** -500,
                   2.0 ** -400, np.nextafter(2.0 ** 500, np.inf), np.nextafter(2.0 ** -500, 0.0)])
    a, b = np.meshgrid(sp, sp)
    a, b = np.ascontiguousarray(a.ravel()), np.ascontiguousarray(b.ravel())
    assert emu.emu_hypot_check(a.ctypes.data, b.ctypes.data, len(a)) == 0


TABLE_VIEWS = [
    # view, iterations, tier; the dc bound's exponent ranges from 0 to far below -1022
    # (the first view's orbit escapes early: a table without levels)
    (SEAHORSE + ("1e-14",), 20_000, None),
    (("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-20"), 20_000, None),
    (("0", "1", "1e-300"), 5000, "scaled"),
    (("0", "1", "1e-400"), 5000, "scaled"),
    (("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28"), 50_000, None),
]


@pytest.mark.parametrize("view3,it,tier", TABLE_VIEWS, ids=lambda v: str(v)[:24])
def test_device_table_builder_equals_host_and_oracle(emu, view3, it, tier):
    """fdc_build_bla's level kernel (fdk::bla_level, Block::single / merge, bla.rs:72-112,
    161-216), run on the host, builds the host builder's table and the oracle's: the same
    kept levels and every block's seven fields bit for bit."""
    v, p, plane, t, r = _setup(view3, 64, 36, it, tier=tier)
    dc, e = fd.bla_dc_bound(v, p)
    host = fd.Bla.build_scaled(r, fd.route.EPS, dc, e)
    re, im = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
    out = np.zeros((max(len(re) - 3, 1), 7))
    levels = emu.emu_bla_build(re.ctypes.data, im.ctypes.data, len(re), fd.route.EPS, dc, e, out.ctypes.data)
    assert levels == host.levels and (levels > 0 or view3[2] == "1e-14")
    total = len(host.blocks)
    assert np.array_equal(out[:total].view(np.uint64), np.asarray(host.blocks).reshape(-1, 7).view(np.uint64))
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    blocks, offs = fdref.Bla(ref, fd.route.EPS, dc, e).export()
    assert np.array_equal(out[:total].reshape(-1).view(np.uint64), np.asarray(blocks).reshape(-1).view(np.uint64))


def test_device_table_builder_on_the_nucleus_orbit(emu):
    """The same on configuration 2's orbit (the seeded 1e-100 nucleus, 10^6 points, a
    999,016-block table over 10 levels) against the host builder."""
    from fractodactyl_b200 import locations
    fr = locations.config2()
    r, bits = fd.reference(fr.view, fr.params)
    dc, e = fd.bla_dc_bound(fr.view, fr.params)
    host = fd.Bla.build_scaled(r, fr.bla_eps, dc, e)
    re, im = np.ascontiguousarray(r.re), np.ascontiguousarray(r.im)
    out = np.zeros((len(re) - 3, 7))
    levels = emu.emu_bla_build(re.ctypes.data, im.ctypes.data, len(re), fr.bla_eps, dc, e, out.ctypes.data)
    assert levels == host.levels
    total = len(host.blocks)
    assert total > 900_000
    assert np.array_equal(out[:total].view(np.uint64), np.asarray(host.blocks).reshape(-1, 7).view(np.uint64))
