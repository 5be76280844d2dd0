"""Pins the CPU oracle (oracle/) to the reference's own golden data.

Each test restates a test or fixture of junovhs/fractodactyl; the oracle is trusted as
the CUDA route's parity checker only because these pass.
"""
import json
import math
import os

import numpy as np
import pytest

import fdref
import truthpack

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KATS = json.load(open(os.path.join(GOLDEN, "kats.json")))
EPS_MAX = 2.0 ** -41
EPS_EXACT = 2.0 ** -50


def v0(bits, it, width, i, j):
    """sample.rs:951-963: reference at the v0 centre and the offset of sample (i, j)."""
    r = fdref.Ref.fixed(KATS["v0"]["re"], KATS["v0"]["im"], bits, it)
    h = width / 960.0
    return r, h * (i + 0.5 - 480.0), -h * (j + 0.5 - 270.0)


@pytest.mark.parametrize("case", KATS["fnv_views"], ids=lambda c: c["width"])
def test_precision_tier_render_bytes(case):
    """sample.rs:715-752: FNV-1a of the 8x4 .fds bytes (minor forced to 0)."""
    job = fdref.make_job(case["re"], case["im"], case["width"], 8, 4, 5000, rotation=0.3, threads=1)
    b = bytearray(fdref.render_fds(job))
    b[10:12] = b"\0\0"
    assert fdref.fnv1a64(b) == int(case["fnv"], 16)


def direct(cr, ci, max_iter):
    x = y = 0.0
    for n in range(1, max_iter + 1):
        x, y = x * x - y * y + cr, 2.0 * x * y + ci
        if x * x + y * y > 1e20:
            return n
    return None


@pytest.mark.parametrize("c", [(0.4, 0.3), (-0.75, 0.1), (-1.8, 0.01), (0.2501, 0.0), (-0.1, 0.9),
                               (-0.7487, 0.0789)])
def test_escape_count_matches_direct_iteration(c):
    """sample.rs:771-788."""
    cr, ci = c
    r = fdref.Ref.f64(cr - 1e-3, ci + 1e-3, 100_000, 1e10)
    o = fdref.iterate(r, None, False, True, (cr, ci), 1e-3, -1e-3, 0, 100_000, 1e20)
    assert o["kind"] == "escaped" and o["n"] == direct(cr, ci, 100_000)


@pytest.mark.parametrize("c", [(-1.7548, 0.0), (-0.1565, 1.0322), (-1.3107, 0.0)])
def test_interior_outside_main_components(c):
    """sample.rs:790-799."""
    cr, ci = c
    r = fdref.Ref.f64(cr - 1e-3, ci + 1e-3, 1_000_000, 1e10)
    assert fdref.iterate(r, None, False, True, c, 1e-3, -1e-3, 0, 1_000_000, 1e20)["kind"] == "interior"


def test_bla_blocks_keep_the_escape_count():
    """sample.rs:897-940."""
    r = fdref.Ref.f64(0.2501, 0.0, 100_000, 1e10)
    bla = fdref.Bla(r, EPS_MAX, 2e-17)
    for ar, ai in [(1e-17, 0.0), (-1e-17, 1e-17), (0.0, -1.4e-17)]:
        plain = fdref.iterate(r, None, False, True, None, ar, ai, 0, 100_000, 1e20)
        fast = fdref.iterate(r, bla, False, True, None, ar, ai, 0, 100_000, 1e20)
        assert plain["kind"] == fast["kind"] == "escaped" and plain["n"] == fast["n"]
        assert abs(plain["zr"] - fast["zr"]) < 1e-6 * abs(plain["zr"])
        assert abs(plain["dr"] - fast["dr"]) < 1e-6 * abs(plain["dr"])
        assert fast["skipped"] > 10 * fast["blocks"] > 0


def test_near_return_that_expands_is_not_interior():
    """sample.rs:965-976 (FIX-02): mpmath escape at n = 788."""
    r, ar, ai = v0(218, 2000, 8.29151e-25, 287, 212)
    o = fdref.iterate(r, None, False, True, None, ar, ai, 0, 2000, 1e20)
    assert o["kind"] == "escaped" and o["n"] == 788


def test_bla_judges_periodicity_at_the_plain_save_points():
    """sample.rs:978-1039: period-3 nucleus agreement and the v0 frame-749 escape at 7412."""
    cr, ci = -1.7548776662466927, 0.0
    r = fdref.Ref.f64(cr, ci, 100_000, 1e10)
    for e in (1e-16, 1e-18):
        bla = fdref.Bla(r, EPS_EXACT, 2.0 * e)
        for k in range(8):
            a = math.pi / 4 * k
            ar, ai = e * math.cos(a), e * math.sin(a)
            plain = fdref.iterate(r, None, False, True, (cr + ar, ci + ai), ar, ai, 0, 100_000, 1e20)
            fast = fdref.iterate(r, bla, False, True, (cr + ar, ci + ai), ar, ai, 0, 100_000, 1e20)
            assert (plain["kind"], plain["n"]) == (fast["kind"], fast["n"]) and plain["kind"] == "interior"
            assert fast["skipped"] > 0
    r, ar, ai = v0(300, 20_000, 2e-49, 324, 10)
    bla = fdref.Bla(r, EPS_EXACT, 2e-49 * 1.15)
    o = fdref.iterate(r, bla, False, True, None, ar, ai, 0, 20_000, 1e20)
    assert o["kind"] == "escaped" and o["n"] == 7412 and o["skipped"] > 4096


def test_scaled_agrees_with_f64_where_both_apply():
    """sample.rs:1166-1201."""
    r = fdref.Ref.f64(-0.7487, 0.0789, 10_000, 1e10)
    for ar, ai in [(1e-5, 2e-5), (-3e-5, 1e-5), (5e-5, -5e-5)]:
        k = 1048576.0
        a = fdref.iterate(r, None, True, True, None, ar * k, ai * k, -20, 10_000, 1e20)
        b = fdref.iterate(r, None, False, True, None, ar, ai, 0, 10_000, 1e20)
        assert a["kind"] == b["kind"] == "escaped" and a["n"] == b["n"]
        assert abs(a["zr"] - b["zr"]) < 1e-6 * abs(b["zr"])
        m1 = math.hypot(a["dr"], a["di"]) * 2.0 ** a["dexp"]
        m2 = math.hypot(b["dr"], b["di"])
        assert abs(m1 - m2) < 1e-6 * m2


def test_escapes_from_far_below_f64_range():
    """sample.rs:1204-1215."""
    r = fdref.Ref.f64(0.0, 1.0, 100_000, 1e10)
    o = fdref.iterate(r, None, True, True, None, 1.0, 0.5, -3000, 100_000, 1e20)
    assert o["kind"] == "escaped" and 1500 < o["n"] < 4000 and o["dexp"] > 2900


@pytest.mark.parametrize("cr,ci,n", [(0.0, 1.0, 887), (0.250001, 0.0, 3145), (-0.75, 0.01, 320)])
def test_deep_repelling_and_near_parabolic_exteriors(cr, ci, n):
    """sample.rs:1218-1229 (mpmath counts at 1200 bits)."""
    r = fdref.Ref.f64(cr, ci, 20_000, 65536.0)
    o = fdref.iterate(r, None, True, True, None, 1.0, 0.5, -1100, 20_000, 1e20)
    assert o["kind"] == "escaped" and o["n"] == n


@pytest.mark.slow
def test_deep_nucleus_neighbours_escape_at_oracle_counts():
    """sample.rs:1258-1340 (FIX-40, FIX-41): the k = 7676 rung, mpmath at 1200 digits."""
    rung = KATS["rung_7676"]
    r = fdref.Ref.fixed(rung["re"], rung["im"], 3456, 150_000)
    o = fdref.iterate(r, None, True, True, None, -0.5737130423454617, 0.290231303774763, -3310, 140_000, 1e20)
    assert o["kind"] == "escaped" and o["n"] == 133_115
    assert abs(o["zr"] / -27519423631.080235 - 1.0) < 1e-6
    assert abs(math.log2(math.hypot(o["dr"], o["di"])) + o["dexp"] - 3359.4391791173814) < 1e-6
    o = fdref.iterate(r, None, True, True, None, 0.006749565204064256, 0.10124347806096384, -3310, 140_000, 1e20)
    assert o["kind"] == "escaped" and o["n"] == 139_850
    job = fdref.make_job(rung["re"], rung["im"], "5.050000000000E-998", 480, 270, 644_640)
    p = fdref.plane(job)
    ux, uy = 184 + 0.5 - 240.0, -(201 + 0.5 - 135.0)
    o = fdref.iterate(r, None, True, True, None, ux * p["h_m"], uy * p["h_m"], p["h_e"], 644_640, 1e20)
    assert o["kind"] == "escaped" and o["n"] == 145_079


def test_bla_find_equals_brute_force():
    """bla.rs:317-350: radii shrink upward; find takes the longest valid block."""
    r = fdref.Ref.f64(-0.743643887037158, 0.131825904205312, 20_000, 1e10)
    t = fdref.Bla(r, EPS_EXACT, 1e-25)
    blocks, offs = t.export()
    levels = [blocks[offs[i]:offs[i + 1]] for i in range(t.levels)]
    assert t.levels > 5
    for i in range(1, len(levels)):
        assert np.all(levels[i][:, 4] <= levels[i - 1][0::2][: len(levels[i]), 4])
    for m in range(0, len(r), 3):
        for d2, budget in [(1e-40, 2**64 - 1), (1e-31, 2**64 - 1), (1e-34, 5), (1e-36, 2), (1e-40, 1)]:
            k = (m - 1) % 2**64
            want = None
            for i in range(len(levels)):
                if not (m > 0 and k % (2 << i) == 0 and (2 << i) <= budget):
                    break
                at = k >> (i + 1)
                if at >= len(levels[i]) or not d2 < levels[i][at, 4] ** 2:
                    break
                want = (i, at, 2 << i)
            assert t.find(m, d2, budget) == want


def test_bla_refusals():
    """bla.rs:352-374."""
    r = fdref.Ref.f64(-0.7453, 0.1127, 2000, 1e10)
    with pytest.raises(ValueError):
        fdref.Bla(r, 2.0 * 2.0 ** -24, 1e-20)
    with pytest.raises(ValueError):
        fdref.Bla(r, 0.0, 1.0)
    t = fdref.Bla(r, EPS_MAX, 1e-20)
    assert t.find(1, 1e-40, 2**64 - 1)[2] > 2
    assert t.find(0, 1e-40, 2**64 - 1) is None and t.find(2, 1e-40, 2**64 - 1) is None
    assert t.find(1, 1e-40, 1) is None and t.find(1, 1e-40, 3)[2] == 2 and t.find(1, 1.0, 2**64 - 1) is None


@pytest.mark.parametrize("width,tier", [("1e-3", 0), ("1e-15", 1), ("1e-260", 1), ("1e-300", 2), ("1e-100000", 2)])
def test_tiers_follow_depth(width, tier):
    """view.rs:167-175."""
    assert fdref.plane(fdref.make_job("-0.5", "0.25", width, 1000, 1000, 100))["tier"] == tier


@pytest.mark.parametrize("name", truthpack.CASES)
def test_truth_pack(name):
    """bench/truth/v1 through examples/truth-pack.rs: plain and BLA (eps 2^-41) routes,
    only the two recorded filament precision edges may mismatch (auto tier), none on the
    Fixed-tier recheck; no scalar failures."""
    edges = truthpack.load_edges()
    case = truthpack.load(name)
    expect = len([e for e in edges if e["case"] == name])
    for tier in ([None, "fx"] if expect else [None]):
        job = fdref.make_job(case["re"], case["im"], case["width"], case["nx"], case["ny"], case["max_iter"],
                             rotation=case["rotation"], escape_radius=case["escape_radius"], tier=tier)
        ref = fdref.Ref.for_job(job)
        dc, e = fdref.bla_dc_bound(job)
        bla = fdref.Bla(ref, EPS_MAX, dc, e)
        for out in (fdref.render(job, ref), fdref.render(job, ref, bla)):
            s = truthpack.compare(case, out["cls"], out["nu"], out["de"], out["normal"], edges, tier is None)
            assert s["scalar_failures"] == 0, s
            assert s["class_mismatches"] == s["known_edges"] == (expect if tier is None else 0), s


def test_kern05_bundle_frames():
    """crates/fd-kernel/fixtures/KERN-05.bundle (minor 0, captured on Windows before later
    kernel fixes): 8 frames byte-identical; the rest drift only by the documented amounts
    (2 seahorse samples Interior -> Unresolved after PERF-08; 1-ulp nu from MSVC's log2)."""
    d = json.load(open(os.path.join(GOLDEN, "kern05.json")))
    exact = 0
    for loc, fr in zip(d["locations"], d["frames"]):
        if loc["name"] == "rung-7676":
            continue  # covered by the slow rung test; 7 s of orbit setup
        job = fdref.make_job(loc["re"], loc["im"], loc["width"], loc["nx"], loc["ny"], loc["iter"],
                             rotation=loc["rotation"], tier=loc["tier"])
        b = bytearray(fdref.render_fds(job))
        b[10:12] = b"\0\0"
        assert len(b) == fr["bytes"] and "pert" in fr["kernel"]
        if "0x%016x" % fdref.fnv1a64(b) == fr["fnv_minor0"]:
            exact += 1
            continue
        n = loc["nx"] * loc["ny"]
        cls = np.frombuffer(bytes(b), np.uint8, n, fr["header_bytes"])
        counts = [int((cls == k).sum()) for k in range(3)]
        assert counts[0] == fr["classes"][0]
        assert abs(counts[1] - fr["classes"][1]) <= 2 and counts[1] + counts[2] == sum(fr["classes"][1:])
    assert exact >= 7


def test_fixed_orbit_reaches_the_mpmath_nucleus_return():
    """crates/fd-fixed/tests/fixtures/v0_orbit.txt (mpmath at 400 digits): from c given to
    78 digits, z_764 of the period-764 nucleus orbit. The fixed-point orbit at 1,400 bits
    (orbit.rs:14-43, the f64 rounding of lib.rs:75-83) lands within one ulp of it on both
    parts, although |z_764| ~ 6e-54 (a relative error of the fixed point's 2^-1400 grown
    by |dz/dc| ~ 2^83 leaves ~1,000 bits to spare), and the nucleus gate finds the period."""
    f = KATS["v0_orbit"]
    period = int(f["period"])
    r = fdref.Ref.fixed(f["c"][0], f["c"][1], 1400, 2 * period + 10)  # the gate reads z_2p (reference.rs:102-120)
    re_, im_ = r.arrays_()
    want = np.array([float(f["z"][0]), float(f["z"][1])])
    got = np.array([re_[period], im_[period]])
    assert np.all(np.abs(got - want) <= np.spacing(np.abs(want))), (got, want)
    assert abs(want[0]) < 1e-53 and abs(want[1]) < 1e-53
    assert r.nucleus_period() == period


MPMATH = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mpmath_checks.json")))


@pytest.mark.parametrize("rec", MPMATH, ids=lambda r: r["name"])
def test_renders_the_mpmath_checker_passed(rec):
    """tests/golden/make_mpmath_checks.py ran the reference's independent mpmath checker
    (tools/oracle.py: direct iteration at depth + 128 bits; class exact, nu / de / normal
    within 1e-3 output pixels) on the oracle's .fds renders of these views (three tiers, BLA
    on and off, rotation, interior samples in and outside the main components); it passed
    every sampled point. The oracle still writes those exact bytes."""
    assert rec["exit"] == 0 and rec["checker"]["ok"] and rec["checker"]["class_mismatch"] == 0
    job = fdref.make_job(rec["re"], rec["im"], rec["width"], rec["nx"], rec["ny"], rec["max_iter"],
                         rotation=rec["rotation"], columns=fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL, threads=2)
    ref = bla = None
    if rec["bla_eps"] is not None:
        ref = fdref.Ref.for_job(job)
        dc, e = fdref.bla_dc_bound(job)
        bla = fdref.Bla(ref, rec["bla_eps"], dc, e)
    data = fdref.render_fds(job, ref, bla)
    assert "0x%016x" % fdref.fnv1a64(data) == rec["fnv"]


def test_mpmath_checks_cover_every_class_and_tier():
    kernels = {r["checker"]["kernel"].split()[0] for r in MPMATH}
    assert kernels == {"pert-f64/1", "pert-fx/1", "pert-fx-scaled/1"}
    assert any("bla/1" in r["checker"]["kernel"] for r in MPMATH)
    assert sum(r["checker"]["samples"] - r["checker"]["escaped"] for r in MPMATH) > 30  # bounded samples
