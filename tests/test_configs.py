"""Configurations 3-5 at reduced sizes against the oracle: the jittered 4-sample frame at
1e-300 (per-sample offsets), a film sharing one orbit across widths from 1e-10 to 1e-500
with a BLA table per frame (one batch), and tiles of mixed locations each with its own orbit and
table (column and row windows in one batch). The plain form's class, count and z at
escape equal the oracle's bit for bit; the precision form's agreement is reported."""
import dataclasses

import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib, locations, workloads

pytestmark = pytest.mark.gpu
KIND = {"escaped": 0, "interior": 1, "unresolved": 2}


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def oracle_tables(r, bla, eps):
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    t = fdref.Bla(ref, eps, bla.dc_max, bla.dc_exp) if bla is not None else None
    return ref, t


def check_frame(got, want, sel=None):
    sel = np.ones(len(want["cls"]), bool) if sel is None else sel
    assert np.array_equal(got["cls"][sel], want["cls"][sel])
    assert np.array_equal(got["n"][sel], want["n"][sel].astype(np.uint32))
    esc = sel & (want["cls"] == 0)
    assert np.array_equal(got["z"][esc], want["z"][esc])


def test_jittered_frame_at_1e300(dev):
    fr = locations.config3(nx=24, ny=16)  # 48x32 samples, 2x2 per pixel, jittered
    js = workloads.jittered(dev, fr)
    try:
        j = js.jobs[0]
        a, cnt, _ = dev.render_job(j, raw=True)
        j.flags |= _lib.F32
        b, _, _ = dev.render_job(j, raw=True)
    finally:
        js.free(dev)
    plane, r, bla = js.planes[0], js.refs[0], js.blas[0]
    ref, t = oracle_tables(r, bla, fr.bla_eps)
    offs = js.keep[0]
    p = fr.params
    r2 = p.escape_radius ** 2
    for k in range(p.nx * p.ny):
        o = fdref.iterate(ref, t, extended=True, derivative=True, ar=offs[k, 0] * plane.h_m,
                          ai=offs[k, 1] * plane.h_m, offset_exp=plane.h_e, max_iter=p.max_iter, r2=r2)
        kind = KIND[o["kind"]]
        assert a["cls"][k] == kind, k
        assert a["n"][k] == (p.max_iter if kind == 2 else o["n"]), k
        if kind == 0:
            assert (a["z"][k, 0], a["z"][k, 1]) == (o["zr"], o["zi"]), k
    ea, eb = a["cls"] == 0, b["cls"] == 0
    same = ((ea == eb) & (~ea | (a["n"] == b["n"]))).mean()
    print(f"jittered 1e-300: {ea.mean():.3f} escaped, precision form counts equal on {same:.4f}, "
          f"escape agreement {(ea == eb).mean():.4f}")
    assert (ea == eb).mean() >= 0.99


def _shrink(frames, nx, ny, max_iter=None):
    out = []
    for f in frames:
        p = dataclasses.replace(f.params, nx=nx, ny=ny, max_iter=max_iter or f.params.max_iter)
        out.append(dataclasses.replace(f, params=p))
    return out


def test_film_shares_one_orbit(dev):
    film = locations.config4()
    frames = _shrink([film[k] for k in (0, 15, 30, 45, 59)], 48, 27)
    js = workloads.film(dev, frames)
    try:
        b = dev.batch(js.jobs, columns=("nu",), raw=True)
        try:
            b.run()
            got = [b.columns(k) for k in range(len(js.jobs))]
        finally:
            b.free()
    finally:
        js.free(dev)
    assert len({pl.tier for pl in js.planes}) >= 2 and js.tiers[0] == 1 and js.tiers[-1] == 2
    assert js.blas[-1] is not None and js.blas[-1].levels > 10  # the deepest frame's table skips
    for f, tier, g, bla in zip(frames, js.tiers, got, js.blas):
        ref, t = oracle_tables(js.refs[0], bla, f.bla_eps)
        v, p = f.view, f.params
        job = fdref.make_job(v.center_re, v.center_im, v.width, p.nx, p.ny, p.max_iter,
                             escape_radius=p.escape_radius, columns=fdref.COL_NU, tier=tier)
        want = fdref.render(job, ref, t, raw=True)
        check_frame(g, want)


def test_mixed_location_tiles(dev):
    c5 = locations.config5()
    # the shallowest, a middle and the deepest location; 64x32 frames cut into 32x32 tiles
    pick = sorted(range(len(c5)), key=lambda k: -float(c5[k].view.width.split("e")[1]))
    frames = _shrink([c5[pick[0]], c5[pick[len(pick) // 2]], c5[pick[-1]]], 64, 32, max_iter=200_000)
    js = workloads.tiles(dev, frames, (32, 32))
    assert len(js.jobs) == 6
    try:
        b = dev.batch(js.jobs, columns=("nu",), raw=True)
        try:
            total, per = b.run()
            got = [b.columns(k) for k in range(len(js.jobs))]
        finally:
            b.free()
        # the tiles of a location sharing its frame (groups): each frame once, every
        # tile's window filled, the same samples and counters
        g = dev.batch(js.jobs, columns=("nu",), raw=True, groups=js.groups)
        try:
            total_g, per_g = g.run()
            shared, host = g.all_columns()
        finally:
            g.free()
    finally:
        js.free(dev)
    assert len(host["cls"]) == len(frames) * 64 * 32
    assert host["status"].all()
    assert total_g.iterations == total.iterations and [c.samples for c in per_g] == [c.samples for c in per]
    for k in range(len(js.jobs)):
        on = got[k]["status"].astype(bool)
        for name in ("cls", "n", "z", "dz", "dexp", "nu"):
            assert np.array_equal(shared[k][name][on], got[k][name][on]), (k, name)
    for loc, f in enumerate(frames):
        r, bla, tier = js.refs[loc], js.blas[loc], js.tiers[2 * loc]
        ref, t = oracle_tables(r, bla, f.bla_eps)
        v, p = f.view, f.params
        job = fdref.make_job(v.center_re, v.center_im, v.width, p.nx, p.ny, p.max_iter,
                             escape_radius=p.escape_radius, columns=fdref.COL_NU, tier=tier)
        want = fdref.render(job, ref, t, raw=True)
        for k in (2 * loc, 2 * loc + 1):
            x0, cw, y0, rh = js.windows[k]
            win = np.zeros((p.ny, p.nx), bool)
            win[y0:y0 + rh, x0:x0 + cw] = True
            win = win.ravel()
            assert np.array_equal(got[k]["status"].astype(bool), win)
            check_frame(got[k], want, win)
            assert per[k].samples == win.sum()
