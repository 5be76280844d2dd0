"""The benchmark configurations at their full size against the oracle (the reference's
CPU algorithm restated), through the CUDA route's plain form.

- Configuration 1 (480x270, 1e-12, 20,000 iterations, bailout 2^8, no BLA) and
  configuration 2 (1920x1080 at the seeded 1e-100 nucleus, 10^6 iterations, BLA from the
  CPU builder, floatexp deltas): every sample of the frame. Class, escape count, z and
  dz/dc (mantissa and exponent) bit-exact, the work counters equal, nu within 1e-12
  relative.
- Configurations 3-5 at full configuration (full grid, full max_iter, each real location's
  orbit and BLA table): a seeded subset of at least 4,096 samples each, rendered through
  a sample mask of the full job and compared with the oracle sample by sample (per-sample
  iteration at the jittered offsets for configuration 3; the oracle's masked render of
  the same frame for the film frames and the mixed locations). Class, escape count and z
  bit-exact.
"""
import ctypes as C
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib, locations, workloads

pytestmark = pytest.mark.gpu
KIND = {"escaped": 0, "interior": 1, "unresolved": 2}
NU_REL = 1e-12


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def oracle_tables(r, bla, eps):
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    return ref, (fdref.Bla(ref, eps, bla.dc_max, bla.dc_exp) if bla is not None else None)


def check_exact(got, want, sel, what):
    assert np.array_equal(got["cls"][sel], want["cls"][sel]), what
    assert np.array_equal(got["n"][sel], want["n"][sel].astype(np.uint32)), what
    esc = sel & (want["cls"] == 0)
    assert np.array_equal(got["z"][esc].view(np.uint64), want["z"][esc].view(np.uint64)), what
    return int(esc.sum())


@pytest.mark.parametrize("config", [1, 2])
def test_whole_frame_equals_the_oracle(dev, config):
    fr = locations.config1() if config == 1 else locations.config2()
    view, p = fr.view, fr.params
    plane, tier = fd.route._setup(view, p)
    r, bits = fd.reference(view, p)
    r.bits = bits
    bla = None
    if fr.bla_eps is not None:
        dc, e = fd.bla_dc_bound(view, p)
        bla = fd.Bla.build_scaled(r, fr.bla_eps, dc, e)
    h = dev.upload(r, bla)
    try:
        flags = (_lib.DERIVATIVE if p.needs_derivative() else 0) | (_lib.BLA if bla is not None else 0)
        got, cnt, _ = dev.render_job(fd.route.make_job(plane, tier, p, h, r.nucleus_period(), flags), raw=True,
                                     columns=p.columns)
    finally:
        dev.free(h)
    cols = fdref.COL_NU * ("nu" in p.columns) | fdref.COL_DE * ("de" in p.columns) | \
        fdref.COL_NORMAL * ("normal" in p.columns)
    job = fdref.make_job(view.center_re, view.center_im, view.width, p.nx, p.ny, p.max_iter,
                         escape_radius=p.escape_radius, columns=cols, tier=tier)
    ref, t = oracle_tables(r, bla, fr.bla_eps)
    want = fdref.render(job, ref, t, raw=True)
    everything = np.ones(p.nx * p.ny, bool)
    esc = check_exact(got, want, everything, fr.name)
    e = want["cls"] == 0
    assert np.array_equal(got["dz"][e].view(np.uint64), want["dz"][e].view(np.uint64))
    assert np.array_equal(got["dexp"][e], want["dexp"][e])
    rel = np.abs(got["nu"][e] - want["nu"][e]) / np.abs(want["nu"][e])
    assert rel.max() <= NU_REL, rel.max()
    st = want["stats"]
    assert (cnt.samples, cnt.iterations) == (p.nx * p.ny, st["iterations"])
    if bla is not None:
        assert (cnt.blocks, cnt.skipped, cnt.fallback_samples, cnt.closed_form_samples) == (
            st["blocks"], st["skipped"], st["fallback_samples"], st["closed_form_samples"])
        assert cnt.blocks > 0 and cnt.skipped > 10 * cnt.blocks
    print(f"{fr.name}: {p.nx * p.ny} samples equal ({esc} escaped), {cnt.iterations} iterations")


def seeded_mask(n, k, seed):
    m = np.zeros(n, np.uint8)
    m[np.random.default_rng(seed).choice(n, min(k, n), replace=False)] = 1
    return m


def test_config3_jittered_subset(dev):
    """The full 3840x2160 x 4-sample jittered frame at 1e-300 (5*10^6 iterations, BLA and
    derivative on): 4,096 seeded samples through the job's mask, each against the oracle's
    iteration at its own jittered offset."""
    fr = locations.config3()
    js = workloads.jittered(dev, fr)
    p = fr.params
    n = p.nx * p.ny
    mask = seeded_mask(n, 4096, 31)
    try:
        j = js.jobs[0]
        j.mask = mask.ctypes.data
        got, cnt, _ = dev.render_job(j, raw=True, columns=("nu",))
    finally:
        js.free(dev)
    sel = mask.astype(bool)
    assert cnt.samples == sel.sum() and np.all(got["status"][sel] == 1) and not got["status"][~sel].any()
    plane, r, bla = js.planes[0], js.refs[0], js.blas[0]
    ref, t = oracle_tables(r, bla, fr.bla_eps)
    offs = js.keep[0]
    r2 = p.escape_radius ** 2
    idx = np.flatnonzero(sel)

    def one(k):
        return fdref.iterate(ref, t, extended=True, derivative=True, ar=offs[k, 0] * plane.h_m,
                             ai=offs[k, 1] * plane.h_m, offset_exp=plane.h_e, max_iter=p.max_iter, r2=r2)

    with ThreadPoolExecutor() as ex:
        outs = list(ex.map(one, idx))
    for k, o in zip(idx, outs):
        kind = KIND[o["kind"]]
        assert got["cls"][k] == kind, k
        assert got["n"][k] == (p.max_iter if kind == 2 else o["n"]), k
        if kind == 0:
            assert (got["z"][k, 0], got["z"][k, 1]) == (o["zr"], o["zi"]), k
    print(f"config 3: {len(idx)} samples equal, {sum(o['kind'] == 'escaped' for o in outs)} escaped")


def test_config4_film_subset(dev):
    """All 60 film frames (1280x720, widths 1e-10..1e-500, 10^7 iterations) over the one
    shared 1,800-bit orbit with per-frame tables: 70 seeded samples per frame (4,200) through
    each frame's mask against the oracle's masked render of that frame."""
    frames = locations.config4()
    js = workloads.film(dev, frames)
    total = 0
    try:
        ref = fdref.Ref.arrays(js.refs[0].re, js.refs[0].im, js.refs[0].bits)
        for k, (f, j, tier, bla) in enumerate(zip(frames, js.jobs, js.tiers, js.blas)):
            p = f.params
            mask = seeded_mask(p.nx * p.ny, 70, 400 + k)
            j.mask = mask.ctypes.data
            got, cnt, _ = dev.render_job(j, raw=True, columns=("nu",))
            t = fdref.Bla(ref, f.bla_eps, bla.dc_max, bla.dc_exp) if bla is not None else None
            job = fdref.make_job(f.view.center_re, f.view.center_im, f.view.width, p.nx, p.ny, p.max_iter,
                                 escape_radius=p.escape_radius, columns=fdref.COL_NU, tier=tier)
            want = fdref.render_columns(job, ref, t, mask=mask)
            sel = mask.astype(bool)
            check_exact(got, want, sel, f.name)
            assert cnt.samples == sel.sum()
            total += int(sel.sum())
    finally:
        js.free(dev)
    assert total >= 4096
    print(f"config 4: {total} samples over {len(frames)} frames equal")


def test_config5_mixed_locations_subset(dev):
    """All 32 seeded locations of the mixed-location set (1024x512 frames, widths
    1e-20..1e-1000, 10^7 iterations), each with its own orbit and table: 128 seeded samples
    per location (4,096) through a mask over that location's whole frame against the
    oracle's masked render."""
    frames = locations.config5()
    js = workloads.tiles(dev, frames, (256, 256))
    total = 0
    try:
        for loc, f in enumerate(frames):
            k0 = js.groups.index(loc)  # the location's first tile job: its orbit and table
            j = _lib.Job()
            C.memmove(C.byref(j), C.byref(js.jobs[k0]), C.sizeof(_lib.Job))
            j.first_col = j.cols = j.first_row = j.rows = 0
            p = f.params
            mask = seeded_mask(p.nx * p.ny, 128, 500 + loc)
            j.mask = mask.ctypes.data
            got, cnt, _ = dev.render_job(j, raw=True, columns=("nu",))
            r, bla, tier = js.refs[loc], js.blas[loc], js.tiers[k0]
            ref, t = oracle_tables(r, bla, f.bla_eps)
            job = fdref.make_job(f.view.center_re, f.view.center_im, f.view.width, p.nx, p.ny, p.max_iter,
                                 escape_radius=p.escape_radius, columns=fdref.COL_NU, tier=tier)
            want = fdref.render_columns(job, ref, t, mask=mask)
            sel = mask.astype(bool)
            check_exact(got, want, sel, f.name)
            assert cnt.samples == sel.sum()
            total += int(sel.sum())
    finally:
        js.free(dev)
    assert total >= 4096
    print(f"config 5: {total} samples over {len(frames)} locations equal")
