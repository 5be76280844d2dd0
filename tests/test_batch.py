"""Batches (fdc_batch_create / fdc_batch_run): jobs of different depths, tiers, flags and
forms rendered by one graph replay equal the same jobs rendered one by one with
fdc_render, bit for bit, on every replay, and so do the per-job counters."""
import numpy as np
import pytest

import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

pytestmark = pytest.mark.gpu

FRAMES = [
    # (re, im, width, nx, ny, max_iter, columns, bla, f32)
    ("0", "1", "1e-300", 96, 64, 5_000, ("nu", "de", "normal"), True, False),
    ("-0.7453", "0.1127", "0.0065", 128, 72, 4_000, ("nu",), False, False),
    ("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28", 80, 48, 20_000,
     ("nu", "de", "normal"), False, False),
    ("-0.7453", "0.1127", "0.0065", 64, 40, 4_000, ("nu", "de"), True, False),
    ("0", "1", "1e-300", 96, 64, 5_000, ("nu", "de", "normal"), True, True),
]


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def _job(dev, frame):
    re_, im_, w, nx, ny, it, cols, use_bla, f32 = frame
    v = fd.View(re_, im_, w)
    p = fd.Params(nx, ny, max_iter=it, columns=cols)
    plane, tier = fd.route._setup(v, p)
    r, bits = fd.reference(v, p)
    r.bits = bits
    bla = None
    if use_bla:
        dc, e = fd.bla_dc_bound(v, p)
        bla = fd.Bla.build_scaled(r, fd.route.EPS, dc, e)
    if bla is not None and bla.levels == 0:
        bla = None
    h = dev.upload(r, bla)
    flags = (_lib.DERIVATIVE if p.needs_derivative() else 0) | (_lib.BLA if bla is not None else 0) | \
        (_lib.F32 if f32 else 0)
    return h, fd.route.make_job(plane, tier, p, h, r.nucleus_period(), flags)


def test_batch_equals_single_renders(dev):
    handles, jobs = zip(*[_job(dev, f) for f in FRAMES])
    # plus a window (rows 4..33, columns 16..95) of the second frame
    hw, jw = _job(dev, FRAMES[1])
    jw.first_row, jw.rows, jw.first_col, jw.cols = 4, 30, 16, 80
    handles, jobs = handles + (hw,), jobs + (jw,)
    singles = [dev.render_job(j, raw=True, columns=("nu", "de", "normal")) for j in jobs]
    b = dev.batch(jobs, columns=("nu", "de", "normal"), raw=True)
    try:
        for replay in range(2):
            total, per = b.run()
            assert total.launches >= 2
            for k, (arrays, cnt, _) in enumerate(singles):
                got = b.columns(k)
                assert np.array_equal(got["status"], arrays["status"]), (replay, k)
                assert got["status"].sum() == cnt.samples, (replay, k)
                for name in ("cls", "n", "z", "dz", "dexp"):
                    assert np.array_equal(got[name], arrays[name]), (replay, k, name)
                for name in ("nu", "de", "normal"):
                    if k < len(FRAMES) and name in FRAMES[k][6]:
                        assert np.array_equal(got[name], arrays[name]), (replay, k, name)
                assert per[k].samples == cnt.samples and per[k].iterations == cnt.iterations, (replay, k)
                assert per[k].blocks == cnt.blocks and per[k].skipped == cnt.skipped, (replay, k)
            assert total.samples == sum(c.samples for _, c, _ in singles)
    finally:
        b.free()
        for h in set(handles):
            dev.free(h)


def test_batch_refuses_host_only_jobs(dev):
    h, j = _job(dev, FRAMES[1])
    try:
        j.mask = np.ones(j.nx * j.ny, np.uint8).ctypes.data
        with pytest.raises(fd.route.RouteError, match="mask"):
            dev.batch([j])
    finally:
        dev.free(h)


def test_orbit_held_while_a_batch_reads_it(dev):
    """A live batch holds its jobs' orbits: freeing one is refused (the batch would read
    recycled device memory) until the batch is freed."""
    h, j = _job(dev, FRAMES[1])
    b = dev.batch([j], columns=("nu",))
    try:
        with pytest.raises(fd.route.RouteError, match="live batch"):
            dev.free(h)
        total, _ = b.run()
        assert total.samples == j.nx * j.ny
    finally:
        b.free()
    dev.free(h)
    with pytest.raises(fd.route.RouteError, match="unknown orbit"):
        dev.free(h)
