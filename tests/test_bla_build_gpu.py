"""BLA tables built on the device (fdc_build_bla: Bla::build_scaled, bla.rs:161-216, over
the uploaded orbit) against the host builder, whose tables equal the oracle's:

- the kept levels and every block's seven fields bit for bit, on views whose dc bound's
  exponent runs from 0 to far below -1022, a view whose table has no level, and
  configuration 2's 10^6-point nucleus orbit (999,016 blocks);
- frames rendered with the device-built table equal the same frames rendered with the
  uploaded host table: every raw column, the iteration count and the BLA counters;
- the upload's refusals (eps, dc_max, unknown orbit) hold for the build.
"""
import dataclasses
import math
import time

import numpy as np
import pytest

import fractodactyl_b200 as fd
from fractodactyl_b200 import locations

pytestmark = pytest.mark.gpu

SPIRAL = ("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139")
VIEWS = [
    # view, iterations, tier (the first view's orbit escapes early: no level is kept)
    (("-0.743643887037158", "0.131825904205312", "1e-14"), 20_000, None),
    (SPIRAL + ("1e-20",), 20_000, None),
    (SPIRAL + ("1e-28",), 50_000, None),
    (("0", "1", "1e-300"), 5000, "scaled"),
    (("0", "1", "1e-400"), 5000, "scaled"),
]


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def built(dev, r, eps, dc, e):
    h = dev.upload(r)
    try:
        return dev.build_bla(h, eps, dc, e, export=True)
    finally:
        dev.free(h)


def same_bits(a, b):
    return np.array_equal(np.asarray(a).reshape(-1).view(np.uint64), np.asarray(b).reshape(-1).view(np.uint64))


@pytest.mark.parametrize("view3,it,tier", VIEWS, ids=lambda v: str(v)[:24])
def test_device_table_equals_host_table(dev, view3, it, tier):
    v, p = fd.View(*view3), fd.Params(64, 36, max_iter=it, tier=tier)
    r, _ = fd.reference(v, p)
    dc, e = fd.bla_dc_bound(v, p)
    host = fd.Bla.build_scaled(r, fd.EPS, dc, e)
    levels, blocks = built(dev, r, fd.EPS, dc, e)
    assert levels == host.levels
    assert len(blocks) == len(host.blocks) and same_bits(blocks, host.blocks)


def test_device_table_on_the_nucleus_orbit(dev):
    fr = locations.config2()
    r, _ = fd.reference(fr.view, fr.params)
    dc, e = fd.bla_dc_bound(fr.view, fr.params)
    host = fd.Bla.build_scaled(r, fr.bla_eps, dc, e)
    t = time.perf_counter()
    levels, blocks = built(dev, r, fr.bla_eps, dc, e)
    ms = (time.perf_counter() - t) * 1e3
    assert levels == host.levels and len(blocks) == len(host.blocks) > 900_000
    assert same_bits(blocks, host.blocks)
    print(f"{len(blocks)} blocks over {levels} levels: upload, build and export {ms:.1f} ms")


@pytest.mark.parametrize("view3,it,tier", VIEWS, ids=lambda v: str(v)[:24])
def test_frame_with_device_table_equals_uploaded_table(dev, view3, it, tier):
    v = fd.View(*view3)
    p = fd.Params(96, 54, max_iter=it, tier=tier)
    orbit = fd.reference(v, p)
    h1, a, st1, b1 = fd.render_bla(v, p, orbit, dev=dev, raw=True)
    h2, b, st2, b2 = fd.render_bla(v, p, orbit, dev=dev, raw=True, device_table=True)
    assert h1 == h2
    for k in ("cls", "n", "z", "dz", "dexp", "status", "nu", "de", "normal"):
        x, y = getattr(a, k), getattr(b, k)
        assert (x is None) == (y is None), k
        if x is not None:
            assert x.dtype == y.dtype and np.array_equal(np.ascontiguousarray(x).view(np.uint8),
                                                         np.ascontiguousarray(y).view(np.uint8)), k
    assert st1.iterations == st2.iterations and st1.reference_len == st2.reference_len
    # shift_px is inf or NaN where h underflows (1e-400 over 96 samples), as in Rust
    assert [str(x) for x in dataclasses.astuple(b1)] == [str(x) for x in dataclasses.astuple(b2)]


def test_device_table_refusals(dev):
    v, p = fd.View(*SPIRAL, "1e-20"), fd.Params(64, 36, max_iter=20_000)
    r, _ = fd.reference(v, p)
    dc, e = fd.bla_dc_bound(v, p)
    h = dev.upload(r)
    try:
        for eps, dmax in ((2.0 ** -20, dc), (0.0, dc), (fd.EPS, 0.0), (fd.EPS, math.nan), (fd.EPS, math.inf)):
            with pytest.raises(fd.RouteError, match="eps"):
                dev.build_bla(h, eps, dmax, e)
        assert dev.build_bla(h, fd.EPS, dc, e) > 0
    finally:
        dev.free(h)
    with pytest.raises(fd.RouteError, match="unknown orbit"):
        dev.build_bla(h, fd.EPS, dc, e)
    with pytest.raises(ValueError, match="eps"):
        fd.render_bla(v, p, (r, 53), dev=dev, eps=2.0 ** -20, device_table=True)
