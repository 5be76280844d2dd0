"""Host copies of 1 MiB and more go through the context's two pinned chunk slots and its
copy threads (in chunks of a quarter of the copy); smaller ones go direct. A frame rendered
whole, with its columns, per-sample offsets and mask staged, equals the same frame rendered
as row windows whose copies are all below the threshold, bit for bit; the whole frame's
class, count and z at escape also equal the oracle's."""
import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

pytestmark = pytest.mark.gpu

STAGE_MIN = 1 << 20  # fdcuda.cu: copies from this size up are staged
VIEW = ("-0.7453", "0.1127", "0.0065")
KIND = {"escaped": 0, "interior": 1, "unresolved": 2}
WIDTH = {"cls": 1, "status": 1, "n": 4, "nu": 8, "de": 4, "normal": 2, "z": 16, "dz": 16, "dexp": 8}


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def _job(dev, nx, ny, max_iter):
    v = fd.View(*VIEW)
    p = fd.Params(nx, ny, max_iter=max_iter, columns=("nu", "de", "normal"))
    plane, tier = fd.route._setup(v, p)
    r, bits = fd.reference(v, p)
    r.bits = bits
    h = dev.upload(r, None)
    return p, plane, tier, r, h, fd.route.make_job(plane, tier, p, h, r.nucleus_period(), _lib.DERIVATIVE)


def _host(n):
    out = {k: np.zeros(n, dt) for k, dt in (("cls", np.uint8), ("status", np.uint8), ("n", np.uint32),
                                            ("nu", np.float64), ("de", np.float32), ("normal", np.uint16),
                                            ("dexp", np.int64))}
    out["z"] = np.zeros((n, 2))
    out["dz"] = np.zeros((n, 2))
    return out


def _whole_and_windows(dev, job, window_rows):
    n = job.nx * job.ny
    job.first_row, job.rows = 0, job.ny
    whole, _, _ = dev.render_job(job, host_out=_host(n))
    parts = _host(n)
    for r0 in range(0, job.ny, window_rows):
        job.first_row, job.rows = r0, min(window_rows, job.ny - r0)
        dev.render_job(job, host_out=parts)
    job.first_row, job.rows = 0, job.ny
    return whole, parts


def _assert_same(whole, parts):
    for k in whole:
        assert np.array_equal(whole[k], parts[k]), k


def test_staged_columns_and_offsets_equal_direct_windows(dev):
    nx, ny, rows = 1024, 288, 32
    p, plane, tier, r, h, job = _job(dev, nx, ny, 2000)
    n = nx * ny
    # the whole frame stages every column of 4 bytes and more (z in 4 chunks), a window none
    assert all(WIDTH[k] * n >= STAGE_MIN for k in ("n", "nu", "de", "z", "dz", "dexp"))
    assert 16 * n >= 4 * STAGE_MIN
    assert all(WIDTH[k] * rows * nx < STAGE_MIN for k in WIDTH)
    try:
        whole, parts = _whole_and_windows(dev, job, rows)
        _assert_same(whole, parts)
        assert whole["status"].all()
        # the staged whole frame against the oracle, every sample
        ref = fdref.Ref.arrays(r.re, r.im, r.bits)
        want = fdref.render(fdref.make_job(*VIEW, nx, ny, p.max_iter, escape_radius=p.escape_radius,
                                           columns=fdref.COL_NU, tier=tier), ref, None, raw=True)
        assert np.array_equal(whole["cls"], want["cls"])
        assert np.array_equal(whole["n"], want["n"].astype(np.uint32))
        esc = want["cls"] == 0
        assert esc.mean() > 0.5
        assert np.array_equal(whole["z"][esc], want["z"][esc])

        # per-sample offsets (16 bytes a sample): staged for the whole frame, direct per window
        rng = np.random.default_rng(7)
        jj, ii = np.divmod(np.arange(n), nx)
        offs = np.empty((n, 2))
        offs[:, 0] = ii + rng.uniform(0.0, 1.0, n) - nx / 2
        offs[:, 1] = -(jj + rng.uniform(0.0, 1.0, n) - ny / 2)
        job.offsets = offs.ctypes.data
        whole_o, parts_o = _whole_and_windows(dev, job, rows)
        _assert_same(whole_o, parts_o)
        assert not np.array_equal(whole_o["n"], whole["n"])  # the offsets moved the samples
        # sampled samples against the oracle's iterate, set up as its grid does per tier
        # (oracle fdref_grid.cpp, after grid.rs:709-723)
        r2 = p.escape_radius ** 2
        step = plane.h()
        for k in rng.choice(n, 300, replace=False):
            ux, uy = offs[k]
            if tier == 2:
                o = fdref.iterate(ref, None, extended=True, ar=ux * plane.h_m, ai=uy * plane.h_m,
                                  offset_exp=plane.h_e, max_iter=p.max_iter, r2=r2)
            else:
                ar, ai = ux * step, uy * step
                c = (plane.c_re + ar, plane.c_im + ai) if tier == 0 else None
                o = fdref.iterate(ref, None, extended=False, c=c, ar=ar, ai=ai, max_iter=p.max_iter, r2=r2)
            kind = KIND[o["kind"]]
            assert whole_o["cls"][k] == kind, k
            assert whole_o["n"][k] == (p.max_iter if kind == 2 else o["n"]), k
            if kind == 0:
                assert (whole_o["z"][k, 0], whole_o["z"][k, 1]) == (o["zr"], o["zi"]), k
    finally:
        job.offsets = None
        dev.free(h)


def test_staged_mask_equals_direct_windows(dev):
    nx, ny, rows = 1024, 1024, 256
    p, plane, tier, r, h, job = _job(dev, nx, ny, 300)
    n = nx * ny
    assert n >= STAGE_MIN and rows * nx < STAGE_MIN  # the mask: staged whole, direct per window
    mask = (np.random.default_rng(11).random(n) < 0.5).astype(np.uint8)
    job.mask = mask.ctypes.data
    try:
        whole, parts = _whole_and_windows(dev, job, rows)
        _assert_same(whole, parts)
        assert np.array_equal(whole["status"], mask)
    finally:
        job.mask = None
        dev.free(h)
