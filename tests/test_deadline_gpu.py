"""A job's deadline on the device (fdc_job.deadline_ms): once it has passed, warps take no
new samples, finish the ones they hold and the render returns FDC_TIMEOUT. Exactly the
finished samples are written (status 1, equal to the unlimited render's), the others
keep zeroed columns and status 0 for the caller's CPU restart (frame.rs:338-341), and
the counters cover the finished samples. The frame (589,824 samples) is larger than one
wave of the persistent grid at any occupancy, so a 1 us deadline always leaves samples
untaken; nothing waits on anything, the kernel ends as soon as its held samples do."""
import numpy as np
import pytest

import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

pytestmark = pytest.mark.gpu


def test_deadline_returns_timeout_and_exact_finished_samples():
    dev = fd.Device(0)
    try:
        v = fd.View("-0.7453", "0.1127", "0.0065")
        p = fd.Params(1024, 576, max_iter=20_000, columns=("nu",))
        plane, tier = fd.route._setup(v, p)
        r, bits = fd.reference(v, p)
        r.bits = bits
        h = dev.upload(r)
        try:
            job = fd.route.make_job(plane, tier, p, h, r.nucleus_period(), 0)
            full, _, st = dev.render_job(job, raw=True, columns=("nu",))
            assert st == _lib.OK and full["status"].all()
            job.deadline_ms = 1e-3
            got, cnt, st = dev.render_job(job, raw=True, columns=("nu",))
        finally:
            dev.free(h)
    finally:
        dev.close()
    done = got["status"] != 0
    assert st == _lib.TIMEOUT
    assert done.sum() < done.size and cnt.samples == done.sum()
    for k in ("cls", "n", "nu", "z"):
        assert np.array_equal(got[k][done], full[k][done]), k
        assert not got[k][~done].any(), k
    assert cnt.iterations == int(got["n"][done].astype(np.int64).sum())


def test_route_returns_finished_samples_and_the_restart_mask():
    """The route's side of the deadline (frame.rs:338-341): render_with with a deadline the
    frame cannot meet raises Incomplete carrying the device's finished samples and the mask
    of the unfinished ones; the CPU render of just those (the oracle's masked render here)
    merged in is the whole frame, with its iteration count."""
    import fdref
    v = fd.View("-0.7453", "0.1127", "0.0065")
    p = fd.Params(1024, 576, max_iter=20_000, columns=("nu",))
    dev = fd.Device(0)
    try:
        with pytest.raises(fd.Incomplete) as ex:
            fd.render_with(v, p, dev=dev, raw=True, deadline_ms=1e-3)
    finally:
        dev.close()
    inc = ex.value
    assert 0 < inc.mask.sum() < p.nx * p.ny and np.array_equal(inc.mask, inc.samples.status == 0)
    plane, tier = fd.route._setup(v, p)
    job = fdref.make_job(v.center_re, v.center_im, v.width, p.nx, p.ny, p.max_iter, columns=fdref.COL_NU, tier=tier)
    ref = fdref.Ref.for_job(job)
    part = fdref.render_columns(job, ref, None, mask=inc.mask.astype(np.uint8))
    cpu = fd.Samples(cls=part["cls"], nu=part["nu"], n=part["n"].astype(np.uint32), z=part["z"], dz=part["dz"],
                     dexp=part["dexp"])
    merged, st = inc.merge(cpu, fd.Stats(0, 0.0, part["stats"]["iterations"]))
    whole = fdref.render(job, ref, None, raw=True)
    assert np.array_equal(merged.cls, whole["cls"]) and np.array_equal(merged.n, whole["n"].astype(np.uint32))
    esc = whole["cls"] == 0
    assert np.array_equal(merged.z[esc], whole["z"][esc])
    assert st.iterations == whole["stats"]["iterations"]
