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
