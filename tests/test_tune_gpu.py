"""The autotuner on a real job: it measures launch settings and both forms on row bands,
picks one, and the settings it applies leave every result unchanged (they only schedule
the same per-sample work differently)."""
import numpy as np
import pytest

import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib, tune

pytestmark = pytest.mark.gpu


def test_tuner_measures_chooses_and_keeps_results():
    dev = fd.Device(0)
    try:
        v = fd.View("-0.7453", "0.1127", "0.0065")
        p = fd.Params(128, 72, max_iter=4000, columns=("nu", "de"))
        plane, tier = fd.route._setup(v, p)
        r, bits = fd.reference(v, p)
        r.bits = bits
        dc, e = fd.bla_dc_bound(v, p)
        bla = fd.Bla.build_scaled(r, 2.0 ** -40, dc, e)
        bla = bla if bla.levels else None
        h = dev.upload(r, bla)
        flags = _lib.DERIVATIVE | (_lib.BLA if bla is not None else 0)
        job = fd.route.make_job(plane, tier, p, h, r.nucleus_period(), flags)
        base, cb, _ = dev.render_job(job, raw=True)
        settings = [tune.Setting(d, b, t) for d in ((1, 8) if bla is not None else (0,)) for b in (0, 3)
                    for t in (8, 32)]
        tuner = tune.Tuner(dev, settings=settings, reps=1)
        choice = tuner.choice(job)
        assert len(choice.table) == len(settings) + 1 and choice.ms > 0 and choice.match is not None
        assert choice.plain_ms == min(ms for s, ms in choice.table if not s.f32)
        assert tuner.choice(job) is choice  # cached per job kind
        s = tuner.apply(job)
        got, cg, _ = dev.render_job(job, raw=True)
        if not s.f32:
            for k in ("cls", "n", "z", "dz", "dexp", "nu", "de"):
                assert np.array_equal(got[k], base[k]), k
            assert (cg.iterations, cg.blocks, cg.skipped) == (cb.iterations, cb.blocks, cb.skipped)
        # row-major order, narrow tiles: still the same results
        dev.tune(defer=1, blocks_per_sm=2, tile_w=1, order=_lib.ORDER_ROWS)
        job.flags &= ~_lib.F32
        again, _, _ = dev.render_job(job, raw=True)
        for k in ("cls", "n", "z", "dz", "dexp"):
            assert np.array_equal(again[k], base[k]), k
        dev.free(h)
    finally:
        dev.close()
