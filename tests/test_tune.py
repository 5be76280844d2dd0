"""The autotuner's selection logic on the CPU, with a fake measurement: it keeps the
fastest plain-form launch setting, and takes the FP32 form only when that is faster and
its escape counts agree with the plain form's on at least the acceptance share."""
import numpy as np

from fractodactyl_b200 import tune


def fake(times, f32_ms, f32_diff):
    """measure() whose plain results are all equal and whose FP32 result differs on
    `f32_diff` of 10,000 samples."""
    base = {"cls": np.zeros(10_000, np.uint8), "n": np.arange(10_000, dtype=np.uint32)}

    def measure(s):
        if s.f32:
            out = {k: v.copy() for k, v in base.items()}
            out["n"][:f32_diff] += 1
            return f32_ms, out
        return times[(s.defer, s.blocks_per_sm, s.tile_w)], base

    return measure


def test_picks_fastest_plain_setting_and_rejects_inaccurate_f32():
    settings = tune.candidates(bla=True, defers=(1, 8), blocks=(0,), tiles=(8, 16))
    times = {(1, 0, 8): 10.0, (8, 0, 8): 7.0, (1, 0, 16): 9.0, (8, 0, 16): 8.0}
    c = tune.choose(fake(times, f32_ms=3.0, f32_diff=100), settings)
    assert c.setting == tune.Setting(8, 0, 8) and c.ms == 7.0
    assert abs(c.match - 0.99) < 1e-12  # faster but below the 99.9% bar: plain form kept
    assert len(c.table) == 5


def test_takes_f32_when_faster_and_accurate():
    settings = tune.candidates(bla=False, blocks=(0, 4), tiles=(8,))
    times = {(0, 0, 8): 5.0, (0, 4, 8): 4.0}
    c = tune.choose(fake(times, f32_ms=3.0, f32_diff=5), settings)
    assert c.setting == tune.Setting(0, 4, 8, f32=True) and c.plain_ms == 4.0
    c = tune.choose(fake(times, f32_ms=4.5, f32_diff=0), settings)  # accurate but slower
    assert c.setting == tune.Setting(0, 4, 8, f32=False)


def test_bands_cover_the_frame_within_bounds():
    for ny in (1, 7, 16, 17, 270, 1080, 2160):
        bs = tune.bands(ny)
        assert bs and all(0 <= f and f + h <= ny for f, h in bs)
        assert len(set(bs)) == len(bs)
    assert tune.bands(1080) == [(127, 16), (397, 16), (667, 16), (937, 16)]


def test_candidates_without_bla_have_no_deferral():
    assert all(s.defer == 0 for s in tune.candidates(bla=False))
    assert {s.defer for s in tune.candidates(bla=True)} == set(tune.DEFERS)


def test_cached_centres_follow_their_recipe():
    """The cached centres of configurations 3-5 carry the seeds, widths and precisions the
    recipe specifies; the cheapest one (a 1e-21 location) is recomputed and equal."""
    from fractodactyl_b200 import locations
    spec = locations.specs()
    for name, entries in spec.items():
        got = locations.cached(name)
        assert [(d["seed"], d["log10_width"], d["bits"]) for d in got] == \
            [(d["seed"], d["log10_width"], d["bits"]) for d in entries]
        assert all(d["period"] > 0 and -3.0 < d["log10_size_over_width"] < -0.5 for d in got)
    d = min(locations.cached("c5"), key=lambda d: d["bits"])
    assert locations._compute({k: d[k] for k in ("seed", "log10_width", "bits")}) == d
