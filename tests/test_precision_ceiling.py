"""The accuracy ceiling of FP32-mantissa deltas, on the CPU with the oracle
(oracle/precision_ceiling.py): the reference's algorithm with every delta rounded to 24
bits, everything else binary64, against the same algorithm unrounded, on a seeded subset
of configuration 2's frame. An ideal FP32 delta already misses the 99.9% escape-count
bar (the full 20,000-sample run measures 91.6%), and so does a cut-over that keeps FP32
deltas to the first 16 iterations; the class (escaped or not) is kept. With the knob
off, the oracle is the reference's algorithm again, bit for bit."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import fdref  # noqa: E402
import precision_ceiling as pc  # noqa: E402


def test_fp32_delta_ceiling_on_config2():
    v = pc.views()[0]
    assert v["name"].startswith("c2-")
    rows, _ = pc.run(v, 2000, [24])
    r = rows[0]
    assert r["samples"] == 2000 and r["escape_agreement"] == 1.0
    assert 0.85 < r["count_match"] < 0.97, r
    job = fdref.make_job(v["re"], v["im"], v["width"], v["nx"], v["ny"], v["max_iter"],
                         escape_radius=v["escape_radius"], columns=fdref.COL_NU, tier=v["tier"])
    ref = fdref.Ref.for_job(job)
    dc, e = fdref.bla_dc_bound(job)
    bla = fdref.Bla(ref, v["bla"], dc, e)
    n = v["nx"] * v["ny"]
    mask = np.zeros(n, np.uint8)
    mask[np.random.default_rng(5).choice(n, 2000, replace=False)] = 1
    sel = mask.astype(bool)
    base = fdref.render_columns(job, ref, bla, mask=mask)
    try:
        fdref.set_delta_bits(24, 0, 16)  # FP32 deltas for the first 16 iterations only
        early = fdref.render_columns(job, ref, bla, mask=mask)
    finally:
        fdref.set_delta_bits(0)
    assert pc.agreement(base, early, sel)["count_match"] < 0.99
    again = fdref.render_columns(job, ref, bla, mask=mask)
    for k in ("cls", "n", "z", "dz", "dexp"):
        assert np.array_equal(again[k][sel], base[k][sel]), k
