"""The oracle's Stripe column (crates/fd-kernel/src/stripe.rs, sample.rs:231-236,
387-403, 470-472, 576-579), checked against the reference's own stripe test restated
(sample.rs:851-893) and frame properties:

- a shallow sample's stripe value equals the last-16 average of 0.5 + 0.5 sin(5 arg z)
  over direct f64 iteration, interpolated with the escape fraction, within 1e-4;
- with BLA blocks skipping iterates, the replay from a kept block start gives the plain
  kernel's value within 1e-4, and recording never changes the outcome;
- on frames (plain and BLA, every tier) the recorder leaves class, count and z as the
  untraced render's, values lie in [0, 1] for escaped samples and are 0 elsewhere, and the
  BLA frame's values stay within 1e-4 of the plain frame's on most samples;
- the .fds writer places the column last, after the others, as f32.
"""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import fdref  # noqa: E402

EPS_MAX = 2.0 ** -41


def direct_stripe(cr, ci, window=16, freq=5.0, r2=1e20):
    zr = zi = 0.0
    terms = []
    while True:
        zr, zi = zr * zr - zi * zi + cr, 2.0 * zr * zi + ci
        terms.append(0.5 + 0.5 * math.sin(freq * math.atan2(zi, zr)))
        f2 = zr * zr + zi * zi
        if f2 > r2:
            n = len(terms)
            now = sum(terms[n - window:]) / window
            before = sum(terms[n - window - 1:n - 1]) / window
            frac = min(max(1.0 - math.log2(math.log(f2) / math.log(r2)), 0.0), 1.0)
            return n, before * (1.0 - frac) + now * frac


def test_stripe_matches_direct_iteration():
    cr, ci, ar, ai = -0.743, 0.1312, 2e-5, -1e-5
    r = fdref.Ref.f64(cr, ci, 100_000, 1e10)
    n, want = direct_stripe(cr + ar, ci + ai)
    o, got = fdref.iterate_stripe(r, None, ar=ar, ai=ai, max_iter=100_000, r2=1e20)
    assert o["kind"] == "escaped" and o["n"] == n
    assert abs(got - want) < 1e-4, (got, want)


@pytest.mark.parametrize("ar,ai", [(1e-17, 0.0), (-1e-17, 1e-17), (0.0, -1.4e-17)])
def test_stripe_survives_bla_blocks(ar, ai):
    r = fdref.Ref.f64(0.2501, 0.0, 100_000, 1e10)
    bla = fdref.Bla(r, EPS_MAX, 2e-17)
    po, plain = fdref.iterate_stripe(r, None, ar=ar, ai=ai, max_iter=100_000, r2=1e20)
    fo, fast = fdref.iterate_stripe(r, bla, ar=ar, ai=ai, max_iter=100_000, r2=1e20)
    untraced = fdref.iterate(r, bla, ar=ar, ai=ai, max_iter=100_000, r2=1e20, derivative=False)
    assert fo["blocks"] > 0 and po["kind"] == "escaped"
    assert (fo["kind"], fo["n"], fo["zr"], fo["zi"]) == (untraced["kind"], untraced["n"], untraced["zr"],
                                                         untraced["zi"])
    assert plain > 0.0 and abs(plain - fast) < 1e-4, (plain, fast)


FRAMES = [
    # view, grid, iterations, BLA eps, tier
    (("-0.7453", "0.1127", "0.0065"), 48, 32, 3000, None, None),
    (("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28"), 48, 32, 30_000,
     2.0 ** -50, None),
    (("0", "1", "1e-300"), 40, 24, 5000, 2.0 ** -50, None),
    (("0", "1", "1e-300"), 40, 24, 5000, 2.0 ** -50, "scaled"),
]


@pytest.mark.parametrize("frame", FRAMES, ids=lambda f: f"{f[0][2]}-{f[5]}")
@pytest.mark.parametrize("window,freq", [(16, 5.0), (64, 2.5), (1, -3.0)])
def test_frame_stripe_properties(frame, window, freq):
    (re_, im_, w), nx, ny, it, eps, tier = frame
    cols = fdref.COL_NU | fdref.COL_STRIPE
    job = fdref.make_job(re_, im_, w, nx, ny, it, columns=cols, tier=tier, threads=2, stripe_window=window,
                         stripe_freq=freq)
    ref = fdref.Ref.for_job(job)
    bla = None
    if eps is not None:
        dc, e = fdref.bla_dc_bound(job)
        bla = fdref.Bla(ref, eps, dc, e)
    traced = fdref.render_columns(job, ref, bla)
    untraced = fdref.render(fdref.make_job(re_, im_, w, nx, ny, it, columns=fdref.COL_NU, tier=tier, threads=2),
                            ref, bla, raw=True)
    for k in ("cls", "n", "z"):
        assert np.array_equal(traced[k], untraced[k]), k
    esc = traced["cls"] == 0
    s = traced["stripe"]
    assert esc.any() and np.all(s[~esc] == 0.0)
    assert np.all((s[esc] >= 0.0) & (s[esc] <= 1.0))
    if bla is not None and bla.levels:
        assert traced["stats"]["blocks"] > 0
        plain = fdref.render_columns(job, ref, None)
        close = np.abs(plain["stripe"][esc] - s[esc]) < 1e-4
        assert close.mean() > 0.9, close.mean()


def test_fds_writes_the_stripe_column_last():
    re_, im_, w = "-0.7453", "0.1127", "0.0065"
    base = fdref.render_fds(fdref.make_job(re_, im_, w, 9, 5, 500, columns=fdref.COL_NU, threads=1))
    with_stripe = fdref.render_fds(fdref.make_job(re_, im_, w, 9, 5, 500, columns=fdref.COL_NU | fdref.COL_STRIPE,
                                                  threads=1))
    job = fdref.make_job(re_, im_, w, 9, 5, 500, columns=fdref.COL_NU | fdref.COL_STRIPE, threads=1)
    s = fdref.render_columns(job)["stripe"]
    col = with_stripe[len(with_stripe) - 184:][:180]  # 45 f32, padded to 8 bytes: the last 184 bytes
    assert np.array_equal(np.frombuffer(col, np.float32), s) and s.any()
    assert len(with_stripe) == len(base) + 184
