"""The Stripe column on the CUDA route (fdc_render_stripe) against the oracle's
(stripe.rs restated): class, escape count and z equal the route's plain render bit for
bit (recording never changes an outcome), and the stripe average of every escaped sample
equals the oracle's within 2e-6 (the terms go through CUDA's hypot / sin / atan2 / log
instead of glibc's; the same kernel source run on the host with glibc is equal bit for
bit, tests/test_kernel_emulation.py). Frames on the F64, Fixed and Scaled tiers, with and
without BLA (block starts kept, incomplete windows replayed), several windows and
frequencies, the route end to end with the .fds writer, and configuration 2's whole
frame with the stripe variant's frame time printed beside the plain kernel's."""
import numpy as np
import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib, fds, locations

pytestmark = pytest.mark.gpu
TOL = 2e-6

FRAMES = [
    (("-0.7453", "0.1127", "0.0065"), 160, 96, 5000, None, None),
    (("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28"), 128, 72, 50_000,
     2.0 ** -50, None),
    (("0", "1", "1e-300"), 96, 64, 5000, 2.0 ** -50, None),
    (("0", "1", "1e-300"), 96, 64, 5000, 2.0 ** -50, "scaled"),
]


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def render_pair(dev, view, p, eps, window, freq):
    plane, tier = fd.route._setup(view, p)
    r, bits = fd.reference(view, p)
    r.bits = bits
    bla = None
    if eps is not None:
        dc, e = fd.bla_dc_bound(view, p)
        bla = fd.Bla.build_scaled(r, eps, dc, e)
        bla = bla if bla.levels else None
    h = dev.upload(r, bla)
    try:
        flags = (_lib.DERIVATIVE if p.needs_derivative() else 0) | (_lib.BLA if bla is not None else 0)
        job = fd.route.make_job(plane, tier, p, h, r.nucleus_period(), flags)
        plain, cp, _ = dev.render_job(job, raw=True, columns=p.columns)
        got, cs, _ = dev.render_job(job, raw=True, columns=p.columns, stripe=(window, freq))
    finally:
        dev.free(h)
    return plane, tier, r, bla, plain, got, cp, cs


def oracle_stripe(view, p, tier, r, bla, window, freq):
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    t = fdref.Bla(ref, bla.eps, bla.dc_max, bla.dc_exp) if bla is not None else None
    cols = fdref.COL_NU | fdref.COL_STRIPE | (fdref.COL_DE if "de" in p.columns else 0)
    job = fdref.make_job(view.center_re, view.center_im, view.width, p.nx, p.ny, p.max_iter,
                         escape_radius=p.escape_radius, columns=cols, tier=tier, stripe_window=window,
                         stripe_freq=freq)
    return fdref.render_columns(job, ref, t)


@pytest.mark.parametrize("frame", FRAMES, ids=lambda f: f"{f[0][2]}-{f[5]}")
@pytest.mark.parametrize("window,freq", [(16, 5.0), (64, 2.5), (5, -3.0)])
def test_stripe_column_equals_oracle(dev, frame, window, freq):
    view3, nx, ny, it, eps, tier = frame
    view = fd.View(*view3)
    p = fd.Params(nx, ny, max_iter=it, columns=("nu", "de"), tier=tier)
    plane, t, r, bla, plain, got, cp, cs = render_pair(dev, view, p, eps, window, freq)
    for k in ("cls", "n", "z", "dz", "dexp", "nu", "status"):
        assert np.array_equal(got[k], plain[k]), k
    assert (cs.iterations, cs.blocks, cs.skipped) == (cp.iterations, cp.blocks, cp.skipped)
    want = oracle_stripe(view, p, t, r, bla, window, freq)
    assert np.array_equal(got["cls"], want["cls"])
    esc = want["cls"] == 0
    assert esc.any() and not got["stripe"][~esc].any()
    err = np.abs(got["stripe"][esc].astype(np.float64) - want["stripe"][esc])
    assert err.max() <= TOL, err.max()
    if bla is not None:
        assert cs.blocks > 0


def test_route_writes_the_stripe_column(dev):
    """render_with with the Stripe column end to end: the header lists it last, the .fds
    file carries it after the other columns, equal to the oracle's within the tolerance."""
    view = fd.View("-0.7453", "0.1127", "0.0065")
    p = fd.Params(64, 40, max_iter=3000, columns=("nu", "stripe"), stripe_window=12, stripe_freq=4.0)
    h, s, st, _ = fd.render_with(view, p, dev=dev)
    assert h.columns == ("class", "nu", "stripe")
    data = fds.encode(h, s)
    col = np.frombuffer(data[len(data) - 64 * 40 * 4:], np.float32)
    assert np.array_equal(col, s.stripe)
    job = fdref.make_job(view.center_re, view.center_im, view.width, 64, 40, 3000,
                         columns=fdref.COL_NU | fdref.COL_STRIPE, stripe_window=12, stripe_freq=4.0)
    want = fdref.render_columns(job)
    assert np.abs(s.stripe.astype(np.float64) - want["stripe"]).max() <= TOL


def test_stripe_on_configuration_2(dev):
    """Configuration 2's whole frame (1920x1080, the 1e-100 nucleus, 10^6 iterations, BLA,
    floatexp deltas) with the Stripe column: every sample against the oracle; the frame
    times of both variants are printed."""
    fr = locations.config2()
    plane, t, r, bla, plain, got, cp, cs = render_pair(dev, fr.view, fr.params, fr.bla_eps, 16, 5.0)
    for k in ("cls", "n", "z"):
        assert np.array_equal(got[k], plain[k]), k
    want = oracle_stripe(fr.view, fr.params, t, r, bla, 16, 5.0)
    esc = want["cls"] == 0
    err = np.abs(got["stripe"][esc].astype(np.float64) - want["stripe"][esc])
    print(f"config 2 stripe: plain kernel {cp.kernel_ms:.1f} ms, stripe kernel {cs.kernel_ms:.1f} ms, "
          f"max stripe error {err.max():.2e} over {esc.sum()} escaped samples")
    assert err.max() <= TOL, err.max()
