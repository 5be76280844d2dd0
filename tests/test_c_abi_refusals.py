"""The C-ABI's refusals, which need no device: every entry point that takes a context
returns FDC_INVALID for a null one (no crash, no CUDA call), the no-op teardown calls
accept null, and the allocation-free entry point checks every argument before it touches
a device, each refusal with its own message (pointers off their element boundary
included); a valid job on a host without a GPU then fails with FDC_NO_DEVICE, as
fdc_open does. The route maps each status to an
exception and never falls back to the CPU (frame.rs:357-368 leaves the restart to the
caller)."""
import ctypes as C

import numpy as np
import pytest

from fractodactyl_b200 import _lib


@pytest.fixture(scope="module")
def L():
    return _lib.lib()


def test_null_context_refused(L):
    c = _lib.Counters()
    job, out, t = _lib.Job(), _lib.Out(), _lib.Tuning()
    a = np.zeros(8)
    orbit = C.c_int32(7)
    assert L.fdc_last_error(None) == b"no context"
    L.fdc_close(None)
    L.fdc_batch_free(None, None)
    assert L.fdc_open(0, None) == _lib.INVALID
    assert L.fdc_upload_orbit(None, a.ctypes.data, a.ctypes.data, 8, 0, C.byref(orbit)) == _lib.INVALID
    assert orbit.value == 7  # untouched
    assert L.fdc_free_orbit(None, 0) == _lib.INVALID
    assert L.fdc_upload_bla(None, 0, a.ctypes.data, a.ctypes.data, 1, 1e-15, 1.0, 0) == _lib.INVALID
    lv = C.c_uint32(5)
    assert L.fdc_build_bla(None, 0, 1e-15, 1.0, 0, C.byref(lv), None) == _lib.INVALID and lv.value == 5
    assert L.fdc_upload_series(None, 0, 8, 4, 1.0, a.ctypes.data, 2) == _lib.INVALID
    assert L.fdc_upload_error_radius(None, 0, a.ctypes.data, 8) == _lib.INVALID
    assert L.fdc_render(None, C.byref(job), C.byref(out), C.byref(c)) == _lib.INVALID
    assert L.fdc_render_bounded(None, C.byref(job), C.byref(out), None, C.byref(c)) == _lib.INVALID
    assert L.fdc_render_bounded(None, C.byref(job), C.byref(out), C.byref(_lib.BoundOut()), C.byref(c)) == _lib.INVALID
    col = np.zeros(4, np.float32)
    assert L.fdc_render_stripe(None, C.byref(job), C.byref(out), C.byref(_lib.Stripe(16, 5.0)), col.ctypes.data,
                               C.byref(c)) == _lib.INVALID
    assert L.fdc_render_stripe(None, C.byref(job), C.byref(out), None, None, C.byref(c)) == _lib.INVALID
    assert L.fdc_set_tuning(None, C.byref(t)) == _lib.INVALID
    assert L.fdc_get_tuning(None, C.byref(t)) == _lib.INVALID
    b = C.c_void_p()
    assert L.fdc_batch_create(None, C.addressof(job), C.addressof(out), 1, C.byref(b)) == _lib.INVALID
    assert L.fdc_batch_run(None, None, C.byref(c), None) == _lib.INVALID


def _job(**kw):
    j = _lib.Job(orbit=0, tier=1, nx=64, ny=32, ss=1, flags=_lib.DERIVATIVE, c_re=-0.75, c_im=0.1, h_m=1.5, h_e=-40,
                 cos_rot=1.0, sin_rot=0.0, max_iter=1000, escape_radius=256.0, nucleus_period=-1)
    for k, v in kw.items():
        setattr(j, k, v)
    return j


_HOLD = np.zeros(64)  # 16-byte aligned host memory; the refusals never touch it


def _noalloc(L, job, orbit_len=100, orbit=True, out=True, device=0, orbit_offset=0, columns=None):
    z = np.zeros(2 * max(orbit_len, 3) + 2)
    err = C.create_string_buffer(256)
    o = _lib.Out()
    for name, off in (columns or {}).items():
        setattr(o, name, _HOLD.ctypes.data + off)
    st = L.fdc_render_noalloc(device, (z.ctypes.data + orbit_offset) if orbit else None, orbit_len, C.byref(job),
                              C.byref(o) if out else None, None, None, None, err, 256)
    return st, err.value.decode()


MASK = np.ones(64 * 32, np.uint8)

REFUSALS = [
    (dict(orbit=False), {}, "null argument"),
    (dict(out=False), {}, "null argument"),
    (dict(device=-1), {}, "device index out of range"),
    (dict(device=64), {}, "device index out of range"),
    ({}, dict(flags=_lib.BLA), "plain form without BLA or series"),
    ({}, dict(flags=_lib.SERIES), "plain form without BLA or series"),
    ({}, dict(flags=_lib.F32), "plain form without BLA or series"),
    ({}, dict(flags=_lib.SHIFT), "plain form without BLA or series"),
    ({}, dict(mask=MASK.ctypes.data), "no mask or offsets"),
    (dict(orbit_len=2), {}, "orbit length"),
    (dict(orbit_len=(1 << 20) + 1), {}, "orbit length"),
    ({}, dict(nx=0), "whole number of pixels"),
    ({}, dict(ss=3), "whole number of pixels"),
    ({}, dict(nx=1 << 16, ny=1 << 15), "larger than 2^31"),
    ({}, dict(tier=3), "unknown tier"),
    ({}, dict(max_iter=1 << 32), "below 2^32"),
    ({}, dict(escape_radius=0.0), "escape radius"),
    ({}, dict(escape_radius=1e200), "escape radius"),
    ({}, dict(escape_radius=float("nan")), "escape radius"),
    ({}, dict(h_m=2.0), "h_m must lie"),
    ({}, dict(h_m=0.75), "h_m must lie"),
    ({}, dict(h_e=-(1 << 31)), "h_e must lie"),
    ({}, dict(nucleus_period=-2), "nucleus_period"),
    ({}, dict(first_row=32), "row range"),
    ({}, dict(first_row=8, rows=25), "row range"),
    ({}, dict(first_col=64), "column range"),
    ({}, dict(first_col=60, cols=5), "column range"),
    ({}, dict(ny=8192), "rows per call"),
    (dict(orbit_offset=8), {}, "orbit must be 16-byte aligned"),
    (dict(columns=dict(z=8)), {}, "column z must be 16-byte aligned"),
    (dict(columns=dict(dz=8)), {}, "column dz must be 16-byte aligned"),
    (dict(columns=dict(nu=4)), {}, "column nu must be 8-byte aligned"),
    (dict(columns=dict(dexp=4)), {}, "column dexp must be 8-byte aligned"),
    (dict(columns=dict(n=2)), {}, "column n must be 4-byte aligned"),
    (dict(columns=dict(de=2)), {}, "column de must be 4-byte aligned"),
    (dict(columns=dict(normal=1)), {}, "column normal must be 2-byte aligned"),
]


@pytest.mark.parametrize("call,fields,message", REFUSALS)
def test_noalloc_refusals(L, call, fields, message):
    st, err = _noalloc(L, _job(**fields), **call)
    assert st == _lib.INVALID and message in err, err


def test_noalloc_valid_job_without_device(L):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ok = dict(rows=8160, ny=16320)  # the largest window one call takes, then ragged windows
    for fields in (ok, dict(first_row=8, rows=24), dict(first_col=60, cols=4), {}):
        st, err = _noalloc(L, _job(**fields))
        assert st == _lib.NO_DEVICE and err.startswith("no CUDA device"), (fields, err)
    # aligned columns of every element size pass the checks and meet the same device test
    st, err = _noalloc(L, _job(), columns=dict(z=16, dz=32, nu=8, dexp=8, n=4, de=4, normal=2, cls=1, status=3))
    assert st == _lib.NO_DEVICE, err
    # the same status fdc_open gives for a host without a usable device
    h = C.c_void_p()
    assert L.fdc_open(0, C.byref(h)) == _lib.NO_DEVICE
    # a short error buffer is truncated and terminated, never overrun
    err = (C.c_char * 8)()
    z = np.zeros(200)
    st = L.fdc_render_noalloc(0, z.ctypes.data, 100, C.byref(_job(tier=9)), C.byref(_lib.Out()), None, None, None,
                              err, 8)
    assert st == _lib.INVALID and bytes(err) == b"unknown\x00"
