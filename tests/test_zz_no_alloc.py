"""The allocation-free entry point (fdc_render_noalloc) against fdc_render.

fdc_render_noalloc is for callers that cannot allocate device memory (a render service
whose device memory all comes from its own pool): they pass the orbit and the output
columns as device buffers and the library allocates nothing, using a fixed device
array for its scratch. This test allocates those buffers itself (with torch), calls the
entry point through the C ABI twice in a row, and checks every output against the
context-based route's on the same frame: class, escape count, z and dz/dc bit-exact,
nu within 1e-12 relative (both are the same kernel arithmetic, so they agree exactly in
practice). It also checks that a job needing more scratch than the array holds is
refused. The file is named to run last.
"""
import ctypes as C

import numpy as np
import pytest

import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib

pytestmark = pytest.mark.gpu

FRAMES = [
    # view, grid, iterations, tier: a Fixed-tier and a Scaled-tier frame, with derivative
    (fd.View("-0.7436438870371587", "0.1318259042053120", "1e-12"), 160, 90, 20_000, None),
    (fd.View("0", "1", "1e-300", 0.4), 128, 72, 20_000, None),
]


def noalloc_render(torch, plane, tier, p, r, nucleus, flags):
    dev = torch.device("cuda", 0)
    n = p.nx * p.ny
    orbit = torch.from_numpy(np.ascontiguousarray(np.stack([r.re, r.im], axis=1).reshape(-1))).to(dev)
    bufs = {"cls": torch.zeros(n, dtype=torch.uint8, device=dev), "n": torch.zeros(n, dtype=torch.int32, device=dev),
            "nu": torch.zeros(n, dtype=torch.float64, device=dev), "z": torch.zeros(2 * n, dtype=torch.float64, device=dev),
            "dz": torch.zeros(2 * n, dtype=torch.float64, device=dev), "dexp": torch.zeros(n, dtype=torch.int64, device=dev),
            "status": torch.zeros(n, dtype=torch.uint8, device=dev)}
    out = _lib.Out()
    for k, t in bufs.items():
        setattr(out, k, t.data_ptr())
    job = fd.route.make_job(plane, tier, p, 0, nucleus, flags)
    rows = np.zeros(p.ny, np.uint64)
    cnt = _lib.Counters()
    err = C.create_string_buffer(512)
    torch.cuda.synchronize()
    st = _lib.lib().fdc_render_noalloc(0, orbit.data_ptr(), len(r), C.byref(job), C.byref(out), rows.ctypes.data,
                                       C.byref(cnt), None, err, 512)
    assert st == _lib.OK, err.value.decode()
    torch.cuda.synchronize()
    host = {k: t.cpu().numpy() for k, t in bufs.items()}
    host["n"] = host["n"].view(np.uint32)
    host["z"] = host["z"].reshape(n, 2)
    host["dz"] = host["dz"].reshape(n, 2)
    return host, rows, cnt


@pytest.mark.parametrize("frame", FRAMES, ids=lambda f: f[0].width)
def test_noalloc_matches_context_route_twice(frame):
    torch = pytest.importorskip("torch")
    view, nx, ny, it, tier_name = frame
    p = fd.Params(nx, ny, max_iter=it, columns=("nu", "de", "normal"), tier=tier_name)
    plane, tier = fd.route._setup(view, p)
    r, bits = fd.reference(view, p)
    r.bits = bits
    nucleus = r.nucleus_period()
    flags = _lib.DERIVATIVE
    ref_dev = fd.Device(0)
    h = ref_dev.upload(r)
    try:
        want, cnt_want, _ = ref_dev.render_job(fd.route.make_job(plane, tier, p, h, nucleus, flags), raw=True,
                                               columns=("nu",))
    finally:
        ref_dev.free(h)
        ref_dev.close()
    for call in range(2):  # two calls in a row share the scratch array
        got, rows, cnt = noalloc_render(torch, plane, tier, p, r, nucleus, flags)
        assert np.array_equal(got["cls"], want["cls"]), call
        assert np.array_equal(got["n"], want["n"]), call
        esc = want["cls"] == 0
        assert np.array_equal(got["z"][esc].view(np.uint64), want["z"][esc].view(np.uint64)), call
        assert np.array_equal(got["dz"][esc].view(np.uint64), want["dz"][esc].view(np.uint64)), call
        assert np.array_equal(got["dexp"][esc], want["dexp"][esc]), call
        rel = np.abs(got["nu"][esc] - want["nu"][esc]) / np.abs(want["nu"][esc])
        assert rel.size == 0 or rel.max() <= 1e-12, call
        assert np.all(got["status"] == 1), call
        assert cnt.samples == nx * ny and cnt.iterations == cnt_want.iterations, call
        assert int(rows.sum()) == cnt.iterations, call


def test_noalloc_refuses_jobs_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    view = fd.View("-0.75", "0.1", "1e-3")
    limit = (65536 - 256) // 8
    p = fd.Params(8, limit + 1, max_iter=100)
    plane, tier = fd.route._setup(view, p)
    r, bits = fd.reference(view, p)
    orbit = torch.zeros(2 * len(r), dtype=torch.float64, device="cuda")
    job = fd.route.make_job(plane, tier, p, 0, None, 0)
    out = _lib.Out()
    err = C.create_string_buffer(512)
    st = _lib.lib().fdc_render_noalloc(0, orbit.data_ptr(), len(r), C.byref(job), C.byref(out), None, None, None,
                                       err, 512)
    assert st == _lib.INVALID and b"rows per call" in err.value
