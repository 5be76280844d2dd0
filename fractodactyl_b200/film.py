"""Zoom films on the CUDA route, written as the sample files fd film reads.

Every frame of a film (one centre, widths zooming in) is rendered by one batch replay
over one shared reference orbit with a BLA table per frame (workloads.film). The device
returns each escaped sample's raw state (z, dz/dc and its exponent); the columns are
encoded on the host with the host's libm (fdh_encode = Store::put, store.rs:66-112),
which makes them the CPU route's bytes, and each frame is written as an .fds v1 file
(fd_samples::write, crates/fd-samples/src/write.rs:8-53) - the files the reference's
film path renders per keyframe through fd_kernel::render_bla (crates/fd-cli/src/film.rs).
"""
import dataclasses
import os
from typing import List, Optional, Sequence

from . import fds, workloads
from .route import Header, Samples, encode_host

ROUTE_SUFFIX = " gpu-perturb-cuda/1"  # appended to the kernel id, as frame.rs:345-349 does for its route


def render_film(dev, frames: Sequence, out_dir: Optional[str] = None, columns=("nu", "de", "normal"),
                suffix: str = ROUTE_SUFFIX, threads: int = 0) -> List[bytes]:
    """The .fds bytes of every frame of `frames` (locations.Frame: view and params of one
    centre); with out_dir, also written there as frame_NNNN.fds. The kernel id is the CPU
    route's (view.rs:90-96 with the shared orbit's bits, " bla/1" where the frame has a
    table) followed by `suffix`."""
    js = workloads.film(dev, list(frames))
    try:
        b = dev.batch(js.jobs, columns=(), raw=True)
        try:
            b.run()
            per, _ = b.all_columns()
        finally:
            b.free()
    finally:
        js.free(dev)
    bits = js.refs[0].bits
    cols = ("class",) + tuple(c for c in ("nu", "de", "normal") if c in columns)
    out = []
    for k, (f, pl, tier, table) in enumerate(zip(frames, js.planes, js.tiers, js.blas)):
        a = per[k]
        s = Samples(cls=a["cls"].copy(), n=a["n"].copy(), z=a["z"].copy(), dz=a["dz"].copy(),
                    dexp=a["dexp"].copy(), status=a["status"].copy())
        plane = dataclasses.replace(pl, bits=bits)  # the shared orbit's precision
        encode_host(plane, f.params.ss, s, columns, threads)
        kernel = plane.kernel(tier) + (" bla/1" if table is not None else "") + suffix
        p = f.params
        data = fds.encode(Header(cols, p.nx, p.ny, p.ss, p.max_iter, p.escape_radius, f.view, kernel), s)
        if out_dir:
            os.makedirs(out_dir, exist_ok=True)
            with open(os.path.join(out_dir, f"frame_{k:04d}.fds"), "wb") as fh:
                fh.write(data)
        out.append(data)
    return out
