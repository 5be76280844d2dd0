"""The sharded frame through the CUDA route on this GPU: shard.render_frame with
shard.cuda_renderer (fdc_render through the rank's stripe mask) and the NCCL all-gather of
the rank's own rows, in a one-rank NCCL group, equals the route's render of the whole
frame sample for sample, with the same counters. The multi-rank split and gather are the
same code, run with two and three gloo ranks in test_shard_gloo.py."""
import datetime
import os
import socket

import numpy as np
import pytest

import fractodactyl_b200 as fd
from fractodactyl_b200 import _lib, shard

pytestmark = pytest.mark.gpu


def test_sharded_frame_through_the_cuda_route():
    import torch
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    dev = fd.Device(0)
    try:
        v = fd.View("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28")
        p = fd.Params(200, 78, max_iter=30_000, columns=("nu", "de", "normal"))
        plane, tier = fd.route._setup(v, p)
        r, bits = fd.reference(v, p)
        r.bits = bits
        dc, e = fd.bla_dc_bound(v, p)
        bla = fd.Bla.build_scaled(r, fd.EPS, dc, e)
        r, bla = shard.share_reference(r, bla)
        h = dev.upload(r, bla)
        try:
            job = fd.route.make_job(plane, tier, p, h, r.nucleus_period(), _lib.DERIVATIVE | _lib.BLA)
            frame, counters = shard.render_frame(p.nx, p.ny, shard.cuda_renderer(dev, job, p.columns))
            whole, cnt, _ = dev.render_job(job, columns=p.columns)
        finally:
            dev.free(h)
    finally:
        dev.close()
        dist.destroy_process_group()
    for k in ("cls", "n", "nu", "de", "normal", "status"):
        assert np.array_equal(frame[k], whole[k]), k
    assert (counters["samples"], counters["iterations"], counters["blocks"], counters["skipped"]) == (
        cnt.samples, cnt.iterations, cnt.blocks, cnt.skipped)
    assert counters["blocks"] > 0
