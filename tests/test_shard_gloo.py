"""Frame and batch sharding over two and three ranks (gloo, CPU), through the same
shard.py code the GPU ranks run: each rank renders only its interleaved stripes (the
oracle's masked render standing in for the per-GPU renderer, shard.cuda_renderer), and the
all-gather of every rank's own rows rebuilds the frame and its counters exactly as one
render of the whole frame, including a ragged last stripe and stripes that do not divide
evenly; a batch's jobs split by static interleave, each job rendered by exactly one rank,
and the counters add up to the whole batch's."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import fdref

VIEW = ("-0.7453", "0.1127", "0.0065", 48, 30, 2000)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from fractodactyl_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        re_, im_, w, nx, ny, it = VIEW
        job = fdref.make_job(re_, im_, w, nx, ny, it, columns=fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL,
                             threads=1)

        def render_masked(mask):
            o = fdref.render_columns(job, mask=mask)  # this rank's samples only, zeros elsewhere
            cols = {k: o[k] for k in ("cls", "n", "nu", "de", "normal")}
            cols["status"] = mask.astype(np.uint8)
            st = o["stats"]
            return cols, {"samples": int(mask.sum()), "iterations": st["iterations"],
                          "closed_form_samples": st["closed_form_samples"], "kernel_ms": 1.0 + rank}

        frame, counters = shard.render_frame(nx, ny, render_masked)
        q.put((rank, {k: v.tolist() for k, v in frame.items()}, counters))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_frame_equals_single_render(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    re_, im_, w, nx, ny, it = VIEW
    o = fdref.render(fdref.make_job(re_, im_, w, nx, ny, it, threads=1), raw=True)
    assert ny % (4 * world) != 0  # stripes that do not divide evenly over the ranks
    for rank, frame, counters in results:
        assert np.array_equal(np.array(frame["cls"], np.uint8), o["cls"])
        assert np.array_equal(np.array(frame["n"], np.uint64), o["n"])
        assert np.array_equal(np.array(frame["nu"]), o["nu"])
        assert np.array_equal(np.array(frame["de"], np.float32), o["de"])
        assert np.array_equal(np.array(frame["normal"], np.uint16), o["normal"])
        assert np.all(np.array(frame["status"], np.uint8) == 1)
        assert counters["samples"] == nx * ny and counters["iterations"] == o["stats"]["iterations"]
        assert counters["closed_form_samples"] == o["stats"]["closed_form_samples"]
        assert counters["kernel_ms"] == float(world)  # the slowest rank's time, not the sum


def test_masks_partition_the_frame():
    from fractodactyl_b200 import shard
    for world in (1, 2, 3, 8):
        m = sum(shard.mask_for(17, 37, r, world).astype(int) for r in range(world))
        assert np.all(m == 1)
        rows = np.concatenate([shard.rows_for(37, r, world) for r in range(world)])
        assert np.array_equal(np.sort(rows), np.arange(37))
        jobs = np.concatenate([shard.jobs_for(11, r, world) for r in range(world)])
        assert np.array_equal(np.sort(jobs), np.arange(11))


BATCH = [("-0.7453", "0.1127", w, 24, 20, 1500) for w in ("0.0065", "1e-5", "3e-8", "1e-11", "2e-13")]


def _batch_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from fractodactyl_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        def run_share(indices):
            cols, it = {}, 0
            for k in indices:
                o = fdref.render(fdref.make_job(*BATCH[k], threads=1))
                cols[k] = o["n"].tolist()
                it += o["stats"]["iterations"]
            return cols, {"jobs": len(indices), "iterations": it}

        cols, counters = shard.render_batch(run_share, len(BATCH))
        q.put((rank, cols, counters))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batch_splits_jobs(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_batch_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [fdref.render(fdref.make_job(*b, threads=1)) for b in BATCH]
    seen = []
    for rank, cols, counters in results:
        assert sorted(cols) == list(range(rank, len(BATCH), world))
        for k, n in cols.items():
            assert np.array_equal(np.array(n, np.uint64), want[k]["n"])
        seen += list(cols)
        assert counters["jobs"] == len(BATCH)
        assert counters["iterations"] == sum(w["stats"]["iterations"] for w in want)
    assert sorted(seen) == list(range(len(BATCH)))


def _share_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import fractodactyl_b200 as fd
    from fractodactyl_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r = bla = None
        if rank == 0:
            v = fd.View("-0.743643887037158704752191506114774", "0.131825904205311970493132056385139", "1e-28")
            p = fd.Params(64, 36, max_iter=20_000, columns=("nu",))
            r, bits = fd.reference(v, p)
            r.bits = bits
            dc, e = fd.bla_dc_bound(v, p)
            bla = fd.Bla.build_scaled(r, 2.0 ** -50, dc, e)
        r, bla = shard.share_reference(r, bla)
        q.put((rank, r.re.tobytes(), r.im.tobytes(), r.bits, bla.blocks.tobytes(), bla.level_offsets.tolist(),
               bla.eps, bla.dc_max, bla.dc_exp))
    finally:
        dist.destroy_process_group()


def test_rank_zero_shares_orbit_and_table():
    """The serial host work runs once: rank 0's orbit and BLA table reach rank 1 bit for bit."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_share_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict((res[0], res[1:]) for res in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == got[1]
    assert len(got[0][3]) > 0 and got[0][2] > 100  # a BLA table and a fixed-point orbit
