"""Frames and batches over several GPUs (one process per GPU, torch.distributed).

Samples are independent and the orbit and BLA table are small, so the work shards with no
exchange during rendering.

- One frame: rank r of W takes the 4-row stripes s with s % W == r (the kernel's tiles are
  4 rows high; interleaving spreads the costly centre of a deep frame over all ranks) and
  renders them through a sample mask. Each rank then contributes only the rows it
  rendered: one all-gather per column of every rank's own rows (padded to the largest
  share), so a rank sends 1/W of the frame, not all of it. Counters are summed with one
  all-reduce; frame time is the max over ranks.
- A batch (a film's frames, a tile set): job k goes to rank k % W (static interleave),
  each rank runs its jobs as one batch, and the counters are summed the same way.

The reference orbit and BLA table are serial host work (up to 2^20 fixed-point steps):
rank 0 computes them and share_reference broadcasts them to the other ranks (NCCL over
NVLink for GPU groups, gloo on the CPU).
"""
from typing import Callable, Dict, List, Sequence

import numpy as np

STRIPE = 4
COLUMNS = ("cls", "n", "nu", "de", "normal", "status")
HOST = {"cls": np.uint8, "n": np.uint32, "nu": np.float64, "de": np.float32, "normal": np.uint16, "status": np.uint8}


def rows_for(ny: int, rank: int, world: int) -> np.ndarray:
    """The rows rank `rank` of `world` renders: the 4-row stripes s with s % world == rank."""
    rows = np.arange(ny)
    return rows[(rows // STRIPE) % world == rank]


def mask_for(nx: int, ny: int, rank: int, world: int) -> np.ndarray:
    """Sample mask (row-major, nx*ny bytes) of the rows this rank renders."""
    m = np.zeros(ny, np.uint8)
    m[rows_for(ny, rank, world)] = 1
    return np.repeat(m, nx)


def _on_device(group) -> bool:
    import torch.distributed as dist
    return dist.get_backend(group) == "nccl"


def gather_rows(nx: int, ny: int, cols: Dict[str, np.ndarray], group=None) -> Dict[str, np.ndarray]:
    """Every rank's own rows of each column (full-frame arrays, the rank's rows written)
    into the whole frame on every rank: one all-gather per column of rows_for's rows,
    padded to the largest share. Columns travel as their bytes (every backend carries
    uint8), so each value arrives with the same bits."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    share = max(len(rows_for(ny, r, world)) for r in range(world))
    mine = rows_for(ny, rank, world)
    dev = "cuda" if _on_device(group) else "cpu"
    out = {}
    for name, arr in cols.items():
        frame = np.asarray(arr).reshape(ny, nx)
        send = np.zeros((share, nx), HOST[name])
        send[:len(mine)] = frame[mine]
        t = torch.from_numpy(send.view(np.uint8)).to(dev)
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        whole = np.zeros((ny, nx), HOST[name])
        for r, part in enumerate(parts):
            rows = rows_for(ny, r, world)
            whole[rows] = part.cpu().numpy().view(HOST[name])[:len(rows)]
        out[name] = whole.reshape(-1)
    return out


def sum_counters(counters: Dict[str, float], group=None, maxed: Sequence[str] = ("kernel_ms",)) -> Dict[str, float]:
    """Each counter summed over the ranks, those named in `maxed` (times: the group's
    frame time is its slowest rank's) taken as the maximum: two all-reduces, the same key
    order on every rank."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if _on_device(group) else "cpu"
    out = {}
    for op, keys in ((dist.ReduceOp.SUM, sorted(k for k in counters if k not in maxed)),
                     (dist.ReduceOp.MAX, sorted(k for k in counters if k in maxed))):
        t = torch.tensor([float(counters[k]) for k in keys] or [0.0], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op, group=group)
        out.update(zip(keys, t.cpu().tolist()))
    return out


def render_frame(nx: int, ny: int, render_masked: Callable[[np.ndarray], tuple], group=None):
    """Render one frame across the group: render_masked(mask) returns this rank's columns
    (full-size arrays, only masked samples written) and a dict of counters. Returns the
    whole frame's columns and the summed counters on every rank."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    cols, counters = render_masked(mask_for(nx, ny, rank, world))
    frame = gather_rows(nx, ny, {k: v for k, v in cols.items() if k in COLUMNS and v is not None}, group)
    return frame, sum_counters(counters, group)


def cuda_renderer(dev, job, columns=("nu", "de", "normal")):
    """render_masked for render_frame on this rank's GPU: the route's job (an uploaded
    orbit, fdc_job fields set) rendered through the rank's sample mask by fdc_render, into
    host columns. Counters: samples, iterations, blocks, skipped, kernel_ms, launches."""
    import ctypes as C

    from . import _lib

    def render_masked(mask: np.ndarray):
        j = _lib.Job()
        C.memmove(C.byref(j), C.byref(job), C.sizeof(_lib.Job))
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        j.mask = m.ctypes.data
        arrays, cnt, _ = dev.render_job(j, columns=columns)
        return arrays, {"samples": cnt.samples, "iterations": cnt.iterations, "blocks": cnt.blocks,
                        "skipped": cnt.skipped, "kernel_ms": cnt.kernel_ms, "launches": cnt.launches}

    return render_masked


def jobs_for(njobs: int, rank: int, world: int) -> List[int]:
    """The jobs of a batch rank `rank` runs: job k goes to rank k % world (a film's frames
    or a tile set's tiles, interleaved so that deep and shallow work spreads evenly)."""
    return list(range(rank, njobs, world))


def render_batch(run_share: Callable[[List[int]], tuple], njobs: int, group=None):
    """One batch across the group: run_share(indices) runs this rank's jobs (jobs_for) and
    returns {job index: columns} and a dict of counters. Returns this rank's columns and
    the counters summed over the ranks (the frames stay on the rank that rendered them)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    cols, counters = run_share(jobs_for(njobs, rank, world))
    return cols, sum_counters(counters, group)


def share_reference(r=None, bla=None, group=None, src: int = 0):
    """Broadcast rank `src`'s reference orbit (and BLA table, if any) to every rank of the
    group; other ranks pass None and receive equal copies (the same f64 bits)."""
    import torch
    import torch.distributed as dist

    from .route import Bla, Reference
    rank = dist.get_rank(group)
    dev = "cuda" if _on_device(group) else "cpu"
    # header: orbit length, bits, table present, level count, block count, dc_exp, eps, dc_max
    hdr = torch.zeros(8, dtype=torch.float64, device=dev)
    if rank == src:
        levels = bla.levels if bla is not None else 0
        nblocks = len(bla.blocks) if bla is not None else 0
        hdr[:] = torch.tensor([len(r.re), r.bits, float(bla is not None), levels, nblocks,
                               bla.dc_exp if bla is not None else 0, bla.eps if bla is not None else 0.0,
                               bla.dc_max if bla is not None else 0.0], dtype=torch.float64)
    dist.broadcast(hdr, src, group=group)
    n, bits, has, levels, nblocks, dc_exp = (int(v) for v in hdr[:6].tolist())
    eps, dc_max = float(hdr[6]), float(hdr[7])

    def cast(arr, shape, dtype):
        t = torch.from_numpy(np.ascontiguousarray(arr)).to(dev) if rank == src else \
            torch.empty(shape, dtype=dtype, device=dev)
        dist.broadcast(t, src, group=group)
        return t.cpu().numpy()

    z = cast(np.stack([r.re, r.im]) if rank == src else None, (2, n), torch.float64)
    ref = r if rank == src else Reference(z[0].copy(), z[1].copy(), bits)
    table = bla
    if has:  # every rank takes part in each broadcast
        blocks = cast(bla.blocks if rank == src else None, (nblocks, 7), torch.float64)
        offs = cast(bla.level_offsets.astype(np.int64) if rank == src else None, (levels + 1,), torch.int64)
        if rank != src:
            table = Bla(blocks, offs.astype(np.uint64), eps, dc_max, dc_exp, n)
    return ref, (table if has else None)
