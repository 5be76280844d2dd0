"""One frame over several GPUs (one process per GPU, torch.distributed).

Samples are independent and the orbit and BLA table are small, so the frame shards with
no exchange during rendering: rank r of W takes the 4-row stripes s with s % W == r (the
kernel's tiles are 4 rows high; interleaving spreads the costly centre of a deep frame
over all ranks), renders them with a sample mask, and one reduction of the columns
(every sample is rendered by exactly one rank, zeros elsewhere) gathers the frame. The
counters are summed the same way; frame time is the max over ranks. The reference orbit
and BLA table are serial host work (the orbit is up to 2^20 fixed-point steps): rank 0
computes them and share_reference broadcasts them to the other ranks (NCCL over NVLink
for GPU groups, gloo on the CPU).
"""
from typing import Callable, Dict

import numpy as np

STRIPE = 4
COLUMNS = ("cls", "n", "nu", "de", "normal")
# exact integer or float carriers for the sum-reduction of each column
CARRIER = {"cls": np.int32, "n": np.int64, "nu": np.float64, "de": np.float64, "normal": np.int32}
OUT = {"cls": np.uint8, "n": np.uint32, "nu": np.float64, "de": np.float32, "normal": np.uint16}


def mask_for(nx: int, ny: int, rank: int, world: int) -> np.ndarray:
    """Sample mask (row-major, nx*ny bytes) of the rows this rank renders."""
    rows = (np.arange(ny) // STRIPE) % world == rank
    return np.repeat(rows.astype(np.uint8), nx)


def combine(parts: Dict[str, np.ndarray], group=None) -> Dict[str, np.ndarray]:
    """Sum-reduce each rank's columns (zeros where it rendered nothing) onto every rank."""
    import torch
    import torch.distributed as dist
    out = {}
    for name, arr in parts.items():
        t = torch.from_numpy(np.ascontiguousarray(arr, dtype=CARRIER[name]))
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out[name] = t.cpu().numpy().astype(OUT[name])
    return out


def render_frame(nx: int, ny: int, render_masked: Callable[[np.ndarray], Dict], group=None):
    """Render one frame across the group: render_masked(mask) returns this rank's columns
    (full-size arrays, only masked samples written) and a dict of counters."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    cols, counters = render_masked(mask_for(nx, ny, rank, world))
    frame = combine({k: v for k, v in cols.items() if k in COLUMNS and v is not None}, group)
    keys = sorted(counters)
    t = torch.tensor([float(counters[k]) for k in keys], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return frame, {k: v for k, v in zip(keys, t.cpu().tolist())}


def share_reference(r=None, bla=None, group=None, src: int = 0):
    """Broadcast rank `src`'s reference orbit (and BLA table, if any) to every rank of the
    group; other ranks pass None and receive equal copies (the same f64 bits)."""
    import torch
    import torch.distributed as dist

    from .route import Bla, Reference
    rank = dist.get_rank(group)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
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
