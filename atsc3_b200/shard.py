"""FEC blocks over ranks: one process per GPU, no exchange during decode.

FEC blocks are independent codewords (lab/m9_gpu.py:9-11, lab/m3_ldpc.py:
295-299), so a batch of blocks splits into contiguous block ranges, one per
rank, each decoded on its own GPU.  Afterwards only the per-block status (a
few int32 per block) is gathered, and a timed region is the maximum over the
ranks.  The collectives are plain ``torch.distributed`` calls: NCCL between
GPUs, gloo on the CPU.
"""
from __future__ import annotations

STATUS_FIELDS = ("conv", "its", "bad", "ok")


def block_range(nblk, rank, world):
    """Contiguous [lo, hi) of the blocks rank `rank` decodes: the first
    nblk % world ranks take one block more."""
    if world < 1 or not 0 <= rank < world or nblk < 0:
        raise ValueError("bad rank/world/nblk")
    q, r = divmod(nblk, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def gather_status(status, nblk, group=None):
    """All-gather each rank's (hi - lo, 4) int32 status rows (columns
    STATUS_FIELDS) into the (nblk, 4) status of the whole batch, in block
    order, on every rank.  Shards are padded to the largest shard so that the
    collective moves equal sizes."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = block_range(nblk, rank, world)
    if tuple(status.shape) != (hi - lo, len(STATUS_FIELDS)):
        raise ValueError(f"status shape {tuple(status.shape)} != "
                         f"({hi - lo}, {len(STATUS_FIELDS)})")
    width = block_range(nblk, 0, world)[1]
    pad = torch.zeros((width, len(STATUS_FIELDS)), dtype=torch.int32,
                      device=status.device)
    pad[:hi - lo] = status.to(torch.int32)
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    rows = []
    for r in range(world):
        a, b = block_range(nblk, r, world)
        rows.append(parts[r][:b - a])
    return torch.cat(rows)


def max_over_ranks(value, device="cpu", group=None):
    """The maximum of a per-rank float (a timed region in ms) over ranks."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(values, device="cpu", group=None):
    """Element-wise sum of a per-rank list of counts (block errors)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return [float(x) for x in t.tolist()]
