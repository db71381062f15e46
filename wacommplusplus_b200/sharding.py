"""Particles sharded over GPUs, one process per GPU.

Particle updates are independent and keyed by each particle's own id, so every rank moves its own
contiguous shard on its own GPU with no data-path exchange. The reference hands each process and
each GPU a contiguous section, the first one taking the remainder
(NumericalHelpers.hpp:76-82, Wacomm.cpp:276-300 and 540-545); `partition_count` and
`partition_offset` restate that split.

The one exchange step is the concentration grid: the reference gathers every particle on rank 0
each interval and counts there (Wacomm.cpp:700-722). Here each rank counts its own shard in the
move kernel's epilogue and the per-interval grid slice (s_rho x eta x xi uint32 counts) is summed
across ranks with one all-reduce. The counts are reduced through a signed 32-bit view: addition
modulo 2^32 gives the same bits for signed and unsigned operands, so the result is the uint32 sum
exactly, even past 2^31.
"""


def partition_count(total, workers, worker):
    """Particles of `worker` out of `total` split over `workers`; worker 0 takes the remainder."""
    return total // workers + (total % workers if worker == 0 else 0)


def partition_offset(total, workers, worker):
    """First particle of `worker`'s contiguous section."""
    return 0 if worker == 0 else partition_count(total, workers, 0) + (worker - 1) * (total // workers)


def shard(records, rank, world):
    """The contiguous section of `records` that rank `rank` of `world` moves."""
    start = partition_offset(len(records), world, rank)
    return records[start:start + partition_count(len(records), world, rank)]


def reduce_counts(counts, group=None):
    """Sums a count tensor (int32 view of uint32 counts, any device) over the ranks of `group`, in
    place, and returns it."""
    import torch
    import torch.distributed as dist
    if counts.dtype != torch.int32:
        raise TypeError(f"counts must be an int32 view of the uint32 grid, not {counts.dtype}")
    if dist.is_initialized():
        dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    return counts


def allreduce_concentration(engine, conc_time_index, group=None):
    """Sums time slice `conc_time_index` of the engine's concentration grid over the ranks of
    `group` on the engine's own stream, so that it follows the kernels that counted it."""
    import torch
    view = engine.concentration_view(conc_time_index)
    stream = torch.cuda.ExternalStream(engine.stream, device=view.device)
    with torch.cuda.stream(stream):
        reduce_counts(view, group)
    return view
