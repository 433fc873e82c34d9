"""Sharding of independent systems across ranks (one process per GPU).

Systems of a batch are independent, so a multi-GPU run splits them with no
data-path collective: each rank solves its own shard with the batched
solver, and the only exchange is a host-side gather of the per-system
results."""
from . import shard_lpt


def system_costs(systems, n_rhs):
    """Work estimate per system: stored entries x right-hand sides."""
    return [float(len(A.cols)) * int(r) for A, r in zip(systems, n_rhs)]


def my_shard(systems, n_rhs, rank: int, world: int):
    """System indices this rank solves (LPT on system_costs)."""
    return shard_lpt(system_costs(systems, n_rhs), world)[rank]


def run_sharded(systems, n_rhs, solve, rank: int, world: int, gather=None):
    """solve(indices) -> {system: result} for this rank's shard; gather
    (e.g. torch.distributed.all_gather_object with a list of `world` slots)
    merges the ranks' results.  Returns (indices, merged results)."""
    mine = my_shard(systems, n_rhs, rank, world)
    local = solve(mine)
    if world == 1 or gather is None:
        return mine, dict(local)
    slots = [None] * world
    gather(slots, local)
    merged = {}
    for part in slots:
        merged.update(part)
    return mine, merged
