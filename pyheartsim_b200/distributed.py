"""Instance-parallel execution over several GPUs (one process per GPU).

Simulation instances are independent, so the path shards by instance with no
data-path collective: each rank advances its own instances; the host gathers
results.  Two ways to split work:

* weak scaling: every rank builds its own batch (seeds offset by rank);
* ``shard``: one global list of instances is split by a greedy bin-packing of
  their cost (voxels x steps), largest first onto the least-loaded rank.

The only collectives are the benchmark's barrier, the MAX of the timed window
and the host-side gather of per-rank results (``gather``).
"""
import torch
import torch.distributed as dist


def shard(costs, world):
    """Greedy longest-processing-time split: returns a list of index lists."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def max_over_ranks(x, device=None):
    """MAX of a float over all ranks (identity without a process group)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather(obj, dst=0):
    """Host-side gather of a picklable per-rank result onto ``dst``."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(obj, out, dst=dst)
    return out
