"""Process-level parallelism: one process per GPU, torch.distributed for
the plumbing.

A single grid fits one GPU, so a multi-GPU job is either replicas of one run
(the throughput benchmark) or a set of independent runs sharded across the
ranks (a constant-k sweep, a population of designs): the reference's
process-level fan-out (utility_scripts/parallel_kmax.py) with no data-path
collective.  The only collectives are a barrier and a max or gather of a few
host numbers at the end.
"""


def shard(items, rank, world):
    """The items rank `rank` of `world` runs: every world-th, from rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of world %d" % (rank, world))
    return list(items)[rank::world]


def max_over_ranks(x, group=None, device=None):
    """max of a host float over the ranks (the job time of replicas that
    started together); x itself without an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_results(values, group=None):
    """Every rank's list of small picklable results, on all ranks, as a list
    of per-rank lists in rank order (end-of-run gather of a sharded sweep;
    unshard puts them back in item order)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [list(values)]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, list(values), group=group)
    return out


def unshard(parts, world):
    """Inverse of shard: the rank-ordered concatenation of every rank's
    shard (as gather_results returns it) back in item order."""
    n = sum(len(p) for p in parts)
    out = [None] * n
    for r, p in enumerate(parts):
        for q, v in enumerate(p):
            out[r + q * world] = v
    return out
