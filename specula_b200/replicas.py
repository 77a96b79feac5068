"""Running independent systems on several GPUs (one process per GPU).

The closed loop of one SCAO system is a sequential chain with no data
exchange worth sharding, so multi-GPU runs are replicas. ``bench.py --gpus
N`` runs one ELT loop per rank. The Monte-Carlo mix is a fixed set of
realisations split across the ranks: every rank steps its own share of
every geometry group with no data-path collective. The only collectives are
a barrier, the max of the ranks' timings, and an all-gather of per-rank
results on the host.

Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU).
"""
import torch
import torch.distributed as dist


def world():
    """(rank, world_size); (0, 1) without an initialised process group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def partition(n, world_size, rank):
    """Contiguous, balanced slice of range(n) for ``rank``: the first
    n % world_size ranks get one extra item."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f'rank {rank} outside a world of {world_size}')
    q, r = divmod(int(n), world_size)
    lo = rank * q + min(rank, r)
    return range(lo, lo + q + (1 if rank < r else 0))


def shard_groups(groups, world_size, rank):
    """Split every geometry group's realisations across the ranks, so each
    rank gets a balanced share of each geometry.  ``groups``: list of
    (template, [realisation configs]).  Groups left empty on this rank are
    dropped."""
    out = []
    for tmpl, reals in groups:
        mine = [reals[i] for i in partition(len(reals), world_size, rank)]
        if mine:
            out.append((tmpl, mine))
    return out


def max_over_ranks(value, device=None):
    """The largest ``value`` over all ranks (a timing: the job ends with its
    slowest rank)."""
    rank, ws = world()
    if ws == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    rank, ws = world()
    if ws == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_objects(obj):
    """Every rank's ``obj`` (picklable), in rank order, on every rank."""
    rank, ws = world()
    if ws == 1:
        return [obj]
    out = [None] * ws
    dist.all_gather_object(out, obj)
    return out
