"""Multi-GPU host logic: one process per GPU, no collective on the data path.

A single case does not shard (the reference's hot path runs one case per
device here), so N GPUs run N replicas; independent cases (batches of
uneven grids) are split across ranks by a balanced partition of their cell
counts.  torch.distributed carries only the plumbing: a barrier around the
timed region, the max over ranks of the device time and the gather of
per-case results.
"""
import datetime
import os


def env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=120):
    """Initialise the process group when WORLD_SIZE > 1; returns the
    torch.distributed module or None."""
    ws, rank, local = env()
    if ws <= 1:
        return None
    import torch
    import torch.distributed as dist
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def balanced_shards(costs, nranks):
    """Longest-processing-time partition of case indices over ranks: cases
    sorted by decreasing cost, each to the currently least-loaded rank.
    Returns a list of index lists, one per rank (deterministic)."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    load = [0.0] * nranks
    shards = [[] for _ in range(nranks)]
    for idx in sorted(range(len(costs)), key=lambda q: (-costs[q], q)):
        r = min(range(nranks), key=lambda q: (load[q], q))
        shards[r].append(idx)
        load[r] += costs[idx]
    return [sorted(s) for s in shards]


def max_over_ranks(dist, value, device=None):
    """Max of a float over all ranks (value itself without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(dist, local_results):
    """Merge {case_index: result} dicts of every rank on every rank."""
    if dist is None:
        return dict(local_results)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, dict(local_results))
    merged = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError("case %r computed on two ranks" % (k,))
            merged[k] = v
    return merged


def run_sharded(dist, costs, run_case, rank=None, world_size=None):
    """Run run_case(index) for this rank's shard of the cases; returns the
    merged results of all ranks and this rank's shard."""
    ws = world_size if world_size is not None else (dist.get_world_size() if dist else 1)
    rk = rank if rank is not None else (dist.get_rank() if dist else 0)
    shard = balanced_shards(costs, ws)[rk]
    local = {idx: run_case(idx) for idx in shard}
    return gather_results(dist, local), shard


def run_sharded_batch(dist, costs, run_batch, rank=None, world_size=None, device=None):
    """Run run_batch(indices) once on this rank's shard of the cases (the
    shard advances together, e.g. through pvof_run_steps_batched); run_batch
    returns ({index: result}, seconds) for exactly those indices.  Returns the
    merged results of all ranks, this rank's shard and the max over ranks of
    the seconds.  Every rank calls it once (it holds collectives)."""
    ws = world_size if world_size is not None else (dist.get_world_size() if dist else 1)
    rk = rank if rank is not None else (dist.get_rank() if dist else 0)
    shard = balanced_shards(costs, ws)[rk]
    local, secs = run_batch(shard)
    if sorted(local) != sorted(shard):
        raise RuntimeError("run_batch returned cases %r for the shard %r" % (sorted(local), shard))
    return gather_results(dist, local), shard, max_over_ranks(dist, secs, device=device)
