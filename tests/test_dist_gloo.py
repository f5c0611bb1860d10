"""Multi-rank host logic on CPU: two gloo ranks split a batch of uneven
cases, every case runs exactly once, and the max over ranks is taken."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, out_dir):
    import datetime
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(repo, "parties-vof-ibm_b200"))
    import torch.distributed as dist
    from pvof import dist as pdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    # each "case" returns (index, rank, a value derived from its cost)
    merged, shard = pdist.run_sharded(dist, costs, lambda q: (q, rank, costs[q] * 2.0))
    t = pdist.max_over_ranks(dist, float(sum(costs[q] for q in shard)))
    with open(os.path.join(out_dir, "r%d.txt" % rank), "w") as f:
        f.write(repr((sorted(merged.items()), shard, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_balanced_shards_cover_each_case_once():
    from pvof.dist import balanced_shards
    costs = [8192, 524288, 65536, 131072, 16384, 262144, 32768, 8192, 131072]
    for n in (1, 2, 3, 8):
        shards = balanced_shards(costs, n)
        flat = sorted(q for s in shards for q in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[q] for q in s) for s in shards]
        assert max(loads) <= max(costs) + sum(costs) / n


def test_two_gloo_ranks_split_and_gather(tmp_path):
    import torch.multiprocessing as mp
    costs = [5.0, 1.0, 3.0, 8.0, 2.0, 2.0, 7.0]
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, costs, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    import ast
    r0 = ast.literal_eval(open(tmp_path / "r0.txt").read())
    r1 = ast.literal_eval(open(tmp_path / "r1.txt").read())
    merged0, shard0, t0 = r0
    merged1, shard1, t1 = r1
    assert merged0 == merged1
    assert [k for k, _ in merged0] == list(range(len(costs)))
    assert sorted(shard0 + shard1) == list(range(len(costs)))
    for k, (q, rank, v) in merged0:
        assert q == k and v == costs[k] * 2.0 and (k in (shard0 if rank == 0 else shard1))
    assert t0 == t1 == max(sum(costs[q] for q in shard0), sum(costs[q] for q in shard1))


def _batch_worker(rank, world, port, n, out_dir):
    import datetime
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(repo, "parties-vof-ibm_b200"))
    import torch.distributed as dist
    from pvof import cases
    from pvof import dist as pdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    allc = cases.droplet_batch(n, seed=3, nxm_max=128)
    costs = [float(g.NXM * g.NYM) for g, _, _, _ in allc]

    def run_batch(idx):
        # the bench's shard set-up on the host: each case's grid, particles
        # and initial liquid volume; "seconds" stands for the shard's cells
        res = {q: (allc[q][0].NXM, allc[q][3][0][3], float(allc[q][2]["F"].sum())) for q in idx}
        return res, sum(costs[q] for q in idx)

    merged, shard, secs = pdist.run_sharded_batch(dist, costs, run_batch)
    with open(os.path.join(out_dir, "b%d.txt" % rank), "w") as f:
        f.write(repr((sorted(merged.items()), shard, secs)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_droplet_batch(tmp_path):
    """The batching form's cases (pvof.cases.droplet_batch) split over two
    gloo ranks by pvof.dist.run_sharded_batch, as bench.py --droplets does:
    every case set up on exactly one rank, both ranks hold the same merged
    results, equal to a single process's, and the time is the max over
    ranks."""
    import ast
    import torch.multiprocessing as mp
    from pvof import cases
    from pvof.dist import balanced_shards
    n = 10
    port = _free_port()
    mp.start_processes(_batch_worker, args=(2, port, n, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    b0 = ast.literal_eval(open(tmp_path / "b0.txt").read())
    b1 = ast.literal_eval(open(tmp_path / "b1.txt").read())
    assert b0[0] == b1[0]
    assert sorted(b0[1] + b1[1]) == list(range(n))
    allc = cases.droplet_batch(n, seed=3, nxm_max=128)
    costs = [float(g.NXM * g.NYM) for g, _, _, _ in allc]
    assert [b0[1], b1[1]] == balanced_shards(costs, 2)
    single = sorted({q: (allc[q][0].NXM, allc[q][3][0][3], float(allc[q][2]["F"].sum())) for q in range(n)}.items())
    assert b0[0] == single
    assert b0[2] == b1[2] == max(sum(costs[q] for q in b0[1]), sum(costs[q] for q in b1[1]))
