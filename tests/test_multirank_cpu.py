"""Multi-process path of bench.py on CPU: world_size 2 over gloo.  Ranks take
disjoint batches of the sweep (no data exchange) and the step time is the
max over ranks."""
import os


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from openrcwa_b200 import workloads
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    B = 8
    mine = [list(range(workloads.shard_start(rank, world, B, k), workloads.shard_start(rank, world, B, k) + B))
            for k in range(3)]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    t = torch.tensor([1.0 + rank])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    q.put((rank, gathered, float(t)))
    dist.destroy_process_group()


def test_two_rank_sharding_over_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, 29511, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=180) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    for rank, gathered, tmax in res:
        assert tmax == 2.0
        idx = [i for per_rank in gathered for batch in per_rank for i in batch]
        assert len(idx) == len(set(idx)) == 2 * 3 * 8
