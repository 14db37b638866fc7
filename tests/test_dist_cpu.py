"""The N > 1 benchmark plumbing on CPU: world size 2 over gloo -- block
sharding covers every block exactly once, and the step time is the max over
ranks."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world_size, port, nblocks, out):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "dsa110-xengine_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world_size), LOCAL_RANK=str(rank))
    from dsax import dist as D
    ws, r, _ = D.world()
    d = D.init("gloo", timeout_s=60)
    mine = list(D.shard(nblocks, r, ws))
    fake_ms = 10.0 + 5.0 * r          # rank 1 is the slow one
    d.barrier()
    worst = D.max_over_ranks(fake_ms)
    gathered = [None] * ws
    d.all_gather_object(gathered, mine)
    d.barrier()
    d.destroy_process_group()
    out.put((r, worst, gathered))


@pytest.mark.parametrize("nblocks", [16, 7])
def test_shard_and_max_over_ranks_gloo(nblocks):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, nblocks, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, worst, gathered in res:
        assert worst == 15.0
        flat = sorted(i for part in gathered for i in part)
        assert flat == list(range(nblocks))
        assert abs(len(gathered[0]) - len(gathered[1])) <= 1
