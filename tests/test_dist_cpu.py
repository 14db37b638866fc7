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


def _ct_worker(rank, world_size, port, out):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "dsa110-xengine_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world_size), LOCAL_RANK=str(rank))
    import numpy as np
    import torch
    from dsax import dist as D
    d = D.init("gloo", timeout_s=60)
    T, NB, C = 6, 8, 3
    # subband `rank`: value encodes (t, beam, global channel)
    loc = np.zeros((T, NB, C), np.int64)
    for t in range(T):
        for b in range(NB):
            for c in range(C):
                loc[t, b, c] = (t * 1000 + b) * 100 + rank * C + c
    got = D.corner_turn_beams(torch.from_numpy(loc))
    d.barrier()
    d.destroy_process_group()
    out.put((rank, got.numpy()))


def test_beam_corner_turn_all_to_all_gloo():
    """World size 2: each rank ends with its half of the beams, all times,
    and the channels of both subbands in rank order."""
    import numpy as np
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ct_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    T, NB, C, W = 6, 8, 3, 2
    for r in range(W):
        got = res[r]
        assert got.shape == (NB // W, T, W * C)
        for bl in range(NB // W):
            for t in range(T):
                for ch in range(W * C):
                    assert got[bl, t, ch] == (t * 1000 + r * (NB // W) + bl) * 100 + ch


def _ct_chain_worker(rank, world_size, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "dsa110-xengine_b200"), os.path.join(root, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world_size), LOCAL_RANK=str(rank))
    import numpy as np
    import torch
    import oracle
    from dsax import dist as D
    d = D.init("gloo", timeout_s=60)
    W = world_size
    T, NB, C, fil_nc, ch0 = 8, 16, 48, 256, 32
    rng = np.random.default_rng(100 + rank)
    beams = rng.integers(0, 256, (T, NB, C), dtype=np.uint8)   # this subband's beamformer output
    # the exchange beam_corner_turn performs around its two device reorders:
    # pack per destination, one all-to-all, place by source rank
    send = torch.from_numpy(oracle.ct_pack(beams, W).reshape(-1).copy())
    recv = torch.empty_like(send)
    d.all_to_all_single(recv, send)
    fil = np.zeros((NB // W, T, fil_nc), np.uint8)
    oracle.ct_unpack(recv.numpy().reshape(W, NB // W, T, C), fil, 0, ch0)
    d.barrier()
    d.destroy_process_group()
    out.put((rank, beams, fil))


def test_beam_corner_turn_pack_exchange_place_gloo():
    """World size 2, the beam corner turn's three steps (dbnic's pack, the
    all-to-all, nicdb's placement at channel ch0 + subband x C): rank r's
    filterbank holds beams r NB/W .. of every rank's subband, channels in
    rank order, guard bands empty."""
    import numpy as np
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ct_chain_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {r: (b, f) for r, b, f in (q.get(timeout=120) for _ in procs)}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    W, T, NB, C, ch0 = 2, 8, 16, 48, 32
    for r in range(W):
        fil = res[r][1]
        for s in range(W):
            np.testing.assert_array_equal(fil[:, :, ch0 + s * C:ch0 + (s + 1) * C],
                                          res[s][0][:, r * NB // W:(r + 1) * NB // W, :]
                                          .transpose(1, 0, 2))
        assert not fil[:, :, :ch0].any() and not fil[:, :, ch0 + W * C:].any()
