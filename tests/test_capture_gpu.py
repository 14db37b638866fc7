"""Packet capture -> block assembly on the GPU (dsax_place_packets,
src/dsaX_capture.c receive_obs :870-960) against the oracle's restatement:
shuffled packets, some late, some for the next block, some beyond it and
some from unknown antennas; blocks and counters identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_place_packets_matches_oracle(dsax, oracle):
    import torch
    rng = np.random.default_rng(31)
    payload, stride, sps = 4608, 4616, 8
    nslots = 6 * sps                  # block of 6 sequence numbers x 8 slots
    seq0 = 1000
    lookup = -np.ones(64, np.int32)
    ant_ids = rng.choice(64, size=sps, replace=False)
    lookup[ant_ids] = np.arange(sps)
    pk = []
    for seq in range(seq0 - 2, seq0 + 14):           # late, current, next, beyond
        for aid in range(sps):
            pk.append(oracle.packet_header(seq, int(rng.integers(8192)), int(ant_ids[aid])) +
                      rng.integers(0, 256, payload, dtype=np.uint8).tobytes())
    for _ in range(5):                               # unknown antennas
        bad = int(np.flatnonzero(lookup < 0)[0])
        pk.append(oracle.packet_header(seq0, 0, bad) + bytes(payload))
    order = rng.permutation(len(pk))
    pkts = b"".join(pk[i] for i in order)
    act0 = seq0 * sps
    want_b, want_n, want_c = oracle.place_packets(pkts, stride, payload, lookup, act0, nslots, sps)
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        d_p = torch.frombuffer(bytearray(pkts), dtype=torch.uint8).cuda()
        d_l = torch.from_numpy(lookup).cuda()
        blk = torch.zeros(nslots * payload, dtype=torch.uint8, device="cuda")
        nxt = torch.zeros(nslots * payload, dtype=torch.uint8, device="cuda")
        cnt = torch.zeros(4, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        ctx.place_packets(d_p, len(pk), stride, payload, d_l, act0, nslots, sps, blk, cnt,
                          next_block=nxt)
        ctx.sync()
        assert cnt.cpu().tolist() == want_c
        assert blk.cpu().numpy().tobytes() == want_b
        assert nxt.cpu().numpy().tobytes() == want_n
    assert want_c[0] == nslots and want_c[1] == nslots and want_c[2] == 2 * sps
