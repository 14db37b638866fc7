"""GPU tests of the beam corner turn (dsax_ct_pack / dsax_ct_unpack) on the
beamformer's own uint8 output, chained into the search-side flagger's data
path, against the oracle restatement of src/dsaX_dbnic.c:84-152 and
src/dsaX_nicdb.c:180-196.  One GPU stands in for the reference's 16
subband nodes (48 channels each, filling channels 128..895 of the 1024) and
its 4 search nodes of 64 beams: the all-to-all between them is a reshuffle of the packed chunks
(its collective is tested on CPU ranks in tests/test_dist_cpu.py).  Byte
moves: bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_corner_turn_beamformer_to_flagger(dsax, oracle):
    import torch
    nsub, ndest, nbeam, npkt, ppo, nchan = 16, 4, 256, 512, 4, 384
    nt, nc, nbl = npkt // ppo, nchan // 8, nbeam // ndest
    fil_nt, fil_nc, ch0 = 2 * nt, 1024, 128
    wre, wim = oracle.random_phase_weights(3, nc, nbeam)
    cfg = dsax.default_config(npkt=npkt, nant_in=63, nchan=nchan, nbeam=nbeam,
                              bf_pkt_per_out=ppo, bf_scale=128.0 / (2 * ppo * 16 * 64 * 2 * 6.25))
    fil = [torch.zeros(nbl * fil_nt * fil_nc, dtype=torch.uint8, device="cuda")
           for _ in range(ndest)]
    want = [np.zeros((nbl, fil_nt, fil_nc), np.uint8) for _ in range(ndest)]
    with dsax.Context(cfg) as ctx:
        ctx.set_weights(wre, wim)
        for tblk in range(2):                     # two consecutive beam blocks in time
            sends, beams_h = [], []
            for s in range(nsub):
                blk = oracle.gen_block(900 + 10 * tblk + s, npkt, 63, nchan, "gauss")
                d = torch.from_numpy(blk.reshape(-1)).cuda()
                beams = torch.empty(nt * nbeam * nc, dtype=torch.uint8, device="cuda")
                send = torch.empty_like(beams)
                torch.cuda.synchronize()
                ctx.beamform(d, beams, None)
                ctx.ct_pack(beams, nt, nbeam, nc, ndest, send)
                ctx.sync()
                sends.append(send.view(ndest, nbl * nt * nc))
                beams_h.append(beams.cpu().numpy().reshape(nt, nbeam, nc))
                np.testing.assert_array_equal(send.cpu().numpy().reshape(ndest, nbl, nt, nc),
                                              oracle.ct_pack(beams_h[-1], ndest))
            for dst in range(ndest):              # the all-to-all, on one GPU
                recv = torch.stack([sends[s][dst] for s in range(nsub)]).contiguous()
                ctx.ct_unpack(recv, nsub, nbl, nt, nc, fil[dst], fil_nt, fil_nc, tblk * nt, ch0)
                oracle.ct_unpack(np.stack([oracle.ct_pack(b, ndest)[dst] for b in beams_h]),
                                 want[dst], tblk * nt, ch0)
        ctx.sync()
        got = [f.cpu().numpy().reshape(nbl, fil_nt, fil_nc) for f in fil]
    for dst in range(ndest):
        np.testing.assert_array_equal(got[dst], want[dst])
    assert got[1][:, :, ch0:ch0 + nsub * nc].any() and not got[1][:, :, :ch0].any()
    assert ch0 + nsub * nc == fil_nc - ch0          # the guard bands are the unfilled channels
    # the search GPU's flagger on the assembled filterbank (uint8 data path,
    # guard band = the unfilled channels), with a saved baseline
    p = dsax.flag_params(nbl, fil_nt, fil_nc, guard=ch0, ts_base=64)
    x = got[2]
    s0 = np.full((nbl, fil_nc), float(np.median(x[:, :, ch0:ch0 + nsub * nc])), np.float32)
    v0 = np.full((nbl, fil_nc), 16.0, np.float32)
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        with ctx.flag_state(p, dsax.flag_clean_params(), dsax.DTYPE_U8) as st:
            st.set_baseline(s0, v0)
            out = x.copy()
            cm = np.zeros((nbl, fil_nc), np.uint8)
            tm = np.zeros((nbl, fil_nt), np.uint8)
            st.clean(out, cm, tm, mem=dsax.MEM_HOST)
    ocl = oracle.CleanOracle(p, dtype=np.uint8)
    ocl.spec0, ocl.var0, ocl.started = s0, v0, True
    ow, ocm, otm, _, (cmg, tmg) = ocl.step(x)
    sure_c, sure_t = cmg > 1e-4, tmg > 1e-4
    np.testing.assert_array_equal(cm[sure_c], ocm[sure_c])
    np.testing.assert_array_equal(tm[sure_t], otm[sure_t])
    if sure_c.all() and sure_t.all():
        np.testing.assert_array_equal(out, ow)
