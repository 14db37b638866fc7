"""GPU tests of the plain flagger through the C-ABI against the oracle.
Masks are index work: they must be identical, except where the oracle's
decision margin |stat - threshold| / MAD is below 1e-4 (a last-bit
difference in an FP32 statistic could flip those; none are expected)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
MARGIN = 1e-4


def _gpu_flag(dsax, x, params, oldspec=None):
    B, T, C = x.shape
    cm = np.zeros((B, C), np.uint8)
    tm = np.zeros((B, T), np.uint8)
    st = np.zeros(4 * B * C + B * T, np.float32)
    cnt = np.zeros(2, np.int32)
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        ctx.flag(params, np.ascontiguousarray(x), cm, tm, oldspec=oldspec, stats=st, counts=cnt,
                 mem=dsax.MEM_HOST)
    return cm, tm, st, cnt


def _compare(dsax, oracle, x, parity=0, oldspec=None, **kw):
    B, T, C = x.shape
    pd = dsax.flag_params(B, T, C, parity=parity, **kw)
    po = oracle.flag_params(B, T, C, guard=pd.guard, filt=pd.filt, tbin=pd.tbin, fbin=pd.fbin,
                            ts_base=pd.ts_base, tsflag=pd.tsflag, parity=parity,
                            thresh=pd.thresh, var_add=pd.var_add, ts_thresh=pd.ts_thresh,
                            perm=list(pd.perm)[:pd.nperm])
    cm, tm, st, cnt = _gpu_flag(dsax, x, pd, oldspec)
    ocm, otm, cmg, tmg, ost = oracle.plain_flag(x, po, oldspec)
    bc = B * C
    np.testing.assert_allclose(st[:bc].reshape(B, C), ost["spec"], rtol=1e-6)
    np.testing.assert_allclose(st[bc:2 * bc].reshape(B, C), ost["var"], rtol=1e-5)
    np.testing.assert_array_equal(st[2 * bc:3 * bc].reshape(B, C), ost["max"]) if not parity else None
    np.testing.assert_allclose(st[3 * bc:4 * bc].reshape(B, C), ost["pp"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(st[4 * bc:].reshape(B, T), ost["ts"], rtol=1e-6)
    sure_c = cmg > MARGIN
    sure_t = tmg > MARGIN
    assert np.array_equal(cm[sure_c], ocm[sure_c].astype(np.uint8))
    assert np.array_equal(tm[sure_t], otm[sure_t].astype(np.uint8))
    assert cnt[0] == cm.sum() and cnt[1] == tm.sum()
    return cm, tm, ocm, otm


def test_flagger_config4_full(dsax, oracle):
    """256 beams x 4096 t x 48 ch chi-square(2) with seeded RFI."""
    x, truth = oracle.gen_filterbank(404)
    cm, tm, ocm, otm = _compare(dsax, oracle, x)
    assert cm.sum() > 0 and tm.sum() > 0
    # injected persistent tones are found
    tone_cols = truth.all(axis=1)
    guard = dsax.flag_params(256, 4096, 48).guard
    inside = np.zeros_like(tone_cols)
    inside[:, guard:48 - guard] = True
    assert (cm[tone_cols & inside] == 1).mean() > 0.9


def test_flagger_parity_mode(dsax, oracle):
    x, _ = oracle.gen_filterbank(405, nbeam=32, ntime=2048)
    _compare(dsax, oracle, x, parity=1)


def test_flagger_oldspec_and_perm(dsax, oracle):
    x, _ = oracle.gen_filterbank(406, nbeam=16, ntime=1024)
    old = x.mean(axis=1).astype(np.float32) * 0.9
    _compare(dsax, oracle, x, oldspec=old, perm=[10, 20], tbin=64)


@pytest.mark.parametrize("B,T,C,guard", [(3, 1000, 48, 6), (5, 512, 64, 8), (2, 300, 32, 0),
                                         (1, 4096, 24, 1), (2, 700, 320, 20), (3, 512, 200, 12),
                                         (2, 256, 4, 0)])
def test_flagger_shapes(dsax, oracle, B, T, C, guard):
    """Ragged shapes: rows past the last whole bin, several 128-channel
    slabs (320), a last slab narrower than the 128-channel TMA box (200: its
    box reads zeros past nchan), and the smallest width (4)."""
    x, _ = oracle.gen_filterbank(B * T + C, nbeam=B, ntime=T, nchan=C, n_tones=B, n_bursts=B,
                                 n_drift=1)
    _compare(dsax, oracle, x, guard=guard, filt=min(21, C - 2 * guard), tbin=100)
