"""GPU channel and error counter against the CPU oracle.

Philox4x32-10 words must match bit for bit.  The quantised LLRs are computed
in float on the GPU and in double by the oracle; they may differ only where
8y falls within float rounding of an integer boundary of the truncation:
tolerance |q_gpu - q_oracle| <= 1, at most 1e-4 of the samples, and only at
samples whose double-precision 8y lies within 1e-3 of an integer.
"""
import numpy as np
import pytest

from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("count,seed,offset", [(1, 1, 0), (1001, 7, 0), (4096, 2 ** 40 + 3, 12345), (65537, 99, 2 ** 33)])
def test_philox_matches_oracle(cuda, count, seed, offset):
    import torch
    d = torch.zeros(count, dtype=torch.int32, device="cuda")
    _lib.check(_lib.lib().ldpc_philox(d.data_ptr(), count, seed, offset, None))
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), oracle.philox(count, seed, offset))


@pytest.mark.parametrize("with_cw", [False, True])
def test_awgn_matches_fp64_oracle(cuda, with_cw):
    import torch
    frames, n, sigma, seed = 257, 1000, 0.8, 11
    cw = None
    d_cw = None
    if with_cw:
        cw = (np.random.default_rng(1).integers(0, 2, size=(5, n))).astype(np.uint8)
        d_cw = torch.from_numpy(cw).cuda()
    d = torch.zeros(frames * n, dtype=torch.int8, device="cuda")
    _lib.check(_lib.lib().ldpc_channel_awgn(d.data_ptr(), frames, n, sigma, seed, 3,
                                            d_cw.data_ptr() if d_cw is not None else None,
                                            0 if cw is None else cw.shape[0], None))
    torch.cuda.synchronize()
    got = d.cpu().numpy().reshape(frames, n).astype(int)
    ref, y8 = oracle.awgn(frames, n, sigma, seed, 3, cw)
    diff = np.abs(got - ref.astype(int))
    assert diff.max() <= 1
    bad = np.flatnonzero(diff.reshape(-1))
    assert bad.size <= 1e-4 * got.size
    if bad.size:
        yb = y8.reshape(-1)[bad]
        assert np.all(np.abs(yb - np.round(yb)) < 1e-3)
    # the LLR sign follows the transmitted bit (bit 1 -> positive mean)
    if with_cw:
        mean_pos = got[:, :][np.tile(cw, (frames // 5 + 1, 1))[:frames] == 1].mean()
        mean_neg = got[np.tile(cw, (frames // 5 + 1, 1))[:frames] == 0].mean()
        assert mean_pos > 5 and mean_neg < -5


def test_sigma_matches_reference_formula(cuda):
    L = _lib.lib()
    for ebn0 in (0.0, 1.0, 2.5):
        for rate in (0.5, 0.75):
            assert abs(L.ldpc_sigma(ebn0, rate, 0) - oracle.sigma(ebn0, rate, False)) < 1e-12
            assert abs(L.ldpc_sigma(ebn0, rate, 1) - oracle.sigma(ebn0, rate, True)) < 1e-12


@pytest.mark.parametrize("with_cw", [False, True])
def test_count_errors_matches_oracle(cuda, with_cw):
    import torch
    rng = np.random.default_rng(5)
    frames, n, nv = 300, 500, 250
    hard = (rng.random((frames, n)) < 0.01).astype(np.uint8)
    hard[::7] = 0
    cw = None
    if with_cw:
        cw = rng.integers(0, 2, size=(3, n)).astype(np.uint8)
        hard = hard ^ np.tile(cw, (frames // 3 + 1, 1))[:frames]
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    d_h = torch.from_numpy(hard).cuda()
    d_cw = torch.from_numpy(cw).cuda() if with_cw else None
    _lib.check(_lib.lib().ldpc_count_errors(d_h.data_ptr(), frames, n, nv, d_cw.data_ptr() if with_cw else None,
                                            3 if with_cw else 0, counts.data_ptr(), None))
    torch.cuda.synchronize()
    c = counts.cpu().numpy()
    ref_hard = hard ^ np.tile(cw, (frames // 3 + 1, 1))[:frames] if with_cw else hard
    be, fe, _ = oracle.count_errors(n, nv, ref_hard)
    assert c.tolist() == [frames, be, fe]
