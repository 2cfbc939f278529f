"""GPU parity of the QC register-message kernel (the path the bench workload
uses: seeded regular (3,6) QC code, Z=256) against the CPU oracle, plus the
level-scheduled kernel on the same code."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import assert_same, gpu_decode, make_llr, oracle_decode
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_regular

pytestmark = pytest.mark.gpu

_CODE = {}


def qc_code():
    if "c" not in _CODE:
        _CODE["c"] = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
    return _CODE["c"]


@pytest.mark.parametrize("kind", ["MS", "OMS", "NMS", "2NMS", "XMS"])
@pytest.mark.parametrize("inp", ["awgn", "uniform", "extreme"])
def test_qc_kernel_parity(cuda, kind, inp):
    code = qc_code()
    words = 12
    llr = make_llr(inp, 4 * words * code.n, 31, sigma=llr_gen.sigma_for(1.5, 0.5))
    dec = Decoder(code, kind, nb_frames=1)
    assert dec.info()["path"] == 1, "QC code should take the register-message kernel"
    dec.close()
    assert_same(gpu_decode(code, kind, llr, 10, words), oracle_decode(code, kind, llr, 10))


@pytest.mark.parametrize("pack", ["SIMD4", "F16X2", "I8"])
def test_level_kernel_on_qc_code(cuda, pack):
    code = qc_code()
    code.no_qc = True
    try:
        words = 6
        llr = make_llr("awgn", 4 * words * code.n, 32, sigma=llr_gen.sigma_for(2.0, 0.5))
        for kind in ("OMS", "2NMS"):
            assert_same(gpu_decode(code, kind, llr, 10, words, pack=pack), oracle_decode(code, kind, llr, 10))
    finally:
        code.no_qc = False


def test_qc_early_termination(cuda):
    code = qc_code()
    words = 40
    llr = make_llr("awgn", 4 * words * code.n, 33, sigma=llr_gen.sigma_for(2.5, 0.5))
    gpu = gpu_decode(code, "2NMS", llr, 25, words)
    ref = oracle_decode(code, "2NMS", llr, 25)
    assert_same(gpu, ref)
    assert len(set(ref["iters"].tolist())) > 1


def test_qc_large_batch_properties(cuda):
    """65536 frames (the bench batch): decode equals the AVX2 oracle on a strided
    subset of words and every frame's hard decision is a codeword at high SNR."""
    import torch
    from oracle import oracle
    code = qc_code()
    frames = 65536
    llr = make_llr("awgn", frames * code.n, 34, sigma=llr_gen.sigma_for(4.0, 0.5))
    dec = Decoder(code, "OMS", nb_frames=frames // 4)
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.empty(frames * code.n, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_out, frames // 4, 10, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().reshape(frames, code.n)
    pick = np.arange(0, frames, 1024)[:, None] + np.arange(32)[None, :]
    sub = llr.reshape(frames, code.n)[pick.reshape(-1)]
    ref = oracle.decode_batch(code, "OMS", sub, 10)
    assert np.array_equal(out[pick.reshape(-1)], ref)
    # all-zero transmitted codeword at 4 dB: (nearly) every decision is the zero codeword
    fer = float((out.sum(axis=1) > 0).mean())
    assert fer < 1e-3


# ---- the 2-frame QC kernel (decoder path 4) on 24-column irregular bases ----

_IRR = {}


def irregular(rate, z):
    key = (rate, z)
    if key not in _IRR:
        from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_irregular
        _IRR[key] = qc_irregular(z=z, rate=rate, seed=500 + z)
    return _IRR[key]


def _pair_decode(code, kind, llr, iters, words, early=False, constants=None, pack="F16X2"):
    import torch
    dec = Decoder(code, kind, nb_frames=words, pack=pack, early_stop=early)
    if constants is not None:
        dec.set_learned(*constants)
    path = dec.info()["path"]
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.full((words,), 77, dtype=torch.int32, device="cuda")   # the decoder zeroes it
    dec.decode_device(d_llr, d_out, words, iters, d_iters=d_it)
    torch.cuda.synchronize()
    dec.close()
    return path, d_out.cpu().numpy().reshape(4 * words, code.n), d_it.cpu().numpy()


@pytest.mark.parametrize("rate,z", [((1, 2), 81), ((2, 3), 54), ((3, 4), 27), ((5, 6), 27), ((1, 2), 64)])
@pytest.mark.parametrize("kind", ["MS", "OMS", "NMS"])
def test_pair_qc_kernel_fixed_iterations(cuda, rate, z, kind):
    from oracle import oracle
    code = irregular(rate, z)
    words = 10
    llr = make_llr("awgn", 4 * words * code.n, 41, sigma=llr_gen.sigma_for(2.5, rate[0] / rate[1]))
    path, hard, its = _pair_decode(code, kind, llr, 12, words)
    assert path == 4
    ref = oracle.decode(code, kind, llr, 12)
    assert np.array_equal(hard, ref["hard"])
    assert (its == 12).all()


@pytest.mark.parametrize("rate,z", [((1, 2), 81), ((3, 4), 54), ((5, 6), 81)])
def test_pair_qc_kernel_early_stop(cuda, rate, z):
    from oracle import oracle
    code = irregular(rate, z)
    words = 24
    r = rate[0] / rate[1]
    llr = np.concatenate([make_llr("awgn", 4 * 8 * code.n, 43 + i, sigma=llr_gen.sigma_for(e, r))
                          for i, e in enumerate((1.5, 3.0, 5.0))])
    path, hard, its = _pair_decode(code, "OMS", llr, 20, words, early=True)
    assert path == 4
    ref = oracle.decode(code, "OMS", llr, 20, early_stop=True, pairs=True)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])
    assert len(set(its.tolist())) > 2


def test_pair_qc_kernel_learned(cuda):
    from oracle import oracle
    code = irregular((2, 3), 81)
    words = 8
    off = np.array([[1, 1], [0, 0], [1, 2]], dtype=np.int8)
    sc = np.array([[120, 128], [112, 104], [128, 96]], dtype=np.uint8)
    oracle.set_learned(off, sc)
    llr = make_llr("awgn", 4 * words * code.n, 47, sigma=llr_gen.sigma_for(2.5, 2 / 3))
    path, hard, _ = _pair_decode(code, "LEARNED", llr, 10, words, early=True, constants=(off, sc))
    assert path == 4
    ref = oracle.decode(code, "LEARNED", llr, 10, early_stop=True, pairs=True)
    assert np.array_equal(hard, ref["hard"])


def test_pair_qc_kernel_other_paths(cuda):
    """AUTO and 2NMS (early termination per word) take the level kernels; host decode
    and the fused simulation run on the 2-frame kernel."""
    import torch
    from oracle import oracle
    code = irregular((1, 2), 64)  # row degrees <= 10: the 2-frame kernel holds it
    words = 6
    llr = make_llr("awgn", 4 * words * code.n, 53, sigma=llr_gen.sigma_for(2.0, 0.5))
    path, hard, _ = _pair_decode(code, "2NMS", llr, 15, words)
    assert path != 4
    assert np.array_equal(hard, oracle.decode(code, "2NMS", llr, 15)["hard"])
    path, hard, _ = _pair_decode(code, "OMS", llr, 15, words, early=True, pack="AUTO")
    assert path == 0
    assert np.array_equal(hard, oracle.decode(code, "OMS", llr, 15, early_stop=True)["hard"])
    dec = Decoder(code, "OMS", nb_frames=words, pack="F16X2")
    assert dec.info()["path"] == 4
    out = np.zeros((4 * words, code.n), dtype=np.uint8)
    dec.decode_host(llr.reshape(4 * words, code.n), out, 15)
    assert np.array_equal(out, oracle.decode(code, "OMS", llr, 15)["hard"])
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    dec.simulate(words, 15, 0.8, 9, 2, counts, d_hard=d_hard, n_vars=code.n)
    torch.cuda.synchronize()
    sim_llr, _ = oracle.awgn(4 * words, code.n, 0.8, 9, 2)
    assert np.array_equal(d_hard.cpu().numpy().reshape(4 * words, code.n), oracle.decode(code, "OMS", sim_llr, 15)["hard"])
    dec.close()


# ---- path 7: the 2-frame QC kernel with each row split over 2 or 4 lanes ----

@pytest.mark.parametrize("rate,z", [((1, 2), 81), ((2, 3), 54), ((3, 4), 27), ((5, 6), 27), ((5, 6), 64),
                                    ((3, 4), 128)])
@pytest.mark.parametrize("kind", ["MS", "OMS", "NMS"])
def test_split_qc_kernel_fixed_iterations(cuda, rate, z, kind):
    """Rows of degree up to 24 split over 4 lanes (Z up to 128, 512 threads): the warp-shuffle
    merge of min1 / min2 / parity equals the serial row update bit for bit."""
    from oracle import oracle
    code = irregular(rate, z)
    words = 10
    llr = make_llr("uniform" if kind == "MS" else "awgn", 4 * words * code.n, 61,
                   sigma=llr_gen.sigma_for(2.5, rate[0] / rate[1]))
    path, hard, its = _pair_decode(code, kind, llr, 12, words, pack="F16X2_SPLIT")
    assert path == 7
    ref = oracle.decode(code, kind, llr, 12)
    assert np.array_equal(hard, ref["hard"])
    assert (its == 12).all()


@pytest.mark.parametrize("rate,z", [((1, 2), 81), ((5, 6), 27)])
def test_split_qc_kernel_early_stop_and_learned(cuda, rate, z):
    from oracle import oracle
    code = irregular(rate, z)
    words = 24
    r = rate[0] / rate[1]
    llr = np.concatenate([make_llr("awgn", 4 * 8 * code.n, 67 + i, sigma=llr_gen.sigma_for(e, r))
                          for i, e in enumerate((1.5, 3.0, 5.0))])
    path, hard, its = _pair_decode(code, "OMS", llr, 20, words, early=True, pack="F16X2_SPLIT")
    assert path == 7
    ref = oracle.decode(code, "OMS", llr, 20, early_stop=True, pairs=True)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])
    assert len(set(its.tolist())) > 2
    off = np.array([[1, 1], [0, 0], [1, 2]], dtype=np.int8)
    sc = np.array([[120, 128], [112, 104], [128, 96]], dtype=np.uint8)
    oracle.set_learned(off, sc)
    path, hard, _ = _pair_decode(code, "LEARNED", llr, 10, words, early=True, constants=(off, sc),
                                 pack="F16X2_SPLIT")
    assert path == 7
    assert np.array_equal(hard, oracle.decode(code, "LEARNED", llr, 10, early_stop=True, pairs=True)["hard"])


def test_split_qc_kernel_refusals(cuda):
    from fast_ldpc_decoder_for_gpu_fixed_b200 import LdpcError
    with pytest.raises(LdpcError):   # the regular 8x16 base has no 2-frame kernel
        Decoder(qc_code(), "OMS", nb_frames=4, pack="F16X2_SPLIT")
    with pytest.raises(LdpcError):   # 2NMS terminates per 4-frame word
        Decoder(irregular((1, 2), 81), "2NMS", nb_frames=4, pack="F16X2_SPLIT")
    with pytest.raises(LdpcError):   # Z = 192: more than 512 threads
        Decoder(irregular((3, 4), 192), "OMS", nb_frames=4, pack="F16X2_SPLIT")
