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
