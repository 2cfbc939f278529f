"""GPU tests of the simulation pipeline around the decoder: the fused
channel -> decode -> error-count step (ldpc_simulate) against the three stages
run separately, and the main.cpp-style C++ driver end to end."""
import json
import os
import subprocess

import numpy as np
import pytest

from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, _lib, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import Encoder, qc_regular
from fast_ldpc_decoder_for_gpu_fixed_b200 import build as native_build

pytestmark = pytest.mark.gpu


def _separate(code, kind, words, iters, sigma, seed, offset, d_cw, n_cw, pack="AUTO"):
    import torch
    dec = Decoder(code, kind, nb_frames=words, pack=pack)
    d_llr = torch.zeros(4 * words * code.n, dtype=torch.int8, device="cuda")
    _lib.check(_lib.lib().ldpc_channel_awgn(d_llr.data_ptr(), 4 * words, code.n, sigma, seed, offset,
                                            d_cw.data_ptr() if d_cw is not None else None, n_cw, None))
    d_out = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_out, words, iters)
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    _lib.check(_lib.lib().ldpc_count_errors(d_out.data_ptr(), 4 * words, code.n, code.n_info,
                                            d_cw.data_ptr() if d_cw is not None else None, n_cw,
                                            counts.data_ptr(), None))
    torch.cuda.synchronize()
    dec.close()
    return d_out.cpu().numpy(), counts.cpu().numpy()


def _fused(code, kind, words, iters, sigma, seed, offset, d_cw, n_cw, pack="AUTO"):
    import torch
    dec = Decoder(code, kind, nb_frames=words, pack=pack)
    d_out = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    dec.simulate(words, iters, sigma, seed, offset, counts, d_codewords=d_cw, n_codewords=n_cw, d_hard=d_out)
    torch.cuda.synchronize()
    dec.close()
    return d_out.cpu().numpy(), counts.cpu().numpy()


@pytest.mark.parametrize("pack", ["SIMD4", "F16X2", "I8"])
@pytest.mark.parametrize("name", ["4000x2000", "576x288"])
def test_fused_equals_separate_stages(cuda, name, pack):
    code = load_table(name)
    args = (code, "OMS", 24, 10, 0.9, 77, 5, None, 0, pack)
    h1, c1 = _separate(*args)
    h2, c2 = _fused(*args)
    assert np.array_equal(h1, h2)
    assert c1.tolist() == c2.tolist()
    assert c1[0] == 96 and 0 <= c1[2] <= 96


def test_fused_qc_with_codewords(cuda):
    import torch
    code = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
    enc = Encoder(code)
    cw = enc.encode(np.random.default_rng(3).integers(0, 2, size=(7, enc.k)))
    d_cw = torch.from_numpy(cw).cuda()
    args = (code, "OMS", 32, 10, 0.75, 5, 9, d_cw, 7)
    h1, c1 = _separate(*args)
    h2, c2 = _fused(*args)
    assert np.array_equal(h1, h2)
    assert c1.tolist() == c2.tolist()
    # decisions really are the transmitted codewords (not all-zero) at this SNR
    hard = h2.reshape(128, code.n)
    ok = (hard == cw[np.arange(128) % 7]).all(axis=1)
    assert ok.mean() > 0.9


def test_driver_runs(cuda):
    exe = native_build.build_tools()
    out = subprocess.run([exe, "-OMS", "-iter", "10", "-n", "64", "-min", "2.0", "-max", "2.6", "-pas", "0.5",
                          "-fer", "20", "-code", "576x288", "-json"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert [round(l["ebn0"], 2) for l in lines] == [2.0, 2.5]
    for l in lines:
        assert 0 <= l["fer"] <= 1 and l["frames"] > 0
        assert l["frame_errors"] >= 20 or l["frames"] > 0
    assert "SNR = 2.00" in out.stdout
    info = subprocess.run([exe, "-info"], capture_output=True, text=True, timeout=120)
    assert info.returncode == 0 and "Multi-Processor" in info.stdout
