"""The two reference-style workloads at their full shapes, bit-exact against the AVX2 /
AVX-512BW batched oracle.

* The reference's default table (4000x2000, one degree group of 6), OMS, 20
  iterations, 4096 frames (the plugin's nb_frames = 1024 words, the run
  `main.cpp -OMS -iter 20 -n 1024 -min 1.0 -max 3.0 -pas 0.5` decodes), at every
  Eb/N0 of that run, through LDPC_PACK_AUTO (the 2-frame fp16x2 level kernel),
  all-zero codeword and the reference quantiser: every frame compared.
* The seeded (3,6) QC code (N=4096) with NMS (x0.75, decoder_nms/cuda/CUDA_NMS_SIMD.cu:73-85),
  10 layered iterations, 65536 frames at 2.0 dB: the QC register kernel against the
  oracle on a strided subset of words spread over the whole batch.
"""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_regular

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ebn0", [1.0, 1.5, 2.0, 2.5, 3.0])
def test_reference_table_full_shape(cuda, ebn0):
    import torch
    code = load_table("4000x2000")
    frames, iters = 4096, 20
    llr = make_llr("awgn", frames * code.n, 700 + int(10 * ebn0), sigma=llr_gen.sigma_for(ebn0, 0.5))
    dec = Decoder(code, "OMS", nb_frames=frames // 4)
    assert dec.info()["path"] == 2  # LDPC_PACK_AUTO: the 2-frame fp16x2 level kernel
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.empty(frames * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(frames // 4, dtype=torch.int32, device="cuda")
    dec.decode_device(d_llr, d_out, frames // 4, iters, d_iters=d_it, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    dec.close()
    out = d_out.cpu().numpy().reshape(frames, code.n)
    ref = oracle.decode_batch(code, "OMS", llr, iters)
    assert np.array_equal(out, ref)
    assert (d_it.cpu().numpy() == iters).all()
    # sanity of the operating point: at 3 dB nearly every frame is the all-zero codeword
    if ebn0 >= 3.0:
        assert float((out.sum(axis=1) > 0).mean()) < 0.01


def test_qc_nms_large_batch_strided(cuda):
    import torch
    code = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
    frames = 65536
    llr = make_llr("awgn", frames * code.n, 35, sigma=llr_gen.sigma_for(2.0, 0.5))
    dec = Decoder(code, "NMS", nb_frames=frames // 4)
    assert dec.info()["path"] == 1
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.empty(frames * code.n, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_out, frames // 4, 10, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    dec.close()
    out = d_out.cpu().numpy().reshape(frames, code.n)
    # 32 consecutive frames (8 words) every 1024 frames, plus the batch's last 32
    starts = list(range(0, frames, 1024)) + [frames - 32]
    pick = (np.array(starts)[:, None] + np.arange(32)[None, :]).reshape(-1)
    ref = oracle.decode_batch(code, "NMS", llr.reshape(frames, code.n)[pick], 10)
    assert np.array_equal(out[pick], ref)
