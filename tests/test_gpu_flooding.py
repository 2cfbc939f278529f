"""LDPC_FLAG_FLOODING (decoder path 6): the flooding schedule on the 4-frame fp16x2 level
kernel, bit-exact against the oracle's flooding mode on hard decisions, final APP, final
messages and per-word iteration counts, with and without the early stop."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import assert_same, make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, LdpcError, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_irregular

pytestmark = pytest.mark.gpu


def _decode(code, kind, llr, iters, words, early):
    import torch
    dec = Decoder(code, kind, nb_frames=words, early_stop=early, flooding=True)
    assert dec.info()["path"] == 6
    d_llr = torch.from_numpy(llr).cuda()
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(words, dtype=torch.int32, device="cuda")
    d_app = torch.zeros(4 * words * code.n, dtype=torch.int8, device="cuda")
    d_msg = torch.zeros(4 * words * code.e, dtype=torch.int8, device="cuda")
    dec.decode_device_state(d_llr, d_hard, words, iters, d_it, d_app, d_msg, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    dec.close()
    return {"hard": d_hard.cpu().numpy().reshape(4 * words, code.n), "iters": d_it.cpu().numpy(),
            "app": d_app.cpu().numpy(), "msg": d_msg.cpu().numpy()}


@pytest.mark.parametrize("name", ["576x288", "4000x2000", "1944x972"])
@pytest.mark.parametrize("kind", ["OMS", "NMS", "MS", "2NMS"])
def test_flooding_fixed_iterations(cuda, name, kind):
    code = load_table(name)
    words = 10
    llr = make_llr("awgn", 4 * words * code.n, 61, sigma=llr_gen.sigma_for(2.0, 0.5))
    got = _decode(code, kind, llr, 8, words, False)
    ref = oracle.decode(code, kind, llr, 8, interleaved=False, want_state=True, flooding=True)
    assert_same(got, ref)


@pytest.mark.parametrize("rate", [(1, 2), (5, 6)])
def test_flooding_early_stop(cuda, rate):
    code = qc_irregular(z=27, rate=rate, seed=500 + rate[0])
    words = 24
    r = rate[0] / rate[1]
    llr = np.concatenate([make_llr("awgn", 4 * 8 * code.n, 63 + i, sigma=llr_gen.sigma_for(e, r))
                          for i, e in enumerate((2.0, 3.5, 5.0))])
    got = _decode(code, "OMS", llr, 20, words, True)
    ref = oracle.decode(code, "OMS", llr, 20, interleaved=False, want_state=True, early_stop=True, flooding=True)
    assert_same(got, ref)
    assert len(set(ref["iters"].tolist())) > 1


def test_flooding_learned_and_rejections(cuda):
    code = load_table("576x288")
    words = 6
    llr = make_llr("awgn", 4 * words * code.n, 65, sigma=llr_gen.sigma_for(2.5, 0.5))
    off = np.array([[1, 1], [0, 1], [1, 0], [1, 1]], np.int8)
    sc = np.array([[128, 120], [112, 128], [128, 128], [104, 128]], np.uint8)
    import torch
    dec = Decoder(code, "LEARNED", nb_frames=words, flooding=True)
    dec.set_learned(off, sc)
    d_llr = torch.from_numpy(llr).cuda()
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_hard, words, 6)
    torch.cuda.synchronize()
    dec.close()
    oracle.set_learned(off, sc)
    ref = oracle.decode(code, "LEARNED", llr, 6, flooding=True)
    assert np.array_equal(d_hard.cpu().numpy().reshape(-1, code.n), ref["hard"])
    for pack in ("SIMD4", "I8", "FRAME"):
        with pytest.raises(LdpcError):
            Decoder(code, "OMS", nb_frames=2, pack=pack, flooding=True)
    with pytest.raises(LdpcError):
        Decoder(code, "OMS", nb_frames=2, early_stop="frame", flooding=True)
