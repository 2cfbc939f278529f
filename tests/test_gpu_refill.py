"""LDPC_FLAG_EARLY_STOP_FRAMES (decoder path 5): the QC register kernel with the
early-stop rule applied to each frame alone and finished frames' slots refilled
with the CTA's next frames.  Decisions and per-frame iteration counts against the
CPU oracle's per-frame rule, with more frames than the resident CTAs hold so that
slots are refilled many times; the error paths of the flag."""
import os

import numpy as np
import pytest

import llr_gen
from gpu_helpers import make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, LdpcError, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_regular

pytestmark = pytest.mark.gpu

_CODES = {}
# about 1.5x the frames the resident CTAs hold (4 per CTA; 2, 4, 8, 16 CTAs per SM at
# Z = 256, 128, 64, 32 on 148 SMs), so that every CTA refills its slots
WORDS = {256: 450, 128: 900, 64: 1800, 32: 3600}


def qc(z):
    if z not in _CODES:
        _CODES[z] = qc_regular(z=z, mb=8, nb=16, wc=3, seed=2024 if z == 256 else 300 + z, name="qc3x6_z%d" % z)
    return _CODES[z]


def mixed_llr(code, words, seed, ebn0s):
    """Frames at several noise levels interleaved frame by frame, so that the frames of
    one 4-frame word stop at different iterations."""
    per = -(-4 * words // len(ebn0s))
    parts = [make_llr("awgn", per * code.n, seed + i, sigma=llr_gen.sigma_for(e, 0.5)).reshape(per, code.n)
             for i, e in enumerate(ebn0s)]
    frames = np.stack(parts, axis=1).reshape(-1, code.n)[:4 * words]
    return np.ascontiguousarray(frames).reshape(-1)


def refill_decode(code, kind, llr, iters, words, constants=None, slack=None, early=True, packed=False):
    import torch
    dec = Decoder(code, kind, nb_frames=words, early_stop="frame")
    if constants is not None:
        dec.set_learned(*constants)
    if slack is not None or not early:
        dec.set_early_stop(early, 128 if slack is None else slack)
    info = dec.info()
    d_llr = torch.from_numpy(llr).cuda()
    nbytes = (code.n + 7) // 8 if packed else code.n
    d_out = torch.zeros(4 * words * nbytes, dtype=torch.uint8, device="cuda")
    d_it = torch.full((4 * words,), -1, dtype=torch.int32, device="cuda")
    dec.decode_device(d_llr, d_out, words, iters, out_format=1 if packed else 0, d_iters=d_it)
    torch.cuda.synchronize()
    dec.close()
    return info, d_out.cpu().numpy().reshape(4 * words, nbytes), d_it.cpu().numpy()


@pytest.mark.parametrize("z", [256, 32])
@pytest.mark.parametrize("kind", ["OMS", "MS", "NMS"])
def test_refill_matches_per_frame_oracle(cuda, z, kind):
    code = qc(z)
    words = WORDS[z]
    llr = mixed_llr(code, words, 61, (1.25, 2.0, 2.5, 3.5))
    info, hard, its = refill_decode(code, kind, llr, 20, words)
    assert info["path"] == 5
    ref = oracle.decode(code, kind, llr, 20, early_stop=True, per_frame=True)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])
    assert its.min() < 8 and its.max() == 20       # frames stopped early and ran to the limit
    # within a word the frames stopped at different iterations
    assert (its.reshape(-1, 4).max(1) != its.reshape(-1, 4).min(1)).mean() > 0.3


def test_refill_learned_per_iteration_constants(cuda):
    """Per-lane iteration numbers select the learned constants: rows that change every
    iteration make a lane that ran the wrong row visible in the decisions."""
    code = qc(256)
    words = WORDS[256]
    off = np.array([[1, 0], [0, 1], [2, 1], [1, 1], [0, 0], [1, 2]], dtype=np.int8)
    sc = np.array([[128, 120], [112, 104], [96, 128], [120, 112], [104, 96], [128, 128]], dtype=np.uint8)
    llr = mixed_llr(code, words, 67, (1.5, 2.25, 3.0))
    info, hard, its = refill_decode(code, "LEARNED", llr, 12, words, constants=(off, sc))
    assert info["path"] == 5
    oracle.set_learned(off, sc)
    ref = oracle.decode(code, "LEARNED", llr, 12, early_stop=True, per_frame=True)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])


def test_refill_deployed_constants(cuda):
    from fast_ldpc_decoder_for_gpu_fixed_b200.learned import TRAINED_DIR, load_constants
    code = qc(256)
    words = WORDS[256]
    off, sc, _ = load_constants(os.path.join(TRAINED_DIR, "qc3x6_z256_T10.json"))
    llr = mixed_llr(code, words, 71, (2.0, 2.25, 2.5))
    _, hard, its = refill_decode(code, "LEARNED", llr, 10, words, constants=(off, sc))
    oracle.set_learned(off, sc)
    ref = oracle.decode(code, "LEARNED", llr, 10, early_stop=True, per_frame=True)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])


@pytest.mark.parametrize("slack", [0, 3, 1 << 20])
def test_refill_slack(cuda, slack):
    code = qc(64)
    words = WORDS[64]
    llr = mixed_llr(code, words, 73, (1.5, 2.5, 3.5))
    _, hard, its = refill_decode(code, "OMS", llr, 20, words, slack=slack)
    ref = oracle.decode(code, "OMS", llr, 20, early_stop=True, early_slack=slack, per_frame=True)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])


def test_refill_without_early_stop_and_packed_output(cuda):
    """Early stop off keeps the per-frame scheduling with every frame running `iters`
    (the reference's fixed-iteration result); packed output holds the same bits."""
    code = qc(128)
    words = WORDS[128]
    llr = mixed_llr(code, words, 79, (1.5, 3.0))
    _, hard, its = refill_decode(code, "OMS", llr, 7, words, early=False)
    ref = oracle.decode(code, "OMS", llr, 7)
    assert (its == 7).all()
    assert np.array_equal(hard, ref["hard"])
    _, packed, its2 = refill_decode(code, "OMS", llr, 15, words, packed=True)
    ref2 = oracle.decode(code, "OMS", llr, 15, early_stop=True, per_frame=True)
    assert np.array_equal(its2, ref2["iters"])
    assert np.array_equal(np.unpackbits(packed, axis=1, bitorder="little")[:, :code.n], ref2["hard"])


def test_refill_host_decode(cuda):
    code = qc(256)
    words = 40
    llr = mixed_llr(code, words, 83, (1.5, 2.5))
    dec = Decoder(code, "NMS", nb_frames=words, early_stop="frame")
    out = np.zeros((4 * words, code.n), dtype=np.uint8)
    dec.decode_host(llr.reshape(4 * words, code.n), out, 20)
    dec.close()
    assert np.array_equal(out, oracle.decode(code, "NMS", llr, 20, early_stop=True, per_frame=True)["hard"])


def test_refill_flag_errors(cuda):
    import torch
    code = qc(256)
    with pytest.raises(LdpcError):
        Decoder(code, "2NMS", nb_frames=8, early_stop="frame")     # 2NMS keeps its own rule
    # without the QC refill kernel (or with an explicit SIMD4) the per-frame stop runs on the
    # SIMD4 level kernel (tests/test_gpu_frames_levels.py); F16X2 level kernels refuse it
    for c, pack in ((load_table("4000x2000"), "AUTO"), (code, "SIMD4")):
        d = Decoder(c, "OMS", nb_frames=8, pack=pack, early_stop="frame")
        assert d.info()["path"] == 0
        d.close()
    c = load_table("4000x2000")
    with pytest.raises(LdpcError):
        Decoder(c, "OMS", nb_frames=8, pack="F16X2", early_stop="frame")
    dec = Decoder(code, "OMS", nb_frames=8, early_stop="frame")
    d_llr = torch.zeros(32 * code.n, dtype=torch.int8, device="cuda")
    d_out = torch.zeros(32 * code.n, dtype=torch.uint8, device="cuda")
    with pytest.raises(LdpcError):
        dec.decode_device(d_llr, d_out, 8, 256)                    # iteration counts are bytes
    with pytest.raises(LdpcError):
        dec.decode_device_state(d_llr, d_out, 8, 10, d_app=torch.zeros_like(d_llr))
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    with pytest.raises(LdpcError):
        dec.simulate(8, 10, 0.8, 1, 0, counts)
    dec.close()
    # LDPC_PACK_FRAME stops per frame already: the flag is accepted there
    dec = Decoder(code, "OMS", nb_frames=8, pack="FRAME", early_stop="frame")
    assert dec.info()["path"] == 3
    dec.close()
