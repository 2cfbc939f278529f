"""LDPC_FLAG_EARLY_STOP (syndrome early stop per 4-frame word): GPU decoders
against the CPU oracle with the same rule, for every packing, the QC kernel and
the fused simulation; final decisions, state and per-word iteration counts."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import assert_same, gpu_decode, make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, LdpcError, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_regular

pytestmark = pytest.mark.gpu


def _qc():
    return qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")


def _ref(code, kind, llr, iters):
    return oracle.decode(code, kind, llr, iters, interleaved=False, want_state=True, early_stop=True)


@pytest.mark.parametrize("pack", ["SIMD4", "F16X2", "I8"])
@pytest.mark.parametrize("name", ["4000x2000", "576x288", "1944x972"])
@pytest.mark.parametrize("kind", ["OMS", "NMS", "MS"])
def test_early_stop_level_kernels(cuda, name, pack, kind):
    code = load_table(name)
    words = 24
    # a spread of noise levels: some words stop after a few iterations, some never
    llr = np.concatenate([make_llr("awgn", 4 * 8 * code.n, 11 + i, sigma=llr_gen.sigma_for(e, 0.5))
                          for i, e in enumerate((1.0, 2.0, 3.5))])
    ref = _ref(code, kind, llr, 30)
    got = gpu_decode(code, kind, llr, 30, words, pack=pack, early_stop=True)
    assert got["info"]["path"] == 0
    assert_same(got, ref)
    assert len(set(ref["iters"].tolist())) > 2    # the words stopped at different iterations


def test_early_stop_qc_kernel(cuda):
    code = _qc()
    words = 48
    llr = np.concatenate([make_llr("awgn", 4 * 16 * code.n, 21 + i, sigma=llr_gen.sigma_for(e, 0.5))
                          for i, e in enumerate((1.25, 2.0, 3.0))])
    for kind in ("OMS", "NMS"):
        ref = _ref(code, kind, llr, 20)
        got = gpu_decode(code, kind, llr, 20, words, early_stop=True)
        assert got["info"]["path"] == 1
        assert_same(got, ref)
        assert ref["iters"].min() < 10 and ref["iters"].max() == 20


@pytest.mark.parametrize("slack", [0, 5, 1 << 20])
def test_early_stop_slack(cuda, slack):
    import torch
    code = _qc()
    words = 32
    llr = np.concatenate([make_llr("awgn", 4 * 16 * code.n, 51 + i, sigma=llr_gen.sigma_for(e, 0.5))
                          for i, e in enumerate((1.75, 2.5))])
    ref = oracle.decode(code, "OMS", llr, 20, interleaved=False, want_state=True, early_stop=True,
                        early_slack=slack)
    for pack in ("AUTO", "SIMD4"):
        dec = Decoder(code, "OMS", nb_frames=words, pack=pack, early_stop=True)
        dec.set_early_stop(True, slack)
        d_llr = torch.from_numpy(llr).cuda()
        d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
        d_it = torch.zeros(words, dtype=torch.int32, device="cuda")
        dec.decode_device(d_llr, d_hard, words, 20, d_iters=d_it)
        torch.cuda.synchronize()
        dec.close()
        assert np.array_equal(d_it.cpu().numpy(), ref["iters"])
        assert np.array_equal(d_hard.cpu().numpy().reshape(4 * words, code.n), ref["hard"])


@pytest.mark.parametrize("kind", ["OMS", "NMS", "MS", "LEARNED", "LEARNED_OFS"])
def test_early_stop_exact_gate_qc_kernel(cuda, kind):
    """LDPC_EARLY_SLACK_ANY on the 4-frame QC kernel: its last-layer gate stops each word
    at the first iteration whose decisions are codewords, like the oracle with an
    unbounded slack (decisions, APP, messages, counts)."""
    import torch
    from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib
    code = _qc()
    words = 48
    llr = np.concatenate([make_llr("awgn", 4 * 16 * code.n, 61 + i, sigma=llr_gen.sigma_for(e, 0.5))
                          for i, e in enumerate((1.5, 2.25, 3.0))])
    constants = None
    if kind == "LEARNED":
        constants = (np.array([[1, 1]] * 3 + [[0, 0]] * 7, dtype=np.int8), np.array([[112, 112]] * 10, dtype=np.uint8))
    elif kind == "LEARNED_OFS":  # every scale 1.0: the offset-only learned kernel
        kind, constants = "LEARNED", (np.array([[0, 0]] * 2 + [[1, 1]] * 8, dtype=np.int8),
                                      np.array([[128, 128]] * 10, dtype=np.uint8))
    if constants is not None:
        oracle.set_learned(*constants)
    ref = oracle.decode(code, kind, llr, 20, interleaved=False, want_state=True, early_stop=True,
                        early_slack=_lib.EARLY_SLACK_ANY)
    got = gpu_decode(code, kind, llr, 20, words, early_stop=True, constants=constants, slack=_lib.EARLY_SLACK_ANY)
    assert got["info"]["path"] == 1
    assert_same(got, ref)
    assert ref["iters"].min() < 8 and ref["iters"].max() == 20
    # the per-frame syndrome flags of the same decode
    dec = Decoder(code, kind, nb_frames=words, early_stop=True)
    if constants is not None:
        dec.set_learned(*constants)
    dec.set_early_stop(True, _lib.EARLY_SLACK_ANY)
    d_llr = torch.from_numpy(llr).cuda()
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_ok = torch.zeros(4 * words, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_hard, words, 20, d_syndrome=d_ok)
    torch.cuda.synchronize()
    dec.close()
    want_ok = (code.syndrome(ref["hard"]).max(axis=1) == 0).astype(np.uint8)
    assert np.array_equal(d_ok.cpu().numpy(), want_ok)
    assert np.array_equal(d_hard.cpu().numpy().reshape(4 * words, code.n), ref["hard"])


def test_early_stop_learned(cuda):
    code = _qc()
    words = 16
    off = np.array([[1, 1]] * 3 + [[0, 0]] * 7, dtype=np.int8)
    sc = np.array([[120, 120]] * 10, dtype=np.uint8)
    oracle.set_learned(off, sc)
    llr = make_llr("awgn", 4 * words * code.n, 31, sigma=llr_gen.sigma_for(2.0, 0.5))
    ref = _ref(code, "LEARNED", llr, 15)
    for pack in ("AUTO", "SIMD4"):
        assert_same(gpu_decode(code, "LEARNED", llr, 15, words, pack=pack, early_stop=True, constants=(off, sc)), ref)


def test_early_stop_never_changes_converged_words(cuda):
    """Words that stop early hold codewords; at high SNR every word stops before the cap."""
    code = _qc()
    words = 32
    llr = make_llr("awgn", 4 * words * code.n, 41, sigma=llr_gen.sigma_for(3.5, 0.5))
    got = gpu_decode(code, "OMS", llr, 30, words, early_stop=True, state=False)
    assert got["iters"].max() < 30
    assert (code.syndrome(got["hard"]) == 0).all()


def test_early_stop_fused_simulation(cuda):
    import torch
    code = load_table("576x288")
    words = 64
    dec = Decoder(code, "OMS", nb_frames=words, early_stop=True)
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    dec.simulate(words, 25, 0.8, 5, 0, counts, d_hard=d_hard)
    torch.cuda.synchronize()
    dec.close()
    llr, _ = oracle.awgn(4 * words, code.n, 0.8, 5, 0)
    ref = _ref(code, "OMS", llr, 25)
    assert np.array_equal(d_hard.cpu().numpy().reshape(4 * words, code.n), ref["hard"])


def test_early_stop_rejected_for_2nms(cuda):
    with pytest.raises(LdpcError):
        Decoder(load_table("576x288"), "2NMS", nb_frames=4, early_stop=True)
