"""LDPC_FLAG_EARLY_STOP_PAIRS on the 4-frame QC register kernel (decoder path 1): each
frame pair of a word (frames 4g, 4g+1 and 4g+2, 4g+3) stops on its own.  Hard
decisions, per-word iteration counts (the larger of the two pairs') and per-frame
syndrome flags must equal the oracle's `pairs` rule (oracle_decode_ex, group 2), which
decodes each pair as its own 2-lane word."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_regular

pytestmark = pytest.mark.gpu

_CODE = {}


def qc_code():
    if "c" not in _CODE:
        _CODE["c"] = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
    return _CODE["c"]


def _mixed(code, words, seed, ebn0s):
    """Frame f of the batch at Eb/N0 ebn0s[f % len]: the pairs of one word see different
    noise levels, so they stop at different iterations."""
    per = -(-4 * words // len(ebn0s))
    parts = [make_llr("awgn", per * code.n, seed + i, sigma=llr_gen.sigma_for(e, 0.5)).reshape(per, code.n)
             for i, e in enumerate(ebn0s)]
    return np.ascontiguousarray(np.stack(parts, axis=1).reshape(-1, code.n)[:4 * words]).reshape(-1)


def _run(code, kind, llr, iters, words, early="pairs", constants=None, slack=None, toggle=None):
    import torch
    dec = Decoder(code, kind, nb_frames=words, early_stop=early)
    assert dec.info()["path"] == 1
    if constants is not None:
        dec.set_learned(*constants)
    if slack is not None:
        dec.set_early_stop(True, slack)
    if toggle is not None:
        dec.set_early_stop(toggle)
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.full((words,), 77, dtype=torch.int32, device="cuda")
    d_syn = torch.full((4 * words,), 7, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_out, words, iters, d_iters=d_it, d_syndrome=d_syn)
    torch.cuda.synchronize()
    dec.close()
    return (d_out.cpu().numpy().reshape(4 * words, code.n), d_it.cpu().numpy(), d_syn.cpu().numpy())


def _flags(code, hard):
    return (code.syndrome(hard).sum(axis=1) == 0).astype(np.uint8)


LEARNED_GENERAL = (np.array([[1, 1], [0, 0], [1, 2], [0, 1]] * 3, dtype=np.int8),
                   np.array([[120, 128], [112, 104], [128, 96], [128, 128]] * 3, dtype=np.uint8))
LEARNED_OFFSETS = (np.array([[1, 1], [2, 2], [1, 1], [0, 0]] * 3, dtype=np.int8),
                   np.full((12, 2), 128, dtype=np.uint8))


@pytest.mark.parametrize("kind,constants", [("MS", None), ("OMS", None), ("NMS", None),
                                            ("LEARNED", LEARNED_GENERAL), ("LEARNED", LEARNED_OFFSETS)],
                         ids=["MS", "OMS", "NMS", "LEARNED", "LEARNED_OFS"])
def test_pairs_match_oracle(cuda, kind, constants):
    code = qc_code()
    words = 48
    # min-sum without correction converges later: a higher mix, so that pairs stop at many counts
    llr = _mixed(code, words, 611, (2.5, 3.5, 4.5) if kind == "MS" else (1.5, 2.25, 3.0))
    if constants is not None:
        oracle.set_learned(*constants)
    hard, its, syn = _run(code, kind, llr, 12, words, constants=constants)
    ref = oracle.decode(code, kind, llr, 12, early_stop=True, pairs=True)
    assert np.array_equal(hard, ref["hard"])
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(syn, _flags(code, ref["hard"]))
    assert len(set(its.tolist())) > 2


@pytest.mark.parametrize("kind,constants", [("MS", None), ("OMS", None), ("NMS", None),
                                            ("LEARNED", LEARNED_GENERAL), ("LEARNED", LEARNED_OFFSETS)],
                         ids=["MS", "OMS", "NMS", "LEARNED", "LEARNED_OFS"])
def test_pairs_exact_gate_match_oracle(cuda, kind, constants):
    """LDPC_EARLY_SLACK_ANY: the per-pair kernel that goes on with the remaining pair
    alone (decode_qc_pairs_kernel).  Decisions, counts, syndrome flags, final APP and
    messages against the oracle's pair rule with an unbounded slack."""
    import torch
    from gpu_helpers import assert_same
    from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib
    code = qc_code()
    words = 48
    llr = _mixed(code, words, 631, (2.5, 3.5, 4.5) if kind == "MS" else (1.5, 2.25, 3.0))
    if constants is not None:
        oracle.set_learned(*constants)
    ref = oracle.decode(code, kind, llr, 12, interleaved=False, want_state=True, early_stop=True,
                        early_slack=_lib.EARLY_SLACK_ANY, pairs=True)
    hard, its, syn = _run(code, kind, llr, 12, words, constants=constants, slack=_lib.EARLY_SLACK_ANY)
    assert np.array_equal(hard, ref["hard"])
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(syn, _flags(code, ref["hard"]))
    assert len(set(its.tolist())) > 2
    # the same decode with the state dumps (APP and messages in the reference layouts)
    dec = Decoder(code, kind, nb_frames=words, early_stop="pairs")
    if constants is not None:
        dec.set_learned(*constants)
    dec.set_early_stop(True, _lib.EARLY_SLACK_ANY)
    d_llr = torch.from_numpy(llr).cuda()
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(words, dtype=torch.int32, device="cuda")
    d_app = torch.zeros(4 * words * code.n, dtype=torch.int8, device="cuda")
    d_msg = torch.zeros(4 * words * code.e, dtype=torch.int8, device="cuda")
    dec.decode_device_state(d_llr, d_hard, words, 12, d_it, d_app, d_msg, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    dec.close()
    got = {"hard": d_hard.cpu().numpy().reshape(4 * words, code.n), "iters": d_it.cpu().numpy(),
           "app": d_app.cpu().numpy(), "msg": d_msg.cpu().numpy()}
    assert_same(got, ref)


@pytest.mark.parametrize("kind,constants", [("OMS", None), ("LEARNED", LEARNED_GENERAL)], ids=["OMS", "LEARNED"])
def test_pairs_exact_gate_large_batch(cuda, kind, constants):
    """The per-pair exact-gate decode (decode_qc_pairs_kernel) on more words than the GPU
    holds at once, at four noise levels: every pair's decisions, its word's count, the
    syndrome flags and the final state must equal the oracle's pair rule."""
    import torch
    from gpu_helpers import assert_same
    from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib
    code = qc_code()
    words = 1200
    llr = _mixed(code, words, 641, (1.75, 2.25, 2.75, 3.5))
    if constants is not None:
        oracle.set_learned(*constants)
    ref = oracle.decode(code, kind, llr, 12, interleaved=False, want_state=True, early_stop=True,
                        early_slack=_lib.EARLY_SLACK_ANY, pairs=True)
    hard, its, syn = _run(code, kind, llr, 12, words, constants=constants, slack=_lib.EARLY_SLACK_ANY)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])
    assert np.array_equal(syn, _flags(code, ref["hard"]))
    dec = Decoder(code, kind, nb_frames=words, early_stop="pairs")
    if constants is not None:
        dec.set_learned(*constants)
    dec.set_early_stop(True, _lib.EARLY_SLACK_ANY)
    d_llr = torch.from_numpy(llr).cuda()
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(words, dtype=torch.int32, device="cuda")
    d_app = torch.zeros(4 * words * code.n, dtype=torch.int8, device="cuda")
    d_msg = torch.zeros(4 * words * code.e, dtype=torch.int8, device="cuda")
    dec.decode_device_state(d_llr, d_hard, words, 12, d_it, d_app, d_msg, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    dec.close()
    got = {"hard": d_hard.cpu().numpy().reshape(4 * words, code.n), "iters": d_it.cpu().numpy(),
           "app": d_app.cpu().numpy(), "msg": d_msg.cpu().numpy()}
    assert_same(got, ref)


def test_pairs_slack_and_toggle(cuda):
    code = qc_code()
    words = 24
    llr = _mixed(code, words, 623, (1.75, 2.5))
    hard, its, _ = _run(code, "OMS", llr, 15, words, slack=0)
    ref = oracle.decode(code, "OMS", llr, 15, early_stop=True, early_slack=0, pairs=True)
    assert np.array_equal(hard, ref["hard"])
    assert np.array_equal(its, ref["iters"])
    # early stop off: the fixed-iteration kernel; back on: the per-pair rule again
    hard, its, _ = _run(code, "OMS", llr, 15, words, toggle=False)
    assert np.array_equal(hard, oracle.decode(code, "OMS", llr, 15)["hard"])
    assert (its == 15).all()


def test_pairs_large_batch_strided(cuda):
    """The bench shape (65536 frames at 2.25 dB): a strided subset of words against the
    oracle, every other word's decisions must be codewords or have run to the limit."""
    import torch
    code = qc_code()
    frames = 65536
    llr = make_llr("awgn", frames * code.n, 629, sigma=llr_gen.sigma_for(2.25, 0.5))
    dec = Decoder(code, "OMS", nb_frames=frames // 4, early_stop="pairs")
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.empty(frames * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(frames // 4, dtype=torch.int32, device="cuda")
    dec.decode_device(d_llr, d_out, frames // 4, 10, d_iters=d_it, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    dec.close()
    out = d_out.cpu().numpy().reshape(frames, code.n)
    its = d_it.cpu().numpy()
    words = np.arange(0, frames // 4, 512)
    pick = (4 * words[:, None] + np.arange(4)[None, :]).reshape(-1)
    ref = oracle.decode(code, "OMS", llr.reshape(frames, code.n)[pick].reshape(-1), 10, early_stop=True, pairs=True)
    assert np.array_equal(out[pick], ref["hard"])
    assert np.array_equal(its[words], ref["iters"])
    assert 4.0 < its.mean() < 8.0


def test_pairs_refused_elsewhere(cuda):
    """Decoders without a per-pair kernel refuse the flag."""
    from fast_ldpc_decoder_for_gpu_fixed_b200 import load_table, LdpcError
    code = load_table("4000x2000")
    with pytest.raises(LdpcError):
        Decoder(code, "OMS", nb_frames=4, early_stop="pairs")
    with pytest.raises(LdpcError):
        Decoder(qc_code(), "OMS", nb_frames=4, pack="SIMD4", early_stop="pairs")
