"""LDPC_FLAG_EARLY_STOP_FRAMES on the SIMD4 level kernel (decoder path 0) and inside the
persistent multi-code batch kernel: each frame (byte lane of the 4-frame word) stops on
its own, its decisions written when it stops while the other frames of its word go on.
Decisions, per-frame iteration counts and syndrome flags must equal the oracle's
per-frame rule (oracle_decode_ex, group 1: each frame decoded alone)."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Batch, Decoder, LdpcError, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_irregular

pytestmark = pytest.mark.gpu


def _mixed(code, words, seed, ebn0s):
    per = -(-4 * words // len(ebn0s))
    rate = code.n_info / code.n
    parts = [make_llr("awgn", per * code.n, seed + i, sigma=llr_gen.sigma_for(e, rate)).reshape(per, code.n)
             for i, e in enumerate(ebn0s)]
    return np.ascontiguousarray(np.stack(parts, axis=1).reshape(-1, code.n)[:4 * words]).reshape(-1)


def _flags(code, hard):
    return (code.syndrome(hard).sum(axis=1) == 0).astype(np.uint8)


@pytest.mark.parametrize("name,kind", [("4000x2000", "OMS"), ("576x288", "OMS"), ("1944x972", "NMS"),
                                       ("576x288", "MS"), ("2304x1152", "LEARNED")])
def test_level_kernel_per_frame(cuda, name, kind):
    import torch
    code = load_table(name)
    words = 24
    llr = _mixed(code, words, 810 + len(name), (1.0, 2.0, 3.0, 4.0))
    constants = None
    if kind == "LEARNED":
        constants = (np.array([[1, 2], [0, 1], [1, 1]], dtype=np.int8),
                     np.array([[120, 128], [112, 104], [128, 96]], dtype=np.uint8))
        oracle.set_learned(*constants)
    dec = Decoder(code, kind, nb_frames=words, early_stop="frame")
    if constants is not None:
        dec.set_learned(*constants)
    info = dec.info()
    assert info["path"] == 0 and info["pack"] == 0
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.full((4 * words,), -1, dtype=torch.int32, device="cuda")
    d_syn = torch.full((4 * words,), 7, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_out, words, 25, d_iters=d_it, d_syndrome=d_syn)
    torch.cuda.synchronize()
    with pytest.raises(LdpcError):   # the per-frame stop cannot be turned off
        dec.set_early_stop(False)
    dec.close()
    ref = oracle.decode(code, kind, llr, 25, early_stop=True, per_frame=True)
    hard = d_out.cpu().numpy().reshape(4 * words, code.n)
    assert np.array_equal(hard, ref["hard"])
    assert np.array_equal(d_it.cpu().numpy(), ref["iters"])
    assert np.array_equal(d_syn.cpu().numpy(), _flags(code, ref["hard"]))
    its = ref["iters"].reshape(words, 4)
    assert (its.max(axis=1) != its.min(axis=1)).sum() > words // 2   # frames of one word stop apart


def test_level_kernel_per_frame_host_and_simulation(cuda):
    """The host call (iteration counts per frame) and the fused channel with error counts."""
    import torch
    code = load_table("1944x972")
    words = 40
    llr = _mixed(code, words, 830, (1.5, 2.5, 3.5))
    dec = Decoder(code, "OMS", nb_frames=words, early_stop="frame")
    out = np.zeros(4 * words * code.n, dtype=np.uint8)
    its = np.full(4 * words, -1, dtype=np.int32)
    syn = np.full(4 * words, 7, dtype=np.uint8)
    dec.decode_host_ex(llr, out, 20, iters_out=its, syndrome_ok=syn)
    ref = oracle.decode(code, "OMS", llr, 20, early_stop=True, per_frame=True)
    assert np.array_equal(out.reshape(4 * words, code.n), ref["hard"])
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(syn, _flags(code, ref["hard"]))
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    dec.simulate(words, 20, 0.8, 5, 3, counts, d_hard=d_hard, n_vars=code.n)
    torch.cuda.synchronize()
    dec.close()
    sim_llr, _ = oracle.awgn(4 * words, code.n, 0.8, 5, 3)
    sref = oracle.decode(code, "OMS", sim_llr, 20, early_stop=True, per_frame=True)
    assert np.array_equal(d_hard.cpu().numpy().reshape(4 * words, code.n), sref["hard"])
    be, fe, _ = oracle.count_errors(code.n, code.n, sref["hard"])
    assert counts.cpu().tolist() == [4 * words, be, fe]


def test_per_frame_refusals(cuda):
    code = load_table("576x288")
    with pytest.raises(LdpcError):   # one frame per byte lane: SIMD4 only
        Decoder(code, "OMS", nb_frames=4, pack="F16X2", early_stop="frame")
    with pytest.raises(LdpcError):
        Decoder(code, "2NMS", nb_frames=4, early_stop="frame")


@pytest.mark.parametrize("strategy", ["persistent", "per_code"])
def test_batch_per_frame(cuda, strategy):
    """The persistent multi-code kernel and the per-code strategy with each frame stopping
    on its own (counts per frame)."""
    import torch
    cs = [qc_irregular(z=27, rate=r, seed=900 + i) for i, r in enumerate(((1, 2), (2, 3), (3, 4), (5, 6)))]
    words = [6, 3, 5, 4]
    host, llrs, outs, its, syns = [], [], [], [], []
    for i, (c, w) in enumerate(zip(cs, words)):
        x = _mixed(c, w, 850 + 10 * i, (1.5, 3.0, 4.5, 6.0))
        host.append(x)
        llrs.append(torch.from_numpy(x).cuda())
        outs.append(torch.zeros(4 * w * c.n, dtype=torch.uint8, device="cuda"))
        its.append(torch.full((4 * w,), -1, dtype=torch.int32, device="cuda"))
        syns.append(torch.full((4 * w,), 7, dtype=torch.uint8, device="cuda"))
    st = torch.cuda.Stream()
    b = Batch(cs, "OMS", early_stop="frame", graph=True)
    if strategy == "per_code":
        b.configure(per_code=True, pack="SIMD4")
    else:
        b.configure(pack="SIMD4", threads=64)
    with torch.cuda.stream(st):
        b.decode(llrs, outs, words, 20, d_iters=its, d_syndrome=syns, stream=st)
    st.synchronize()
    b.close()
    stopped_apart = 0
    for c, w, x, o, it, sy in zip(cs, words, host, outs, its, syns):
        ref = oracle.decode(c, "OMS", x, 20, early_stop=True, per_frame=True)
        assert np.array_equal(o.cpu().numpy().reshape(4 * w, c.n), ref["hard"]), c.name
        assert np.array_equal(it.cpu().numpy(), ref["iters"]), c.name
        assert np.array_equal(sy.cpu().numpy(), _flags(c, ref["hard"])), c.name
        r = ref["iters"].reshape(w, 4)
        stopped_apart += int((r.max(axis=1) != r.min(axis=1)).sum())
    assert stopped_apart > 4
