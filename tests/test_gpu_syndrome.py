"""Per-frame syndrome flags (d_syndrome_ok of ldpc_decode_device, ldpc_batch_decode and
ldpc_decode_host_ex) on every decoder path.  The flag of a frame must be 1 exactly when
the oracle's hard decisions for it satisfy every check (code.syndrome == 0), whether the
frame stopped early on the syndrome, ran to the iteration limit or has no early stop.
The consumer this serves is the reference's error analyser, which can only compare
against the transmitted word (ber_analyzer/CErrorAnalyzer.cpp:142-158)."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Batch, Decoder, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import ira, qc_irregular, qc_regular

pytestmark = pytest.mark.gpu

_CACHE = {}


def _code(key):
    if key not in _CACHE:
        if key == "qc":
            _CACHE[key] = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
        elif key == "irr":
            _CACHE[key] = qc_irregular(z=27, rate=(5, 6), seed=527)
        elif key == "ira":
            _CACHE[key] = ira(n=14400, k=7200, seed=7)
        else:
            _CACHE[key] = load_table(key)
    return _CACHE[key]


def _mixed(code, words, seed, ebn0s, rate=0.5):
    """Frames at several noise levels interleaved frame by frame: in one word some frames
    converge and some do not."""
    per = -(-4 * words // len(ebn0s))
    parts = [make_llr("awgn", per * code.n, seed + i, sigma=llr_gen.sigma_for(e, rate)).reshape(per, code.n)
             for i, e in enumerate(ebn0s)]
    return np.ascontiguousarray(np.stack(parts, axis=1).reshape(-1, code.n)[:4 * words]).reshape(-1)


def _flags_of(code, hard):
    return (code.syndrome(hard).sum(axis=1) == 0).astype(np.uint8)


def _device(code, kind, llr, iters, words, pack="AUTO", early=False, packed=False):
    import torch
    dec = Decoder(code, kind, nb_frames=words, pack=pack, early_stop=early)
    path = dec.info()["path"]
    nb = (code.n + 7) // 8 if packed else code.n
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.zeros(4 * words * nb, dtype=torch.uint8, device="cuda")
    d_syn = torch.full((4 * words,), 7, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_out, words, iters, out_format=1 if packed else 0, d_syndrome=d_syn)
    torch.cuda.synchronize()
    dec.close()
    out = d_out.cpu().numpy().reshape(4 * words, nb)
    if packed:
        out = np.unpackbits(out, axis=1, bitorder="little")[:, :code.n]
    return path, out, d_syn.cpu().numpy()


# (code, kind, pack, early stop, expected path, Eb/N0 mix, iterations)
CASES = [
    ("4000x2000", "OMS", "SIMD4", False, 0, (1.0, 2.0, 3.0), 8),
    ("576x288", "NMS", "I8", True, 0, (1.0, 2.5, 4.0), 15),
    ("1944x972", "2NMS", "F16X2", False, 0, (1.0, 3.0), 20),
    ("4000x2000", "OMS", "AUTO", False, 2, (1.0, 2.0, 3.0), 6),
    ("qc", "OMS", "AUTO", False, 1, (1.5, 2.25, 3.0), 6),
    ("qc", "NMS", "AUTO", True, 1, (1.5, 2.25, 3.0), 10),
    ("irr", "OMS", "F16X2", False, 4, (2.5, 4.0, 6.0), 8),
    ("irr", "MS", "F16X2", True, 4, (2.5, 4.0, 6.0), 15),
    ("ira", "OMS", "FRAME", True, 3, (1.0, 1.6, 2.5), 25),
    ("576x288", "MS", "FRAME", False, 3, (1.0, 2.5), 5),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "%s-%s-%s-%s" % c[:4])
def test_syndrome_flags_every_path(cuda, case):
    name, kind, pack, early, want_path, ebn0s, iters = case
    code = _code(name)
    rate = code.n_info / code.n
    words = 12
    llr = _mixed(code, words, 90 + len(name), ebn0s, rate)
    path, hard, syn = _device(code, kind, llr, iters, words, pack=pack, early=early)
    assert path == want_path
    kw = {"early_stop": True} if early else {}
    if path == 3 and early:
        kw["per_frame"] = True
    if path == 4 and early:
        kw["pairs"] = True
    ref = oracle.decode(code, kind, llr, iters, **kw)
    assert np.array_equal(hard, ref["hard"])
    want = _flags_of(code, ref["hard"])
    assert np.array_equal(syn, want)
    assert 0 < want.sum() < want.size   # both outcomes occur


def test_syndrome_flags_per_frame_refill(cuda):
    """Path 5: frames stopped by their syndrome and frames stopped by the limit, packed output."""
    import torch
    code = _code("qc")
    words = 600  # more frames than the resident CTAs hold, so slots are refilled
    llr = _mixed(code, words, 71, (1.25, 2.0, 3.0))
    dec = Decoder(code, "OMS", nb_frames=words, early_stop="frame")
    assert dec.info()["path"] == 5
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.zeros(4 * words * code.n // 8, dtype=torch.uint8, device="cuda")
    d_syn = torch.full((4 * words,), 7, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_out, words, 12, out_format=1, d_syndrome=d_syn)
    torch.cuda.synchronize()
    dec.close()
    hard = np.unpackbits(d_out.cpu().numpy().reshape(4 * words, -1), axis=1, bitorder="little")
    ref = oracle.decode(code, "OMS", llr, 12, early_stop=True, per_frame=True)
    assert np.array_equal(hard, ref["hard"])
    want = _flags_of(code, ref["hard"])
    assert np.array_equal(d_syn.cpu().numpy(), want)
    assert 0 < want.sum() < want.size


def test_syndrome_flags_batch(cuda):
    import torch
    cs = [qc_irregular(z=27, rate=r, seed=300 + i) for i, r in enumerate(((1, 2), (3, 4), (5, 6)))]
    words = [5, 3, 4]
    llrs, outs, syns, host = [], [], [], []
    for i, (c, w) in enumerate(zip(cs, words)):
        x = _mixed(c, w, 200 + i, (1.5, 3.0, 5.0), c.n_info / c.n)
        host.append(x)
        llrs.append(torch.from_numpy(x).cuda())
        outs.append(torch.zeros(4 * w * c.n, dtype=torch.uint8, device="cuda"))
        syns.append(torch.full((4 * w,), 7, dtype=torch.uint8, device="cuda"))
    for per_code in (False, True):
        b = Batch(cs, "OMS", early_stop=True)
        b.configure(per_code=per_code, pack="SIMD4")
        b.decode(llrs, outs, words, 15, d_syndrome=syns)
        torch.cuda.synchronize()
        total = 0
        for c, w, x, o, s in zip(cs, words, host, outs, syns):
            ref = oracle.decode(c, "OMS", x, 15, early_stop=True)
            assert np.array_equal(o.cpu().numpy().reshape(4 * w, c.n), ref["hard"])
            want = _flags_of(c, ref["hard"])
            assert np.array_equal(s.cpu().numpy(), want)
            total += want.sum()
        assert 0 < total < 4 * sum(words)
        b.close()


@pytest.mark.parametrize("packed", [False, True])
def test_host_ex_packed_counts_and_flags(cuda, packed):
    """ldpc_decode_host_ex: the pipelined host call (several chunks) with packed or byte
    output, per-word iteration counts and per-frame flags, against the oracle."""
    code = _code("qc")
    words = 1024  # 4 chunks of 256 words
    llr = _mixed(code, words, 301, (1.5, 2.25, 3.0))
    dec = Decoder(code, "OMS", nb_frames=words, early_stop=True)
    nb = (code.n + 7) // 8 if packed else code.n
    out = np.zeros(4 * words * nb, dtype=np.uint8)
    its = np.full(words, -1, dtype=np.int32)
    syn = np.full(4 * words, 7, dtype=np.uint8)
    dec.decode_host_ex(llr, out, 10, out_format=1 if packed else 0, iters_out=its, syndrome_ok=syn)
    dec.close()
    hard = out.reshape(4 * words, nb)
    if packed:
        hard = np.unpackbits(hard, axis=1, bitorder="little")[:, :code.n]
    ref = oracle.decode(code, "OMS", llr, 10, early_stop=True)
    assert np.array_equal(hard, ref["hard"])
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(syn, _flags_of(code, ref["hard"]))
