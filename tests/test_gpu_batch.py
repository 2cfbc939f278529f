"""Batches of several codes in one persistent launch (ldpc_batch_*): every code's
decisions and per-word iteration counts against the CPU oracle, for every
packing, with and without the early stop, graph capture and replay, the
autotuner, LDPC_LEARNED constants, and argument errors."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Batch, LdpcError, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_irregular

pytestmark = pytest.mark.gpu

_CODES = []


def codes():
    """The mixed-batch codes: four irregular QC codes, 24-column base, rates 1/2..5/6."""
    if not _CODES:
        for i, (z, rate) in enumerate(zip((27, 54, 81, 54), ((1, 2), (2, 3), (3, 4), (5, 6)))):
            _CODES.append(qc_irregular(z=z, rate=rate, seed=300 + i))
    return _CODES


def _inputs(cs, words, seed):
    import torch
    llrs, outs, its = [], [], []
    host = []
    for i, (c, w) in enumerate(zip(cs, words)):
        rate = c.n_info / c.n
        parts = [make_llr("awgn", 4 * c.n, seed + 10 * i + k, sigma=llr_gen.sigma_for(e, rate))
                 for k, e in zip(range(w), np.linspace(1.0, 4.0, w))]
        llr = np.concatenate(parts)
        host.append(llr)
        llrs.append(torch.from_numpy(llr).cuda())
        outs.append(torch.zeros(4 * w * c.n, dtype=torch.uint8, device="cuda"))
        its.append(torch.zeros(w, dtype=torch.int32, device="cuda"))
    return host, llrs, outs, its


def _check(cs, words, host, outs, its, kind, iters, early, batch=None):
    """Each code against the oracle; with `batch` in the per-code strategy, under the
    schedule of the kernel chosen for that code (flooding, or the 2-frame QC kernel's
    per-pair early stop)."""
    import torch
    torch.cuda.synchronize()
    per_code = batch is not None and batch.info()["per_code"]
    for i, (c, w, llr, o, it) in enumerate(zip(cs, words, host, outs, its)):
        kw = {}
        if per_code:
            ci = batch.code_info(i)
            kw["flooding"] = ci["candidate"] == "FLOODING"
            kw["pairs"] = ci["path"] in (4, 7) and early
        ref = oracle.decode(c, kind, llr, iters, interleaved=False, early_stop=early, **kw)
        assert np.array_equal(o.cpu().numpy().reshape(4 * w, c.n), ref["hard"]), (c.name, kw)
        assert np.array_equal(it.cpu().numpy(), ref["iters"]), (c.name, kw)


@pytest.mark.parametrize("early", [False, True])
@pytest.mark.parametrize("pack", ["SIMD4", "F16X2", "I8"])
def test_batch_matches_oracle(cuda, pack, early):
    cs = codes()
    words = [3, 1, 5, 2]
    host, llrs, outs, its = _inputs(cs, words, 1)
    b = Batch(cs, "OMS", pack=pack, early_stop=early)
    assert b.info()["pack"] == {"SIMD4": 0, "F16X2": 1, "I8": 2}[pack]
    b.decode(llrs, outs, words, 20, d_iters=its)
    _check(cs, words, host, outs, its, "OMS", 20, early)
    b.close()


def test_batch_graph_replay(cuda):
    import torch
    cs = codes()
    words = [2, 4, 1, 3]
    st = torch.cuda.Stream()
    host, llrs, outs, its = _inputs(cs, words, 2)
    b = Batch(cs, "OMS", early_stop=True, graph=True)
    with torch.cuda.stream(st):
        b.decode(llrs, outs, words, 20, d_iters=its, stream=st)
    st.synchronize()
    _check(cs, words, host, outs, its, "OMS", 20, True)
    # replay with new contents in the same buffers
    host2, llrs2, _, _ = _inputs(cs, words, 3)
    for a, h in zip(llrs, host2):
        a.copy_(torch.from_numpy(h))
    torch.cuda.synchronize()
    with torch.cuda.stream(st):
        b.decode(llrs, outs, words, 20, d_iters=its, stream=st)
    st.synchronize()
    _check(cs, words, host2, outs, its, "OMS", 20, True)
    # other sizes: captured again
    words3 = [1, 1, 2, 1]
    host3, llrs3, outs3, its3 = _inputs(cs, words3, 4)
    with torch.cuda.stream(st):
        b.decode(llrs3, outs3, words3, 20, d_iters=its3, stream=st)
    st.synchronize()
    _check(cs, words3, host3, outs3, its3, "OMS", 20, True)
    assert b.info()["graph"] == 1
    with pytest.raises(LdpcError):
        b.decode(llrs3, outs3, words3, 20)   # the legacy default stream cannot be captured
    b.close()


def test_batch_autotune(cuda):
    cs = codes()
    words = [8, 2, 6, 4]
    host, llrs, outs, its = _inputs(cs, words, 5)
    b = Batch(cs, "OMS", early_stop=True)
    ms = b.autotune(llrs, outs, words, 20, d_iters=its)
    info = b.info()
    assert ms > 0 and (info["per_code"] == 1 or (info["grid"] >= 148 // 2 and info["threads"] in (64, 128, 256)))
    for o in outs:
        o.zero_()
    b.decode(llrs, outs, words, 20, d_iters=its)
    _check(cs, words, host, outs, its, "OMS", 20, True, batch=b)
    b.close()


@pytest.mark.parametrize("cand", ["FLOODING", "QC", "QC_SPLIT"])
def test_batch_per_code_candidates(cuda, cand):
    """Every code on the flooding schedule, or on the QC register kernel, through the
    per-code strategy, against the oracle under that schedule."""
    from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib
    cs = codes()
    words = [3, 2, 4, 2]
    host, llrs, outs, its = _inputs(cs, words, 17)
    b = Batch(cs, "OMS", early_stop=True)
    b.configure(per_code=True, pack="SIMD4")
    took = 0
    for i in range(len(cs)):
        try:
            b.set_code_kernel_one(i, {"FLOODING": 4, "QC": 3, "QC_SPLIT": 5}[cand])
            took += 1
        except LdpcError as e:   # a QC shape without an instantiated register kernel
            assert cand.startswith("QC") and e.code == -3
    assert took >= (len(cs) if cand == "FLOODING" else 2)
    b.decode(llrs, outs, words, 20, d_iters=its)
    assert sum(b.code_info(i)["candidate"] == cand for i in range(len(cs))) == took
    _check(cs, words, host, outs, its, "OMS", 20, True, batch=b)
    b.close()


@pytest.mark.parametrize("strategy", ["persistent", "per_code"])
def test_batch_strategies(cuda, strategy):
    import torch
    cs = codes()
    words = [4, 3, 2, 5]
    st = torch.cuda.Stream()
    host, llrs, outs, its = _inputs(cs, words, 8)
    b = Batch(cs, "NMS", early_stop=True, graph=True)
    if strategy == "per_code":
        b.configure(per_code=True, pack="F16X2")
    else:
        b.configure(pack="I8", threads=96, ctas_per_sm=2)
    with torch.cuda.stream(st):
        b.decode(llrs, outs, words, 15, d_iters=its, stream=st)
    st.synchronize()
    _check(cs, words, host, outs, its, "NMS", 15, True)
    assert b.info()["per_code"] == (strategy == "per_code")
    b.close()


def test_batch_learned_and_tables(cuda):
    cs = codes()[:2] + [load_table("576x288"), load_table("1944x972")]
    words = [2, 2, 3, 1]
    off = np.array([[1, 2], [0, 1], [1, 0]], dtype=np.int8)
    sc = np.array([[128, 120], [112, 128], [120, 104]], dtype=np.uint8)
    oracle.set_learned(off, sc)
    host, llrs, outs, its = _inputs(cs, words, 6)
    for pack in ("SIMD4", "F16X2"):
        b = Batch(cs, "LEARNED", pack=pack, early_stop=True)
        b.set_learned(off, sc)
        b.decode(llrs, outs, words, 12, d_iters=its)
        _check(cs, words, host, outs, its, "LEARNED", 12, True)
        b.close()
    b = Batch(cs, "OMS", pack="I8")    # the reference tables' first-iteration quirk
    b.decode(llrs, outs, words, 12, d_iters=its)
    _check(cs, words, host, outs, its, "OMS", 12, False)
    b.close()


def test_batch_rejections(cuda):
    cs = codes()
    with pytest.raises(LdpcError):
        Batch(cs, "XMS")
    with pytest.raises(LdpcError):
        Batch(cs, "2NMS", early_stop=True)
    b = Batch(cs, "LEARNED")
    host, llrs, outs, its = _inputs(cs, [1, 1, 1, 1], 7)
    with pytest.raises(LdpcError):
        b.decode(llrs, outs, [1, 1, 1, 1], 5)   # constants not set
    b.close()
