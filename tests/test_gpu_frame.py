"""LDPC_PACK_FRAME (one frame per CTA, packed row state in shared memory): GPU decoders
against the CPU oracle for every kind it serves, with and without the
per-frame early stop, on the reference tables and on the long IRA code whose
state only this path can hold; the fused simulation and the plugin path."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, LdpcError, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import ira

pytestmark = pytest.mark.gpu


def _decode(code, kind, llr, iters, words, early=False, slack=None, constants=None):
    import torch
    dec = Decoder(code, kind, nb_frames=words, pack="FRAME", early_stop=early)
    if slack is not None:
        dec.set_early_stop(True, slack)
    if constants is not None:
        dec.set_learned(*constants)
    assert dec.info()["path"] == 3
    d_llr = torch.from_numpy(np.ascontiguousarray(llr)).cuda()
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(4 * words, dtype=torch.int32, device="cuda")
    dec.decode_device(d_llr, d_hard, words, iters, d_iters=d_it)
    torch.cuda.synchronize()
    assert dec.status() == 0   # no wait on the copy engine gave up
    dec.close()
    return d_hard.cpu().numpy().reshape(4 * words, code.n), d_it.cpu().numpy()


@pytest.mark.parametrize("kind", ["MS", "OMS", "NMS", "XMS"])
@pytest.mark.parametrize("name", ["4000x2000", "576x288", "1944x972"])
def test_frame_fixed_iterations(cuda, name, kind):
    code = load_table(name)
    words = 6
    llr = make_llr("awgn", 4 * words * code.n, 3, sigma=llr_gen.sigma_for(1.5, 0.5))
    ref = oracle.decode(code, kind, llr, 12)
    hard, its = _decode(code, kind, llr, 12, words)
    assert np.array_equal(hard, ref["hard"])
    assert (its == 12).all()


@pytest.mark.parametrize("slack", [0, 128])
@pytest.mark.parametrize("name", ["576x288", "1944x972"])
def test_frame_early_stop_per_frame(cuda, name, slack):
    code = load_table(name)
    words = 12
    llr = np.concatenate([make_llr("awgn", 4 * 4 * code.n, 7 + i, sigma=llr_gen.sigma_for(e, 0.5))
                          for i, e in enumerate((1.0, 2.5, 4.0))])
    ref = oracle.decode(code, "OMS", llr, 25, early_stop=True, early_slack=slack, per_frame=True)
    hard, its = _decode(code, "OMS", llr, 25, words, early=True, slack=slack)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])
    assert len(set(its.tolist())) > 3


@pytest.mark.parametrize("llr_kind", ["uniform", "extreme"])
@pytest.mark.parametrize("kind", ["MS", "OMS", "NMS", "LEARNED"])
def test_frame_saturated_inputs(cuda, kind, llr_kind):
    """Every int8 value (uniform) or the saturation edges -128/127 with many ties
    (extreme): the wrapped |-128|, equal minima and odd row degrees (a dummy edge in
    the last fp16 pair) on the 4000x2000 table (degrees 6 and 7)."""
    code = load_table("4000x2000")
    words = 6
    llr = make_llr(llr_kind, 4 * words * code.n, 19)
    constants = None
    if kind == "LEARNED":
        constants = (np.array([[1, -2], [0, 3]], dtype=np.int8), np.array([[200, 128], [96, 71]], dtype=np.uint8))
        oracle.set_learned(*constants)
    ref = oracle.decode(code, kind, llr, 8)
    hard, _ = _decode(code, kind, llr, 8, words, constants=constants)
    assert np.array_equal(hard, ref["hard"])


def test_frame_learned(cuda):
    code = load_table("1944x972")
    words = 4
    off = np.array([[1, 2], [1, 1], [0, 1]], dtype=np.int8)
    sc = np.array([[128, 120], [112, 128], [120, 104]], dtype=np.uint8)
    oracle.set_learned(off, sc)
    llr = make_llr("awgn", 4 * words * code.n, 9, sigma=llr_gen.sigma_for(1.75, 0.5))
    ref = oracle.decode(code, "LEARNED", llr, 10)
    hard, _ = _decode(code, "LEARNED", llr, 10, words, constants=(off, sc))
    assert np.array_equal(hard, ref["hard"])


def test_long_ira_code_takes_the_frame_path(cuda):
    code = ira()   # N = 64800: the 4-frame state does not fit in shared memory
    words = 2
    dec = Decoder(code, "OMS", nb_frames=words, early_stop=True)
    assert dec.info()["path"] == 3
    dec.close()
    llr = make_llr("awgn", 4 * words * code.n, 11, sigma=llr_gen.sigma_for(1.2, 0.5))
    ref = oracle.decode(code, "OMS", llr, 30, early_stop=True, per_frame=True)
    hard, its = _decode(code, "OMS", llr, 30, words, early=True)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])
    stopped = its < 30          # frames that stopped early hold codewords
    assert stopped.sum() >= 4 and (code.syndrome(hard[stopped]) == 0).all()


def test_frame_fused_simulation(cuda):
    import torch
    code = load_table("1944x972")
    words = 16
    dec = Decoder(code, "OMS", nb_frames=words, pack="FRAME", early_stop=True)
    d_hard = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    dec.simulate(words, 20, 0.85, 3, 1, counts, d_hard=d_hard, n_vars=code.n)
    torch.cuda.synchronize()
    dec.close()
    llr, _ = oracle.awgn(4 * words, code.n, 0.85, 3, 1)
    ref = oracle.decode(code, "OMS", llr, 20, early_stop=True, per_frame=True)
    assert np.array_equal(d_hard.cpu().numpy().reshape(4 * words, code.n), ref["hard"])
    be, fe, _ = oracle.count_errors(code.n, code.n, ref["hard"])
    assert counts.cpu().tolist() == [4 * words, be, fe]


def test_frame_host_decode(cuda):
    code = load_table("576x288")
    words = 40
    llr = make_llr("awgn", 4 * words * code.n, 13, sigma=llr_gen.sigma_for(1.5, 0.5))
    dec = Decoder(code, "OMS", nb_frames=words, pack="FRAME")
    hard = np.zeros((4 * words, code.n), dtype=np.uint8)
    dec.decode_host(llr.reshape(4 * words, code.n), hard, 15)
    dec.close()
    assert np.array_equal(hard, oracle.decode(code, "OMS", llr, 15)["hard"])


def test_frame_rejections(cuda):
    import torch
    code = load_table("576x288")
    with pytest.raises(LdpcError):
        Decoder(code, "2NMS", nb_frames=4, pack="FRAME")
    dec = Decoder(code, "OMS", nb_frames=4, pack="FRAME")
    d = torch.zeros(16 * code.n, dtype=torch.int8, device="cuda")
    h = torch.zeros(16 * code.n, dtype=torch.uint8, device="cuda")
    with pytest.raises(LdpcError):
        dec.decode_device_state(d, h, 4, 5, d_app=d)
    dec.close()


def test_reference_long_table(cuda):
    """The reference's 64800x32400 table (its table order is a serial schedule)
    decodes on the one-frame-per-CTA path exactly like the oracle."""
    code = load_table("64800x32400")
    words = 2
    llr = make_llr("awgn", 4 * words * code.n, 17, sigma=llr_gen.sigma_for(1.5, 0.5))
    ref = oracle.decode(code, "OMS", llr, 3)
    dec = Decoder(code, "OMS", nb_frames=words)
    assert dec.info()["path"] == 3
    dec.close()
    hard, _ = _decode(code, "OMS", llr, 3, words)
    assert np.array_equal(hard, ref["hard"])


def _small_code(name, rows, n, seed):
    """A code whose rows are the given column lists (layer order)."""
    from fast_ldpc_decoder_for_gpu_fixed_b200.codes import Code
    ptr = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    return Code(name, n, ptr, np.concatenate(rows).astype(np.int32))


@pytest.mark.parametrize("shape", ["one_level", "three_levels", "split_level"])
def test_frame_few_stages(cuda, shape):
    """Schedules of fewer than four stages (each stage issued when it starts, no copy
    ahead) and a level wider than the CTA (cut into stages of at most 512 rows)."""
    rng = np.random.default_rng(5)
    if shape == "one_level":      # 12 disjoint rows of degree 5..7: one level, one stage
        n, rows, start = 96, [], 0
        for d in rng.integers(5, 8, size=12):
            rows.append(np.arange(start, start + d))
            start += d
    elif shape == "three_levels":  # a chain: row i shares a variable with row i-1
        n = 64
        rows = [np.array([0, 1, 2, 3, 4, 5]), np.array([5, 6, 7, 8, 9, 10, 11]), np.array([11, 12, 13, 14, 15])]
    else:                          # 1000 disjoint rows of degree 3 and 4: one level of 1000 rows
        degs = rng.integers(3, 5, size=1000)
        n = int(degs.sum()) + 8
        rows, start = [], 0
        for d in degs:
            rows.append(rng.permutation(np.arange(start, start + d)))
            start += d
    code = _small_code(shape, rows, n, 5)
    words = 8
    llr = make_llr("uniform", 4 * words * code.n, 23)
    for kind in ("OMS", "NMS"):
        ref = oracle.decode(code, kind, llr, 6)
        hard, its = _decode(code, kind, llr, 6, words)
        assert np.array_equal(hard, ref["hard"])
        assert (its == 6).all()


def test_frame_many_frames_per_cta(cuda):
    """More frames than resident CTAs (each persistent CTA decodes several frames in a
    row, the copies it issued ahead for a frame that stopped early are drained first),
    mixed noise so that frames stop at many different iterations."""
    code = load_table("576x288")
    words = 240  # 960 frames, about three per CTA
    llr = np.concatenate([make_llr("awgn", 4 * 80 * code.n, 29 + i, sigma=llr_gen.sigma_for(e, 0.5))
                          for i, e in enumerate((1.0, 2.5, 4.0))])
    ref = oracle.decode(code, "OMS", llr, 20, early_stop=True, per_frame=True)
    hard, its = _decode(code, "OMS", llr, 20, words, early=True)
    assert np.array_equal(its, ref["iters"])
    assert np.array_equal(hard, ref["hard"])
    assert len(set(its.tolist())) > 5
