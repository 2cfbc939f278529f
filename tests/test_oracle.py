"""CPU checks of the oracle itself: the batched AVX2 decoder equals the scalar
restatement, layouts round-trip, the error analyser and channel quantiser
restatements behave as the reference code reads, and hand-built check rows
give the values the reference's byte arithmetic gives."""
import numpy as np
import pytest

import llr_gen
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Code, load_table


@pytest.mark.parametrize("isa", ["best", "avx2"])
@pytest.mark.parametrize("name", ["4000x2000", "576x288", "1944x972", "2048x384"])
@pytest.mark.parametrize("kind", ["MS", "OMS", "NMS", "XMS"])
def test_batch_equals_scalar(name, kind, isa):
    """Both vector paths (AVX-512BW 64-frame groups where the CPU has it, and AVX2);
    96 frames = one 64-frame group plus a 32-frame tail on the AVX-512BW path."""
    if not oracle.batch_supported():
        pytest.skip("host without AVX2")
    code = load_table(name)
    llr = llr_gen.llr("uniform", 96 * code.n, 3)
    a = oracle.decode(code, kind, llr, 7)["hard"]
    oracle.force_avx2(isa == "avx2")
    try:
        b = oracle.decode_batch(code, kind, llr, 7)
    finally:
        oracle.force_avx2(False)
    assert np.array_equal(a, b)


def test_batch_isa_reported():
    assert oracle.batch_isa() in ("avx512bw", "avx2", None)
    assert oracle.cpu_model() is None or isinstance(oracle.cpu_model(), str)


def test_interleave_roundtrip():
    n, W = 40, 8
    x = llr_gen.llr("uniform", 4 * W * n, 1)
    words = oracle.interleave(n, W, x)
    # word (v, g) byte k = frame 4g+k, variable v
    f, v = 4 * 3 + 2, 17
    assert words[(v * W + 3) * 4 + 2] == x[f * n + v]
    hd = oracle.deinterleave_hd(n, W, words)
    assert np.array_equal(hd.reshape(-1), (x > 0).astype(np.uint8))


def test_count_errors():
    n, nv = 10, 6
    hard = np.zeros((3, n), dtype=np.uint8)
    hard[1, 2] = 1
    hard[1, 7] = 1   # beyond the first n_vars bytes: not counted (CErrorAnalyzer.cpp:147-150)
    hard[2, 0:3] = 1
    be, fe, per = oracle.count_errors(n, nv, hard)
    assert (be, fe) == (4, 2)
    assert per.tolist() == [0, 1, 3]


def test_quantizer_and_sigma():
    q = oracle.lib().oracle_quantize
    assert q(0.0, 1.0) == -8            # -1 * 8
    assert q(10.0, 1.0) == 31           # clipped
    assert q(-10.0, 1.0) == -31
    assert q(0.9, 1.0) == 0             # -0.8 truncates to 0
    assert q(0.85, 1.0) == -1           # 8 * -0.15 = -1.2 -> -1
    assert abs(oracle.sigma(0.0, 0.5) - 1.0) < 1e-12   # R = 1/2, Eb/N0 = 0 dB -> sigma = 1
    assert abs(oracle.sigma(3.0, 0.5) - 10 ** (-0.15)) < 1e-12


def _one_row(vals, kind, iters=1, cls=0):
    """Decode a single check row over len(vals) variables; returns (app, msg) of frame 0."""
    d = len(vals)
    code = Code("row", d, np.array([0, d]), np.arange(d), np.array([cls], dtype=np.uint8))
    llr = np.zeros((4, d), dtype=np.int8)
    llr[0] = vals
    out = oracle.decode(code, kind, llr.reshape(-1), iters, interleaved=False, want_state=True)
    app = out["app"].reshape(d, 1, 4)[:, 0, 0]
    msg = out["msg"].reshape(d, 1, 4)[:, 0, 0]
    return app.astype(int).tolist(), msg.astype(int).tolist()


def test_check_node_known_answers():
    # OMS: min1 = 3 (edge 1), min2 = 5 -> c1 = 4 (to edge 1), c2 = 2; signs: positives {0, 2}
    app, msg = _one_row([5, -3, 9, -20], "OMS")
    # edge0: others' positives = {2} -> odd -> +c2 = 2 ; edge1: {0,2} even -> -c1 = -4
    # edge2: {0} odd -> +2 ; edge3: {0,2} even -> -2
    assert msg == [2, -4, 2, -2]
    assert app == [7, -7, 11, -22]
    # MS on the same row: no offset
    _, msg = _one_row([5, -3, 9, -20], "MS")
    assert msg == [3, -5, 3, -3]
    # ties at the minimum: both minimum edges get min2 = min1
    _, msg = _one_row([-4, -4, -9], "MS")
    assert msg == [-4, -4, -4]           # no positive edge: every extrinsic sign is "0" -> negative
    # clip at 31 (MS) and saturation of APP
    app, msg = _one_row([100, 120, 127, 110], "MS")
    assert msg == [31, 31, 31, 31] and app == [127, 127, 127, 127]
    # zero counts as "not positive"
    _, msg = _one_row([0, 6, 7], "MS")
    assert msg == [-6, 0, 0]
    # -128: |t| wraps to 128 > 127, never the minimum; min1 stays at the initial 127
    _, msg = _one_row([-128, -128, -128], "NMS")
    assert msg == [-95, -95, -95]        # floor(127*0.75) = 95, all edges "not minimum"
    # NMS / 2NMS scaling truncation
    _, msg = _one_row([-10, -13, -40], "NMS")
    assert msg == [-9, -7, -7]           # floor(13*.75)=9 to edge0, floor(10*.75)=7 to others
    _, msg = _one_row([-10, -13, -40], "2NMS")
    assert msg == [-11, -7, -7]          # floor(13*.875)=11
    # OMS min 0: offset saturates at 0
    _, msg = _one_row([0, 0, 5], "OMS")
    assert msg == [0, 0, 0]


def test_oms_first_iteration_quirk():
    """Second-degree-group rows skip the 31-clip in OMS's first iteration only
    (decoder_oms/cuda/CUDA_OMS_SIMD.cu:115-116); MS and xMS never skip it."""
    _, msg = _one_row([-100, -90, -80], "OMS", cls=1)
    assert msg == [-79, -79, -89]
    _, msg = _one_row([-100, -90, -80], "OMS", cls=0)
    assert msg == [-31, -31, -31]
    _, msg = _one_row([-100, -90, -80], "XMS", cls=1)
    assert msg == [-31, -31, -31]


def test_layered_order_matters():
    """Rows update APP in place: the second row sees the first row's result."""
    code = Code("two", 3, np.array([0, 2, 4]), np.array([0, 1, 1, 2]))
    llr = np.zeros((4, 3), dtype=np.int8)
    llr[0] = [10, -2, 20]
    out = oracle.decode(code, "MS", llr.reshape(-1), 1, interleaved=False, want_state=True)
    app = out["app"].reshape(3, 1, 4)[:, 0, 0].tolist()
    # row0: t=(10,-2): msgs (-2, 10) -> app (8, 8); row1 over (v1=8, v2=20): msgs (20->min 20, 8) -> (28, 28)
    assert app == [8, 28, 28]


@pytest.mark.parametrize("kind", ["OMS", "NMS"])
def test_early_stop_groups_agree_on_copied_frames(kind):
    """The early-stop groupings (per frame, per frame pair, per 4-frame word) agree when a
    group's frames are copies of one frame and the slack scales with the group: the group's
    odd-row count is then the frame's times the group size and its syndrome is the
    frame's, so every frame stops at the same iteration in all three modes."""
    code = load_table("576x288")
    frames = 48
    base = np.concatenate([llr_gen.llr("awgn", frames * code.n // 3, 31 + i, sigma=llr_gen.sigma_for(e, 0.5))
                           for i, e in enumerate((1.5, 2.5, 4.0))]).reshape(frames, code.n)
    for slack in (0, 5, 40):
        per_frame = oracle.decode(code, kind, base.reshape(-1), 25, early_stop=True, early_slack=slack,
                                  per_frame=True)
        words = np.repeat(base, 4, axis=0)                     # word g = 4 copies of frame g
        per_word = oracle.decode(code, kind, words.reshape(-1), 25, early_stop=True, early_slack=4 * slack)
        assert np.array_equal(per_word["iters"], per_frame["iters"])
        assert np.array_equal(per_word["hard"][::4], per_frame["hard"])
        pairs = np.repeat(base, 2, axis=0)                     # pair p = 2 copies of frame p
        per_pair = oracle.decode(code, kind, pairs.reshape(-1), 25, early_stop=True, early_slack=2 * slack,
                                 pairs=True)
        assert np.array_equal(per_pair["iters"], np.maximum(per_frame["iters"][0::2], per_frame["iters"][1::2]))
        assert np.array_equal(per_pair["hard"][::2], per_frame["hard"])
    assert len(set(per_frame["iters"].tolist())) > 3
