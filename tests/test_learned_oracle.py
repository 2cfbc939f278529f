"""CPU tests of the FP64 learned min-sum model (oracle/learned_ref.py): its
analytic gradients against central finite differences, its quantized forward
pass against the int8 LDPC_LEARNED oracle, and the constant quantiser."""
import numpy as np
import pytest

from oracle import learned_ref, oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.learned import quantize
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_regular


def _llr(rng, frames, n, sigma):
    y = -1.0 + sigma * rng.standard_normal((frames, n))
    return np.trunc(np.clip(8.0 * y, -31, 31))


@pytest.mark.parametrize("name,weighted,frame", [("576x288", False, False), ("qc", False, False),
                                                 ("576x288", True, False), ("576x288", True, True),
                                                 ("qc", False, True)])
def test_gradients_match_finite_differences(name, weighted, frame):
    code = load_table(name) if name != "qc" else qc_regular(z=16, mb=8, nb=16, wc=3, seed=3)
    rng = np.random.default_rng(1)
    F, T = 6, 3
    sigma = 0.65 if frame else 0.9   # the frame loss needs frames close to decoding
    llr = _llr(rng, F, code.n, sigma)
    bits = rng.integers(0, 2, size=(F, code.n))
    llr = np.where(bits == 1, -llr, llr)   # the transmitted bits flip the BPSK sign
    if frame:   # the frame loss needs frames that can decode: send the all-zero codeword
        bits[:] = 0
        llr = _llr(np.random.default_rng(1), F, code.n, sigma)
    kappa = np.full(F, 1.0 / (4 * sigma * sigma))
    alpha = rng.uniform(0.6, 1.0, (T, 2))
    beta = rng.uniform(0.2, 1.5, (T, 2))
    w = np.array([0.25, 0.5, 1.0]) if weighted else None
    loss, app, da, db = learned_ref.forward_backward(code, llr, bits, kappa, alpha, beta, weights=w,
                                                     frame_loss=frame)
    assert np.abs(app).max() < 127          # no saturation: the model is smooth here
    eps = 1e-6
    f = lambda a, b: learned_ref.forward_backward(code, llr, bits, kappa, a, b, backward=False, weights=w,
                                                  frame_loss=frame)[0]
    assert np.abs(da).max() > 1e-3 and np.abs(db).max() > 1e-3
    used = sorted(set(code.row_class.tolist()))
    for t in range(T):
        for g in used:
            e = np.zeros((T, 2))
            e[t, g] = eps
            fd_a = (f(alpha + e, beta) - f(alpha - e, beta)) / (2 * eps)
            fd_b = (f(alpha, beta + e) - f(alpha, beta - e)) / (2 * eps)
            assert fd_a == pytest.approx(da[t, g], rel=1e-5, abs=1e-9)
            assert fd_b == pytest.approx(db[t, g], rel=1e-5, abs=1e-9)
    for g in set((0, 1)) - set(used):
        assert (da[:, g] == 0).all() and (db[:, g] == 0).all()


@pytest.mark.parametrize("name", ["576x288", "1944x972", "4000x2000"])
def test_quantized_forward_is_the_int8_learned_decoder(name):
    code = load_table(name)
    rng = np.random.default_rng(2)
    F, T = 8, 4
    off = rng.integers(-1, 3, (T, 2)).astype(np.int8)
    sc = rng.integers(80, 140, (T, 2)).astype(np.uint8)
    oracle.set_learned(off, sc)
    llr = _llr(rng, F, code.n, 0.95).astype(np.int8)
    ref = oracle.decode(code, "LEARNED", llr, T, interleaved=False, want_state=True)
    _, app, _, _ = learned_ref.forward_backward(code, llr.astype(np.float64), None, np.ones(F), sc / 128.0,
                                                off.astype(np.float64), quantized=True, backward=False)
    assert np.array_equal((app > 0).astype(np.uint8), ref["hard"])
    W = F // 4
    ref_app = ref["app"].reshape(code.n, W, 4).transpose(1, 2, 0).reshape(F, code.n)
    assert np.array_equal(app.astype(np.int64), ref_app.astype(np.int64))


def test_quantize_rounds_and_saturates():
    off, sc = quantize([[1.0, 0.5], [2.5, -0.1]], [[0.6, -200.0], [1.49, 300.0]], scale_step=1)
    assert off.tolist() == [[1, -31], [1, 31]]
    assert sc.tolist() == [[128, 64], [255, 0]]
    _, sc8 = quantize([[0.96, 0.91], [2.5, 0.0]], [[0, 0], [0, 0]])   # the fp16 kernels' 1/16 grid
    assert sc8.tolist() == [[120, 120], [248, 0]]


def test_float32_forward_stays_close_to_float64():
    code = load_table("576x288")
    rng = np.random.default_rng(5)
    llr = _llr(rng, 4, code.n, 0.9)
    args = (code, llr, None, np.ones(4), np.full((3, 2), 0.8), np.full((3, 2), 0.3))
    l64, a64, _, _ = learned_ref.forward_backward(*args, backward=False)
    l32, a32, _, _ = learned_ref.forward_backward(*args, backward=False, forward_dtype=np.float32)
    assert a32.dtype == np.float64 and np.abs(a32 - a64).max() < 1e-3
    assert l32 == pytest.approx(l64, rel=1e-5)
