"""GPU tests of the learned min-sum training kernels (ldpc_train_step): loss,
soft output and gradients against the FP64 CPU model (oracle/learned_ref.py),
the quantized forward pass against the int8 LDPC_LEARNED decoder, and what a
trained network gains over plain min-sum."""
import numpy as np
import pytest

from oracle import learned_ref, oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, LdpcError, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_regular

pytestmark = pytest.mark.gpu


def _gpu_step(code, llr, bits, kappa, alpha, beta, quantized, backward=True, kind="OMS", weights=None,
              frame_loss=False):
    import torch
    F = llr.shape[0]
    T = alpha.shape[0]
    dec = Decoder(code, kind, nb_frames=1)
    d = lambda x, dt: torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).cuda()
    d_llr, d_kappa = d(llr, np.float32), d(kappa, np.float32)
    d_bits = d(bits, np.uint8) if bits is not None else None
    d_a, d_b = d(alpha, np.float32), d(beta, np.float32)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    app = torch.zeros(F, code.n, dtype=torch.float32, device="cuda")
    ga = torch.zeros(T, 2, dtype=torch.float32, device="cuda") if backward else None
    gb = torch.zeros(T, 2, dtype=torch.float32, device="cuda") if backward else None
    stash = torch.empty(dec.train_stash_bytes(F, T), dtype=torch.uint8, device="cuda") if backward else None
    d_w = d(weights, np.float32) if weights is not None else None
    dec.train_step(d_llr, d_kappa, F, T, d_a, d_b, loss, d_bits=d_bits, quantized=quantized, d_grad_alpha=ga,
                   d_grad_beta=gb, d_stash=stash, d_app=app, d_weights=d_w, frame_loss=frame_loss)
    torch.cuda.synchronize()
    dec.close()
    out = [float(loss.item()), app.cpu().numpy()]
    out += [ga.cpu().numpy(), gb.cpu().numpy()] if backward else [None, None]
    return out


def _frames(code, F, sigma, seed, zero=False):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2, size=(F, code.n)).astype(np.uint8)
    if zero:   # the all-zero codeword (frames that can decode)
        bits[:] = 0
    y = (2.0 * bits - 1.0) + sigma * rng.standard_normal((F, code.n))
    return np.trunc(np.clip(8.0 * y, -31, 31)), bits, np.full(F, 1.0 / (4 * sigma * sigma))


@pytest.mark.parametrize("name,weighted,frame", [("576x288", False, False), ("1944x972", False, False),
                                                 ("qc", False, False), ("576x288", True, False), ("qc", True, False),
                                                 ("576x288", True, True), ("qc", False, True)])
def test_train_step_matches_fp64_model(cuda, name, weighted, frame):
    code = load_table(name) if name != "qc" else qc_regular(z=64, mb=8, nb=16, wc=3, seed=5)
    F, T = 12, 4
    llr, bits, kappa = _frames(code, F, 0.65 if frame else 0.9, 3, zero=frame)
    rng = np.random.default_rng(4)
    alpha = rng.uniform(0.6, 1.1, (T, 2)).astype(np.float32)
    beta = rng.uniform(-0.5, 1.5, (T, 2)).astype(np.float32)
    w = np.array([0.1, 0.2, 0.4, 1.0]) if weighted else None
    # forward: the FP32 emulation (one rounding per operation) is bit-exact;
    # loss and gradients: FP64 from the same decisions
    l_ref, app_ref, ga_ref, gb_ref = learned_ref.forward_backward(code, llr, bits, kappa, alpha, beta, weights=w,
                                                                  forward_dtype=np.float32, frame_loss=frame)
    l_gpu, app_gpu, ga, gb = _gpu_step(code, llr, bits, kappa, alpha, beta, False, weights=w, frame_loss=frame)
    assert np.array_equal(app_gpu.astype(np.float64), app_ref)
    assert l_gpu == pytest.approx(l_ref, rel=1e-5)
    scale = max(np.abs(ga_ref).max(), np.abs(gb_ref).max())
    assert scale > 1e-4
    # tolerance: FP32 accumulation over frames x rows x iterations (atomics in any order)
    assert np.abs(ga - ga_ref).max() <= 5e-4 * scale
    assert np.abs(gb - gb_ref).max() <= 5e-4 * scale


@pytest.mark.parametrize("name", ["4000x2000", "576x288"])
def test_quantized_train_forward_equals_int8_decoder(cuda, name):
    code = load_table(name)
    F, T = 16, 6
    llr, _, kappa = _frames(code, F, 0.85, 5)
    llr = np.where(np.random.default_rng(0).random(llr.shape) < 0.5, llr, -llr)   # mixed signs
    rng = np.random.default_rng(6)
    off = rng.integers(0, 3, (T, 2)).astype(np.int8)
    sc = rng.integers(90, 129, (T, 2)).astype(np.uint8)
    oracle.set_learned(off, sc)
    ref = oracle.decode(code, "LEARNED", llr.astype(np.int8), T, interleaved=False, want_state=True)
    _, app, _, _ = _gpu_step(code, llr, None, kappa, sc / 128.0, off.astype(np.float64), True, backward=False)
    W = F // 4
    ref_app = ref["app"].reshape(code.n, W, 4).transpose(1, 2, 0).reshape(F, code.n)
    assert np.array_equal(app.astype(np.int64), ref_app.astype(np.int64))


def test_train_step_argument_errors(cuda):
    import torch
    code = load_table("576x288")
    dec = Decoder(code, "OMS", nb_frames=1)
    x = torch.zeros(4, code.n, dtype=torch.float32, device="cuda")
    k = torch.ones(4, dtype=torch.float32, device="cuda")
    p = torch.ones(33, 2, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    with pytest.raises(LdpcError):
        dec.train_step(x, k, 4, 33, p, p, loss)                # too many iterations
    with pytest.raises(LdpcError):
        dec.train_step(x, k, 4, 2, p, p, loss, d_grad_alpha=p)  # gradients without a stash
    dec.close()


def test_training_gains_over_plain_min_sum(cuda):
    """What training gains: started from plain min-sum (scale 1, offset 0, the
    decoder without a learned correction), quantisation-aware training on
    channel frames finds constants whose FER at 2.0 dB is a small fraction of
    min-sum's and close to hand-tuned OMS (offset 1), the reference's best
    plain decoder, which stays the yardstick of FER."""
    from fast_ldpc_decoder_for_gpu_fixed_b200.learned import Trainer, evaluate
    code = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
    tr = Trainer(code, iters=10, batch=2048, sub=512, lr=0.01, seed=3, weights="all", init_alpha=1.0,
                 init_beta=0.0)
    v0 = tr.validation_loss(2.0)
    tr.train(2048 * 300, qat_fraction=1.0)
    v1 = tr.validation_loss(2.0)
    consts = tr.constants()
    tr.close()
    assert v1 < v0
    ms = evaluate(code, "MS", 10, 2.0, 131072)
    oms = evaluate(code, "OMS", 10, 2.0, 131072)
    learned = evaluate(code, "LEARNED", 10, 2.0, 131072, constants=consts)
    assert ms["frame_errors"] > 2000 and oms["frame_errors"] > 100
    assert learned["fer"] < ms["fer"] / 10
    assert learned["fer"] < 2.0 * oms["fer"]
