"""LDPC_LEARNED (per-iteration int8 offsets, Q1.7 scales): GPU decoders against
the CPU oracle with the same constants, for every packing and the QC kernel."""
import numpy as np
import pytest

import llr_gen
from gpu_helpers import assert_same, gpu_decode, make_llr
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, LdpcError, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_regular

pytestmark = pytest.mark.gpu


def _tables(its, seed, step=1):
    """Random constants; step=8 puts the scales on the 1/16 grid the fp16 kernels take."""
    rng = np.random.default_rng(seed)
    off = rng.integers(0, 4, size=(its, 2)).astype(np.int8)
    sc = (rng.integers(72 // step, 128 // step + 1, size=(its, 2)) * step).astype(np.uint8)
    return off, sc


def _gpu(code, llr, iters, words, pack, off, sc):
    import torch
    dec = Decoder(code, "LEARNED", nb_frames=words, pack=pack)
    dec.set_learned(off, sc)
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_out, words, iters, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    info = dec.info()
    dec.close()
    return d_out.cpu().numpy().reshape(4 * words, code.n), info


@pytest.mark.parametrize("pack", ["SIMD4", "F16X2", "I8"])
@pytest.mark.parametrize("name", ["4000x2000", "576x288", "1944x972"])
def test_learned_level_kernels(cuda, name, pack):
    code = load_table(name)
    words = 8
    off, sc = _tables(7, 3, step=8 if pack == "F16X2" else 1)
    oracle.set_learned(off, sc)
    for inp in ("awgn", "uniform"):
        llr = make_llr(inp, 4 * words * code.n, 5, sigma=llr_gen.sigma_for(1.5, 0.5))
        got, _ = _gpu(code, llr, 12, words, pack, off, sc)
        ref = oracle.decode(code, "LEARNED", llr, 12, interleaved=False)["hard"]
        assert np.array_equal(got, ref)


def test_learned_qc_kernel(cuda):
    code = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
    words = 10
    off, sc = _tables(10, 4, step=8)
    oracle.set_learned(off, sc)
    llr = make_llr("awgn", 4 * words * code.n, 6, sigma=llr_gen.sigma_for(1.5, 0.5))
    got, info = _gpu(code, llr, 10, words, "AUTO", off, sc)
    assert info["path"] == 1
    assert np.array_equal(got, oracle.decode(code, "LEARNED", llr, 10, interleaved=False)["hard"])


def test_learned_equals_oms_without_quirk(cuda):
    code = load_table("4000x2000")   # single row group: no first-iteration quirk, so LEARNED(1.0, 1) = OMS
    words = 6
    llr = make_llr("awgn", 4 * words * code.n, 7, sigma=llr_gen.sigma_for(1.5, 0.5))
    got, _ = _gpu(code, llr, 20, words, "F16X2", np.ones((1, 2)), np.full((1, 2), 128))
    ref = gpu_decode(code, "OMS", llr, 20, words, pack="F16X2", state=False)["hard"]
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("early", [False, True])
def test_learned_oms_constants_on_the_qc_kernel(cuda, early):
    """Constants equal to OMS's (scale 1.0, offset 1 in every iteration and group) run the OMS
    QC kernel with the first-iteration quirk off (a QC code has one row group, so the quirk
    never applies there anyway): decisions and iteration counts equal the oracle's LEARNED
    decode with those constants."""
    import torch
    code = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
    words = 12
    off, sc = np.ones((10, 2), dtype=np.int8), np.full((10, 2), 128, dtype=np.uint8)
    oracle.set_learned(off, sc)
    llr = make_llr("awgn", 4 * words * code.n, 8, sigma=llr_gen.sigma_for(2.25, 0.5))
    dec = Decoder(code, "LEARNED", nb_frames=words, early_stop=early)
    dec.set_learned(off, sc)
    assert dec.info()["path"] == 1
    d_llr = torch.from_numpy(llr).cuda()
    d_out = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(words, dtype=torch.int32, device="cuda")
    dec.decode_device(d_llr, d_out, words, 10, d_iters=d_it)
    torch.cuda.synchronize()
    dec.close()
    ref = oracle.decode(code, "LEARNED", llr, 10, interleaved=False, early_stop=early)
    assert np.array_equal(d_out.cpu().numpy().reshape(4 * words, code.n), ref["hard"])
    assert np.array_equal(d_it.cpu().numpy(), ref["iters"])
    if early:
        assert len(set(ref["iters"].tolist())) > 1


def test_learned_requires_constants(cuda):
    import torch
    code = load_table("576x288")
    dec = Decoder(code, "LEARNED", nb_frames=2)
    d = torch.zeros(8 * code.n, dtype=torch.int8, device="cuda")
    with pytest.raises(LdpcError):
        dec.decode_device(d, d, 2, 5)
    with pytest.raises(LdpcError):
        dec.set_learned(np.zeros((33, 2)), np.zeros((33, 2)))


def test_fp16_learned_needs_the_sixteenth_grid(cuda):
    code = load_table("576x288")
    dec = Decoder(code, "LEARNED", nb_frames=2, pack="F16X2")
    with pytest.raises(LdpcError) as e:
        dec.set_learned(np.ones((2, 2)), np.full((2, 2), 100))
    assert e.value.code == -3
    with pytest.raises(LdpcError):
        dec.set_learned(np.full((2, 2), 40), np.full((2, 2), 128))
    dec.set_learned(np.full((2, 2), -31), np.full((2, 2), 248))
    dec.close()
    dec = Decoder(code, "LEARNED", nb_frames=2, pack="SIMD4")
    dec.set_learned(np.ones((2, 2)), np.full((2, 2), 100))   # tables take any constants
    dec.close()


def test_fp16_learned_extreme_constants(cuda):
    """The arithmetic fp16 magnitude against the oracle's table at the corners of its range."""
    code = load_table("1944x972")
    words = 6
    off = np.array([[-31, 31], [0, -5], [3, 0], [-1, 1]], dtype=np.int8)
    sc = np.array([[248, 8], [128, 200], [64, 136], [240, 96]], dtype=np.uint8)
    oracle.set_learned(off, sc)
    llr = make_llr("uniform", 4 * words * code.n, 21)
    got, _ = _gpu(code, llr, 9, words, "F16X2", off, sc)
    assert np.array_equal(got, oracle.decode(code, "LEARNED", llr, 9, interleaved=False)["hard"])
