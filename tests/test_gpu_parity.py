"""GPU parity: the sm_100a decoder (through the C ABI) against the CPU oracle.

Bit-exact on every output: hard decisions, final APP and final messages in the
reference's device layouts, and iterations executed per word (2NMS early
termination).  Inputs cover the reference channel's value range and the whole
int8 range (saturations, |-128| wrap), every plugin kind, every frame packing.
"""
import numpy as np
import pytest

from gpu_helpers import assert_same, gpu_decode, make_llr, oracle_decode, table
import llr_gen

pytestmark = pytest.mark.gpu

CODES = ["4000x2000", "576x288", "1944x972", "2304x1152", "1024x518", "816x408", "2048x384", "9972x4986"]
KINDS = ["MS", "OMS", "NMS", "2NMS", "XMS"]
PACKS = ["SIMD4", "F16X2", "I8"]


def _inputs(code, words, seed):
    rate = code.n_info / code.n
    count = 4 * words * code.n
    return {
        "awgn": make_llr("awgn", count, seed, sigma=llr_gen.sigma_for(2.0, rate)),
        "uniform": make_llr("uniform", count, seed + 1),
    }


@pytest.mark.parametrize("name", CODES)
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("pack", PACKS)
def test_parity_reference_tables(cuda, name, kind, pack):
    code = table(name)
    words = 8
    for inp, llr in _inputs(code, words, 100 + CODES.index(name)).items():
        gpu = gpu_decode(code, kind, llr, 20, words, pack=pack)
        ref = oracle_decode(code, kind, llr, 20)
        assert_same(gpu, ref)


@pytest.mark.parametrize("iters", [1, 2, 3, 7])
@pytest.mark.parametrize("pack", PACKS)
def test_parity_iteration_counts(cuda, iters, pack):
    code = table("576x288")  # two degree groups: exercises the OMS first-iteration quirk
    llr = make_llr("uniform", 4 * 16 * code.n, 7 + iters)
    for kind in KINDS:
        assert_same(gpu_decode(code, kind, llr, iters, 16, pack=pack), oracle_decode(code, kind, llr, iters))


@pytest.mark.parametrize("value", [-128, -127, -1, 0, 1, 31, 127])
def test_parity_constant_inputs(cuda, value):
    code = table("4000x2000")
    llr = make_llr("const", 4 * 4 * code.n, 0, value=value)
    for pack in PACKS:
        for kind in KINDS:
            assert_same(gpu_decode(code, kind, llr, 5, 4, pack=pack), oracle_decode(code, kind, llr, 5))


@pytest.mark.parametrize("words", [1, 3, 33, 130])
def test_parity_ragged_batches(cuda, words):
    code = table("1944x972")
    llr = make_llr("extreme", 4 * words * code.n, 55 + words)
    for pack in PACKS:
        for kind in ("OMS", "2NMS", "XMS"):
            assert_same(gpu_decode(code, kind, llr, 12, words, pack=pack), oracle_decode(code, kind, llr, 12))


def test_parity_early_termination_varies(cuda):
    """2NMS at high SNR: words stop at different iterations; counts must match."""
    code = table("4000x2000")
    words = 64
    llr = make_llr("awgn", 4 * words * code.n, 99, sigma=llr_gen.sigma_for(3.0, 0.5))
    for pack in PACKS:
        gpu = gpu_decode(code, "2NMS", llr, 30, words, pack=pack)
        ref = oracle_decode(code, "2NMS", llr, 30)
        assert_same(gpu, ref)
    assert len(set(ref["iters"].tolist())) > 1, "test input should stop at several different iterations"


def test_odd_length_code(cuda):
    """n not a multiple of 4 (byte-wise prologue/epilogue path), irregular rows."""
    from fast_ldpc_decoder_for_gpu_fixed_b200 import Code
    rng = np.random.default_rng(3)
    n, m = 203, 90
    rows = [sorted(rng.choice(n, size=int(rng.integers(3, 9)), replace=False).tolist()) for _ in range(m)]
    code = Code.from_rows("odd203", n, rows)
    llr = make_llr("uniform", 4 * 5 * n, 4)
    for pack in PACKS:
        for kind in KINDS:
            assert_same(gpu_decode(code, kind, llr, 9, 5, pack=pack), oracle_decode(code, kind, llr, 9))
