"""GPU tests of the public entry points: host-buffer decode (the reference
plugins' decode()), device decode with both output formats, the Python plugin
mirrors, error statuses, and an exhaustive check of the per-byte SIMD
operations the SIMD4 packing uses against the oracle's byte semantics."""
import ctypes

import numpy as np
import pytest

import llr_gen
from gpu_helpers import gpu_decode, make_llr, oracle_decode, table
from oracle import oracle
import fast_ldpc_decoder_for_gpu_fixed_b200 as fl
from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["MS", "OMS", "NMS", "2NMS", "XMS"])
def test_decode_host_matches_oracle(cuda, kind):
    code = table("4000x2000")
    words = 600  # several pipelined chunks
    llr = make_llr("awgn", 4 * words * code.n, 5, sigma=llr_gen.sigma_for(1.5, 0.5))
    hard = np.zeros(4 * words * code.n, dtype=np.uint8)
    dec = fl.Decoder(code, kind, nb_frames=words)
    dec.decode_host(llr, hard, 20)
    ref = oracle_decode(code, kind, llr, 20)
    assert np.array_equal(hard.reshape(4 * words, code.n), ref["hard"])


def test_plugin_classes(cuda):
    fl.select_code("4000x2000")
    code = fl.selected_code()
    nb = 128
    llr = make_llr("awgn", 4 * nb * code.n, 9, sigma=llr_gen.sigma_for(2.0, 0.5))
    for flag, cls in fl.PLUGINS.items():
        dec = cls(nb, code.n, code.m, code.e)
        dec.initialize()
        out = np.zeros(4 * nb * code.n, dtype=np.uint8)
        dec.decode(llr, out, 20)
        ref = oracle_decode(code, cls.KIND, llr, 20)
        assert np.array_equal(out.reshape(-1, code.n), ref["hard"]), flag
        dec.close()
    with pytest.raises(ValueError):
        fl.CGPU_Decoder_OMS_SIMD(nb, 1000, 500, 3000)


@pytest.mark.parametrize("pack", ["SIMD4", "F16X2", "I8"])
def test_packed_output(cuda, pack):
    import torch
    code = table("1944x972")
    words = 40
    llr = make_llr("awgn", 4 * words * code.n, 11, sigma=llr_gen.sigma_for(2.0, 0.5))
    dec = fl.Decoder(code, "OMS", nb_frames=words, pack=pack)
    d_llr = torch.from_numpy(llr).cuda()
    nb = (code.n + 7) // 8
    d_bits = torch.zeros(4 * words * nb, dtype=torch.uint8, device="cuda")
    d_bytes = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, d_bits, words, 20, out_format=_lib.OUT_PACKED, stream=torch.cuda.current_stream())
    dec.decode_device(d_llr, d_bytes, words, 20, out_format=_lib.OUT_BYTES, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    bytes_ = d_bytes.cpu().numpy().reshape(4 * words, code.n)
    expect = np.packbits(bytes_, axis=1, bitorder="little")
    assert np.array_equal(d_bits.cpu().numpy().reshape(4 * words, nb), expect)


def test_error_statuses(cuda):
    code = table("576x288")
    dec = fl.Decoder(code, "OMS", nb_frames=8)
    llr = np.zeros(4 * 8 * code.n, dtype=np.int8)
    hard = np.zeros_like(llr, dtype=np.uint8)
    with pytest.raises(fl.LdpcError) as e:
        dec.decode_host(llr, hard, 0)
    assert e.value.code == -1
    import torch
    d = torch.zeros(4 * 9 * code.n, dtype=torch.int8, device="cuda")
    with pytest.raises(fl.LdpcError) as e:
        dec.decode_device(d, d, 9, 10)
    assert e.value.code == -5
    with pytest.raises(fl.LdpcError):
        fl.Decoder(code, "OMS", nb_frames=0)


def test_oversized_code_rejected(cuda):
    """The 4-frame state of N = 64800 does not fit in shared memory: an explicit
    4-frame packing is rejected, and AUTO takes the one-frame-per-CTA path."""
    for pack in ("SIMD4", "F16X2", "I8"):
        with pytest.raises(fl.LdpcError) as e:
            fl.Decoder(table("64800x32400"), "OMS", nb_frames=4, pack=pack)
        assert e.value.code == -3
    dec = fl.Decoder(table("64800x32400"), "OMS", nb_frames=4)
    assert dec.info()["path"] == 3
    dec.close()


@pytest.mark.parametrize("op", range(10))
def test_simd_ops_exhaustive(cuda, op):
    """All 65536 byte pairs in every byte lane, device intrinsic vs oracle semantics."""
    import torch
    a = np.repeat(np.arange(256, dtype=np.uint32), 256)
    b = np.tile(np.arange(256, dtype=np.uint32), 256)
    table_ = np.array([oracle.byte_op(op, x, y) for x in range(256) for y in range(256)], dtype=np.uint32)
    rng = np.random.default_rng(op)
    for lane in range(4):
        other = rng.integers(0, 2 ** 32, size=a.size, dtype=np.uint64).astype(np.uint32)
        mask = np.uint32(0xFF << (8 * lane))
        A = (other & ~mask) | (a << np.uint32(8 * lane))
        B = (other[::-1] & ~mask) | (b << np.uint32(8 * lane))
        dA, dB = torch.from_numpy(A.view(np.int32)).cuda(), torch.from_numpy(B.view(np.int32)).cuda()
        dO = torch.zeros_like(dA)
        _lib.check(_lib.lib().ldpc_simd_selftest(op, dA.data_ptr(), dB.data_ptr(), dO.data_ptr(), a.size, None))
        torch.cuda.synchronize()
        got = (dO.cpu().numpy().view(np.uint32) >> np.uint32(8 * lane)) & np.uint32(0xFF)
        assert np.array_equal(got, table_), "op %d lane %d" % (op, lane)


def test_decoders_sharing_a_kernel(cuda):
    """Two decoders whose codes use the same kernel with different shared-memory
    sizes: creating the smaller one after the larger must not break the larger."""
    import torch
    big, small = table("1944x972"), table("576x288")   # both: the SIMD4 OMS kernel for degree <= 8
    d_big = fl.Decoder(big, "OMS", nb_frames=4, pack="SIMD4")
    d_small = fl.Decoder(small, "OMS", nb_frames=4, pack="SIMD4")
    for code, dec in ((big, d_big), (small, d_small)):
        llr = make_llr("awgn", 16 * code.n, 3, sigma=llr_gen.sigma_for(2.0, 0.5))
        out = torch.zeros(16 * code.n, dtype=torch.uint8, device="cuda")
        dec.decode_device(torch.from_numpy(llr).cuda(), out, 4, 8)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().reshape(16, code.n), oracle_decode(code, "OMS", llr, 8)["hard"])
        dec.close()
