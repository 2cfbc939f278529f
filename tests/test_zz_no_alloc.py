"""The allocation-free decode entry point (ldpc_decode_noalloc), through the C ABI.

It serves callers that may not allocate device memory while running (real-time
receive chains, hosts whose memory pool owns the GPU).  Its results must equal
those of the regular entry point bit for bit, on two calls in a row with
different codes and inputs (the static table array is rewritten by each call).
This file is collected last on purpose; it passes alone and after the others.
"""
import ctypes

import numpy as np
import pytest

import llr_gen
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, _lib, load_table
from fast_ldpc_decoder_for_gpu_fixed_b200.decoder import NativeCode

pytestmark = pytest.mark.gpu


def _regular(code, kind, pack, d_llr, words, iters):
    import torch
    dec = Decoder(code, kind, nb_frames=words, pack=pack)
    out = torch.zeros(4 * words * code.n, dtype=torch.uint8, device="cuda")
    dec.decode_device(d_llr, out, words, iters, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    dec.close()
    return out.cpu().numpy()


def _noalloc(native, kind, pack, d_llr, words, iters):
    import torch
    out = torch.zeros(4 * words * native.code.n, dtype=torch.uint8, device="cuda")
    rc = _lib.lib().ldpc_decode_noalloc(native.handle, _lib.KINDS[kind], _lib.PACKS[pack], d_llr.data_ptr(),
                                         out.data_ptr(), words, iters, torch.cuda.current_stream().cuda_stream)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_regular_entry_point_twice(cuda):
    import torch
    # consecutive calls with different codes, kinds and packings; the regular decoder
    # takes other kernels for some of them (F16X2 OMS / xMS: 2 frames per CTA), which
    # must decide identically
    cases = [("4000x2000", "OMS", "SIMD4", 37, 20), ("576x288", "2NMS", "F16X2", 21, 15),
             ("1944x972", "OMS", "F16X2", 9, 12), ("4000x2000", "XMS", "F16X2", 5, 10),
             ("576x288", "MS", "I8", 13, 8), ("2304x1152", "NMS", "I8", 6, 7)]
    for name, kind, pack, words, iters in cases:
        code = load_table(name)
        native = NativeCode(code)
        llr = llr_gen.llr("awgn", 4 * words * code.n, 17 + words, sigma=llr_gen.sigma_for(2.0, 0.5))
        d_llr = torch.from_numpy(llr).cuda()
        got = _noalloc(native, kind, pack, d_llr, words, iters)
        want = _regular(code, kind, pack, d_llr, words, iters)
        assert np.array_equal(got, want), (name, kind, pack)
        native.close()


def test_noalloc_rejects_oversized_tables(cuda):
    """The 64800-column table needs more than the 256 KiB static array: a clear error, no launch."""
    import torch
    native = NativeCode(load_table("64800x32400"))
    d = torch.zeros(4 * 64800, dtype=torch.int8, device="cuda")
    rc = _lib.lib().ldpc_decode_noalloc(native.handle, 1, 0, d.data_ptr(), d.data_ptr(), 1, 5, None)
    assert rc == -3
    assert "static array" in _lib.last_error()
