"""The oracle's flooding schedule (LDPC_FLAG_FLOODING, this library's own mode) against an
independent numpy statement of it: every row reads the previous iteration's APP, the
messages follow the reference's check update, and APP = sat8(LLR + sum of the new messages)."""
import numpy as np
import pytest

import llr_gen
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import load_table


def _numpy_flood_oms(code, llr, iters):
    F = llr.size // code.n
    x = llr.reshape(F, code.n).astype(np.int32)
    llr0 = x.copy()
    msg = np.zeros((F, code.e), np.int32)
    for it in range(iters):
        acc = llr0.copy()
        for r in range(code.m):
            b, e = code.row_ptr[r], code.row_ptr[r + 1]
            cols = code.cols[b:e]
            t = x[:, cols] if it == 0 else np.clip(x[:, cols] - msg[:, b:e], -128, 127)
            a = np.abs(t)                                  # |-128| = 128 as an unsigned byte
            srt = np.sort(a, axis=1)
            mn1, mn2 = np.minimum(srt[:, 0], 127), np.minimum(srt[:, 1], 127)
            cls = code.row_class[r]
            c1, c2 = np.maximum(mn2 - 1, 0), np.maximum(mn1 - 1, 0)
            if not (it == 0 and cls == 1):
                c1, c2 = np.minimum(c1, 31), np.minimum(c2, 31)
            sgn = np.bitwise_xor.reduce(t > 0, axis=1)
            re = np.where(a == mn1[:, None], c1[:, None], c2[:, None])
            out = np.where(sgn[:, None] ^ (t > 0), re, -re)
            msg[:, b:e] = out
            np.add.at(acc, (slice(None), cols), out)
        x = np.clip(acc, -128, 127)
    return (x > 0).astype(np.uint8), x.astype(np.int8)


@pytest.mark.parametrize("name,iters", [("576x288", 1), ("576x288", 6), ("816x408", 4)])
def test_oracle_flooding_matches_numpy(name, iters):
    code = load_table(name)
    llr = llr_gen.llr("awgn", 8 * code.n, 41, sigma=llr_gen.sigma_for(2.0, 0.5))
    r = oracle.decode(code, "OMS", llr, iters, want_state=True, flooding=True)
    hard, app = _numpy_flood_oms(code, llr, iters)
    assert np.array_equal(r["hard"], hard)
    # the oracle's APP is in the word-interleaved layout word[v*W+g], byte k = frame 4g+k
    W = 2
    app_frames = r["app"].reshape(code.n, W, 4).transpose(1, 2, 0).reshape(4 * W, code.n)
    assert np.array_equal(app_frames, app)


def test_flooding_differs_from_layered():
    code = load_table("576x288")
    llr = llr_gen.llr("awgn", 8 * code.n, 42, sigma=llr_gen.sigma_for(1.5, 0.5))
    a = oracle.decode(code, "OMS", llr, 3, want_state=True)["app"]
    b = oracle.decode(code, "OMS", llr, 3, want_state=True, flooding=True)["app"]
    assert not np.array_equal(a, b)
    # and the layered default is restored after a flooding call
    assert np.array_equal(oracle.decode(code, "OMS", llr, 3, want_state=True)["app"], a)
