"""Shared helpers of the GPU tests: run the CUDA decoder through the C ABI and
compare it with the CPU oracle (tests only)."""
import hashlib

import numpy as np

import llr_gen
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, load_table

_oracle_cache = {}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make_llr(kind, count, seed, sigma=None, value=0):
    return llr_gen.llr(kind, count, seed, sigma=sigma, value=value)


def gpu_decode(code, kind, llr, iters, words, pack="AUTO", state=True, early_stop=False, constants=None,
               slack=None):
    """Decodes 4*words frames on cuda:0; returns hard [frames, n], app/msg (reference
    device layouts, bytes) and the per-word iteration counts."""
    import pytest
    import torch
    from fast_ldpc_decoder_for_gpu_fixed_b200 import LdpcError
    try:
        dec = Decoder(code, kind, nb_frames=words, pack=pack, early_stop=early_stop)
        if constants is not None:
            dec.set_learned(*constants)
        if slack is not None:
            dec.set_early_stop(True, slack)
    except LdpcError as e:
        if e.code == -3:  # the code's state does not fit one CTA with this packing
            pytest.skip(str(e))
        raise
    n = code.n
    d_llr = torch.from_numpy(np.ascontiguousarray(llr)).cuda()
    d_hard = torch.zeros(4 * words * n, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(words, dtype=torch.int32, device="cuda")
    d_app = torch.zeros(4 * words * n, dtype=torch.int8, device="cuda") if state else None
    d_msg = torch.zeros(4 * words * code.e, dtype=torch.int8, device="cuda") if state else None
    st = torch.cuda.current_stream()
    dec.decode_device_state(d_llr, d_hard, words, iters, d_it, d_app, d_msg, stream=st)
    torch.cuda.synchronize()
    out = {"hard": d_hard.cpu().numpy().reshape(4 * words, n), "iters": d_it.cpu().numpy(),
           "info": dec.info()}
    if state:
        out["app"] = d_app.cpu().numpy()
        out["msg"] = d_msg.cpu().numpy()
    dec.close()
    return out


def oracle_decode(code, kind, llr, iters):
    key = (code.name, code.n, code.e, kind, sha(llr), iters)
    if key not in _oracle_cache:
        _oracle_cache[key] = oracle.decode(code, kind, llr, iters, want_state=True)
    return _oracle_cache[key]


def assert_same(gpu, ref, what=("hard", "app", "msg", "iters")):
    for k in what:
        a, b = np.asarray(gpu[k]).reshape(-1), np.asarray(ref[k]).reshape(-1)
        if not np.array_equal(a, b):
            bad = np.flatnonzero(a != b)
            raise AssertionError("%s differs at %d of %d positions (first %s: gpu %s vs oracle %s)"
                                 % (k, bad.size, a.size, bad[:5], a[bad[:5]], b[bad[:5]]))


def table(name):
    return load_table(name)
