"""ctypes front-end of the CPU oracle (oracle/ldpc_oracle.c, oracle/ldpc_oracle_batch.c).

TEST INFRASTRUCTURE ONLY.  tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of bench.py use it as the checker; the product path never
imports it.  ``build()`` compiles the C sources with gcc into
oracle/_build/liboracle.so.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
SOURCES = [os.path.join(HERE, "ldpc_oracle.c"), os.path.join(HERE, "ldpc_oracle_batch.c")]

KINDS = {"MS": 0, "OMS": 1, "NMS": 2, "2NMS": 3, "XMS": 4, "LEARNED": 5}

_lib = None


def build(force=False):
    os.makedirs(BUILD, exist_ok=True)
    stale = force or not os.path.exists(LIB) or any(
        os.path.getmtime(s) > os.path.getmtime(LIB) for s in SOURCES)
    if stale:
        cmd = ["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", LIB] + SOURCES + ["-lm"]
        subprocess.check_call(cmd)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        i = ctypes.c_int
        L.oracle_decode.argtypes = [i, i, P, P, P, i, i, i, i, P, P, P, P, P, i]
        L.oracle_decode.restype = i
        L.oracle_decode_ex.argtypes = [i, i, P, P, P, i, i, i, i, P, P, P, P, P, i, i, i]
        L.oracle_decode_ex.restype = i
        L.oracle_decode_batch.argtypes = [i, i, P, P, P, i, i, i, i, P, P, i]
        L.oracle_decode_batch.restype = i
        L.oracle_batch_supported.restype = i
        L.oracle_batch_isa.restype = i
        L.oracle_batch_force_avx2.argtypes = [i]
        L.oracle_byte_op.argtypes = [i, i, i]
        L.oracle_byte_op.restype = i
        L.oracle_interleave.argtypes = [i, i, P, P]
        L.oracle_deinterleave_hd.argtypes = [i, i, P, P]
        L.oracle_count_errors.argtypes = [i, i, i, P, P, P, P]
        L.oracle_quantize.argtypes = [ctypes.c_float, ctypes.c_float]
        L.oracle_quantize.restype = i
        L.oracle_sigma.argtypes = [ctypes.c_double, ctypes.c_double, i]
        L.oracle_sigma.restype = ctypes.c_double
        L.oracle_set_learned.argtypes = [i, P, P]
        L.oracle_set_learned.restype = i
        L.oracle_set_schedule.argtypes = [i]
        L.oracle_set_schedule.restype = i
        L.oracle_philox.argtypes = [P, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_awgn.argtypes = [P, P, ctypes.c_size_t, i, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64, P,
                                  ctypes.c_size_t]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def set_schedule(flooding):
    """Layered (False, the reference's) or flooding (True) schedule for decode()."""
    lib().oracle_set_schedule(int(bool(flooding)))


def decode(code, kind, llr, iters, interleaved=None, want_state=False, nthreads=None, early_stop=False,
           early_slack=128, per_frame=False, pairs=False, flooding=False):
    """Decodes ``llr`` (int8, nframes*n bytes, frame-major unless interleaved).

    Returns dict with ``hard`` [nframes, n] uint8, ``iters`` [nframes/4] and,
    if ``want_state``, ``app`` / ``msg`` in the reference's word-interleaved
    device layouts (n*nframes and e*nframes bytes).  ``early_stop``: the
    syndrome early stop of LDPC_FLAG_EARLY_STOP (per 4-frame word) with
    ``early_slack`` (ldpc_decoder_set_early_stop); ``per_frame``: every frame
    stops on its own and ``iters`` has one entry per frame (LDPC_PACK_FRAME,
    LDPC_FLAG_EARLY_STOP_FRAMES);
    ``pairs``: frames 4g, 4g+1 and 4g+2, 4g+3 stop as pairs and ``iters`` has the
    larger count of each word (the 2-frame QC kernel, decoder path 4);
    ``flooding``: the flooding schedule of LDPC_FLAG_FLOODING instead of the layered one.
    """
    k = KINDS[kind.upper()] if isinstance(kind, str) else int(kind)
    if interleaved is None:
        interleaved = (k == KINDS["XMS"])
    llr = np.ascontiguousarray(llr, dtype=np.int8).reshape(-1)
    nframes = llr.size // code.n
    hard = np.zeros((nframes, code.n), dtype=np.uint8)
    it = np.zeros(nframes if per_frame else nframes // 4, dtype=np.int32)
    app = np.zeros(code.n * nframes, dtype=np.int8) if want_state else None
    msg = np.zeros(code.e * nframes, dtype=np.int8) if want_state else None
    nt = nthreads or os.cpu_count() or 1
    set_schedule(flooding)
    try:
        rc = lib().oracle_decode_ex(code.n, code.m, _p(code.row_ptr), _p(code.cols), _p(code.row_class),
                                    k, int(iters), nframes, int(bool(interleaved)), _p(llr), _p(hard),
                                    _p(app), _p(msg), _p(it), nt, 1 + int(early_slack) if early_stop else 0,
                                    1 if per_frame else (2 if pairs else 4))
    finally:
        set_schedule(False)
    if rc != 0:
        raise ValueError("oracle_decode rejected the arguments")
    out = {"hard": hard, "iters": it}
    if want_state:
        out["app"] = app
        out["msg"] = msg
    return out


def batch_supported():
    return bool(lib().oracle_batch_supported())


def batch_isa():
    """The vector ISA decode_batch uses on this CPU: "avx512bw", "avx2" or None."""
    return {2: "avx512bw", 1: "avx2"}.get(lib().oracle_batch_isa())


def force_avx2(on):
    """Makes decode_batch use its AVX2 path even where AVX-512BW exists (tests)."""
    lib().oracle_batch_force_avx2(int(bool(on)))


def cpu_model():
    """The host CPU's model name (from /proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def decode_batch(code, kind, llr, iters, interleaved=None, nthreads=None):
    """Lock-step vector decoder (same results as decode()): 64-frame groups with
    AVX-512BW, 32-frame groups with AVX2; frames must be a multiple of 32."""
    k = KINDS[kind.upper()] if isinstance(kind, str) else int(kind)
    if interleaved is None:
        interleaved = (k == KINDS["XMS"])
    llr = np.ascontiguousarray(llr, dtype=np.int8).reshape(-1)
    nframes = llr.size // code.n
    hard = np.zeros((nframes, code.n), dtype=np.uint8)
    nt = nthreads or os.cpu_count() or 1
    rc = lib().oracle_decode_batch(code.n, code.m, _p(code.row_ptr), _p(code.cols),
                                   _p(code.row_class), k, int(iters), nframes,
                                   int(bool(interleaved)), _p(llr), _p(hard), nt)
    if rc != 0:
        raise ValueError("oracle_decode_batch: unsupported kind/size or no AVX2")
    return hard


def byte_op(op, a, b):
    return lib().oracle_byte_op(op, a, b)


def interleave(n, W, frames):
    frames = np.ascontiguousarray(frames, dtype=np.int8).reshape(-1)
    out = np.zeros(n * W * 4, dtype=np.int8)
    lib().oracle_interleave(n, W, _p(frames), _p(out))
    return out


def deinterleave_hd(n, W, words):
    words = np.ascontiguousarray(words, dtype=np.int8).reshape(-1)
    out = np.zeros(n * W * 4, dtype=np.uint8)
    lib().oracle_deinterleave_hd(n, W, _p(words), _p(out))
    return out.reshape(4 * W, n)


def count_errors(n, n_vars, hard):
    hard = np.ascontiguousarray(hard, dtype=np.uint8).reshape(-1)
    nframes = hard.size // n
    be = np.zeros(1, dtype=np.int64)
    fe = np.zeros(1, dtype=np.int64)
    per = np.zeros(nframes, dtype=np.int32)
    lib().oracle_count_errors(n, n_vars, nframes, _p(hard), _p(be), _p(fe), _p(per))
    return int(be[0]), int(fe[0]), per


def sigma(ebn0, rate, es_n0=False):
    return lib().oracle_sigma(float(ebn0), float(rate), int(es_n0))


def philox(count, seed, offset=0):
    out = np.zeros(count, dtype=np.uint32)
    lib().oracle_philox(_p(out), count, seed, offset)
    return out


def awgn(frames, n, sigma, seed, offset=0, codewords=None):
    """Returns (int8 LLRs [frames, n], pre-quantisation 8y in double)."""
    out = np.zeros(frames * n, dtype=np.int8)
    y8 = np.zeros(frames * n, dtype=np.float64)
    cw = None if codewords is None else np.ascontiguousarray(codewords, dtype=np.uint8)
    lib().oracle_awgn(_p(out), _p(y8), frames, n, float(sigma), seed, offset, _p(cw),
                      0 if cw is None else cw.shape[0])
    return out.reshape(frames, n), y8.reshape(frames, n)


def set_learned(offsets, scales):
    """Per-iteration [n_iters][2] int8 offsets and uint8 Q1.7 scales of the LEARNED kind."""
    off = np.ascontiguousarray(offsets, dtype=np.int8).reshape(-1, 2)
    sc = np.ascontiguousarray(scales, dtype=np.uint8).reshape(-1, 2)
    if lib().oracle_set_learned(off.shape[0], _p(off), _p(sc)) != 0:
        raise ValueError("bad learned table")
