"""Deterministic int8 LLR generators for parity tests and golden fixtures.

Bit-identical on every machine: a counter-based SplitMix64 stream, and only
IEEE basic operations (no libm), so the golden fixtures made on the GPU box
and the inputs re-made by the tests here agree exactly.

kinds:
  awgn     BPSK all-zero codeword over AWGN, quantised like the reference
           channel (awgn_channel/CChanel_AWGN_SIMD.cu:21-24):
           q = trunc(clamp(8*(-1 + sigma*n), -31, 31)); n is a sum of 12
           uniforms minus 6 (an exact, libm-free Gaussian approximation).
  uniform  every int8 value equally likely (exercises saturation and |-128|).
  extreme  values drawn from {-128,-127,-1,0,1,126,127}.
  const    every byte = `value`.
"""
import numpy as np

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed, count, stream=0):
    idx = np.arange(count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)
        z = z + (idx + np.uint64(1)) * _G
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def llr(kind, count, seed, sigma=None, value=0):
    if kind == "awgn":
        u = splitmix64(seed, 6 * count).reshape(count, 6)
        lo = (u & np.uint64(0xFFFFFFFF)).astype(np.float64)
        hi = (u >> np.uint64(32)).astype(np.float64)
        s = lo.sum(axis=1) + hi.sum(axis=1)
        n = s * (2.0 ** -32) - 6.0
        v = -1.0 + float(sigma) * n
        q = np.trunc(np.clip(8.0 * v, -31.0, 31.0))
        return q.astype(np.int8)
    if kind == "uniform":
        u = splitmix64(seed, count)
        return (u & np.uint64(0xFF)).astype(np.uint8).view(np.int8)
    if kind == "extreme":
        vals = np.array([-128, -127, -1, 0, 1, 126, 127], dtype=np.int8)
        u = splitmix64(seed, count)
        return vals[(u % np.uint64(len(vals))).astype(np.int64)]
    if kind == "const":
        return np.full(count, value, dtype=np.int8)
    raise ValueError(kind)


def sigma_for(ebn0_db, rate):
    """Noise deviation of the reference channel (CChanel_AWGN_SIMD.cu:63-73)."""
    interm = -0.1 * (ebn0_db + 10.0 * np.log10(rate))
    return float(np.sqrt(10.0 ** interm / 2.0))


def case_llr(case, n):
    """LLRs of a golden-fixture case (see make_golden.make_input)."""
    inp = case["input"]
    words = 1 if inp.get("tile") else case["W"]
    x = llr(inp["type"], 4 * words * n, inp["seed"], sigma=inp.get("sigma"), value=inp.get("value", 0))
    return np.tile(x, case["W"]) if inp.get("tile") else x
