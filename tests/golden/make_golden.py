"""Makes the golden fixtures that pin the CPU oracle to the reference itself.

Runs on a machine with a B200.  It loads the reference's own decoder kernels,
built unmodified from the reference sources by ``oracle/build_ref.sh`` into
``oracle/_ref/libref_<code>.so``, feeds them deterministic inputs from
``llr_gen.py``, and records SHA-256 digests of what they produce: the hard
decisions the plugin's decode() returns, and the final APP and message arrays
in the reference's device layouts.  It also runs the CPU oracle on the same
inputs and records whether it agreed (informational; the tests re-check).

    python tests/golden/make_golden.py [--out tests/golden/reference_decoder.json]
    python tests/golden/make_golden.py --time ref_kernel_times.json
"""
import argparse
import ctypes
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import llr_gen  # noqa: E402
from oracle import oracle  # noqa: E402
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import load_table  # noqa: E402

REF_DIR = os.path.join(ROOT, "oracle", "_ref")
# The reference's default table (src/matrix/code.h: CODE 4000, one degree group of 6),
# the three tables with two degree groups (576x288: 7 and 6, 1944x972: 8 and 7,
# 2304x1152: 7 and 6), whose second group runs the separate DEG_2 row loops, the OMS
# first-iteration no-clip (decoder_oms/cuda/CUDA_OMS_SIMD.cu:115-116) and xMS's
# LDPC_Sched_Stage_1_MS_SIMD_Two_CN_Degs, and 816x408 (one group of degree 10).
# Each library is built by oracle/build_ref.sh for its own table.
CODES = {4000: "4000x2000", 576: "576x288", 1944: "1944x972", 2304: "2304x1152", 816: "816x408"}
KINDS = ["MS", "OMS", "NMS", "2NMS", "XMS"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


class RefLib:
    def __init__(self, code_id):
        self.lib = ctypes.CDLL(os.path.join(REF_DIR, "libref_%d.so" % code_id))
        self.lib.ref_decode.restype = ctypes.c_double
        P = ctypes.c_void_p
        self.lib.ref_decode.argtypes = [ctypes.c_int, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]
        info = (ctypes.c_int * 8)()
        self.lib.ref_info(info)
        self.n, self.k, self.m, self.nb_degres, self.deg1 = info[0], info[1], info[2], info[3], info[4]

    def decode(self, kind, llr, W, iters, block=32, want_state=True):
        hard = np.zeros(4 * W * self.n, dtype=np.uint8)
        app = np.zeros(self.n * W * 4, dtype=np.int8) if want_state else None
        msg = np.zeros(self.m * W * 4, dtype=np.int8) if want_state else None
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None else None
        us = self.lib.ref_decode(KINDS.index(kind), p(llr), W, iters, block, p(hard), p(app), p(msg))
        if us < 0:
            raise RuntimeError("ref_decode failed")
        return hard, app, msg, us


def xms_supported(ref):
    return ref.nb_degres != 1 or ref.deg1 in (6, 7)


def cases():
    """The default table's 24 cases (unchanged seeds), then those of the other tables."""
    out = []
    seed = 1000
    for cid, name in CODES.items():
        if cid != 4000:
            continue
        code = load_table(name)
        rate = code.n_info / code.n
        inputs = [
            {"type": "awgn", "ebn0": 1.0, "sigma": llr_gen.sigma_for(1.0, rate)},
            {"type": "awgn", "ebn0": 2.5, "sigma": llr_gen.sigma_for(2.5, rate)},
            {"type": "uniform"},
            {"type": "extreme"},
        ]
        for kind in KINDS:
            for inp in inputs:
                seed += 1
                # The reference 2NMS kernel (EARLY_TERM 1) leaves its iteration loop per
                # thread while the other threads of the CTA keep executing the row loops'
                # __syncthreads(); words of one CTA that stop at different iterations
                # leave those barriers divergent and the kernel hangs (seen on a B200 with
                # the 4000x2000 code at Eb/N0 2.5 dB).  Its cases therefore repeat one
                # word across the batch, so that every thread stops at the same iteration.
                tile = {"tile": True} if kind == "2NMS" else {}
                out.append({"code": name, "lib": cid, "kind": kind, "iters": 20, "W": 32,
                            "input": dict(inp, seed=seed, **tile)})
        for iters in (1, 2, 3):
            seed += 1
            out.append({"code": name, "lib": cid, "kind": "OMS", "iters": iters, "W": 32,
                        "input": {"type": "uniform", "seed": seed}})
        seed += 1
        out.append({"code": name, "lib": cid, "kind": "2NMS", "iters": 30, "W": 32,
                    "input": {"type": "awgn", "ebn0": 3.5, "sigma": llr_gen.sigma_for(3.5, rate),
                              "seed": seed, "tile": True}})
    seed = 5000
    for cid, name in CODES.items():
        if cid == 4000:
            continue
        code = load_table(name)
        rate = code.n_info / code.n
        lo = {"type": "awgn", "ebn0": 1.0, "sigma": llr_gen.sigma_for(1.0, rate)}
        hi = {"type": "awgn", "ebn0": 2.5, "sigma": llr_gen.sigma_for(2.5, rate)}
        plan = []
        for kind in ("MS", "OMS", "NMS", "XMS"):
            for inp in (lo, hi, {"type": "uniform"}):
                plan.append((kind, 20, inp, False))
        for kind in ("MS", "OMS"):
            plan.append((kind, 20, {"type": "extreme"}, False))
        # OMS after 1, 2 and 3 iterations: the first iteration's second-group rows keep
        # magnitudes above 31, which uniform and extreme inputs reach
        for iters in (1, 2, 3):
            plan.append(("OMS", iters, {"type": "uniform"}, False))
        plan.append(("OMS", 1, {"type": "extreme"}, False))
        plan.append(("XMS", 2, {"type": "uniform"}, False))
        for inp in (lo, hi):
            plan.append(("2NMS", 20, inp, True))
        for kind, iters, inp, tile in plan:
            seed += 1
            extra = {"tile": True} if tile else {}
            out.append({"code": name, "lib": cid, "kind": kind, "iters": iters, "W": 32,
                        "input": dict(inp, seed=seed, **extra)})
    return out


def make_input(case, n):
    """Deterministic LLRs of a case.  With "tile", one 4-frame word is generated
    and repeated in every word of the batch (used for every 2NMS case, see cases())."""
    return llr_gen.case_llr(case, n)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "reference_decoder.json"))
    ap.add_argument("--time", default=None, help="only time the reference kernels (config-1 size)")
    ap.add_argument("--limit", type=int, default=0, help="stop after this many cases (0 = all)")
    ap.add_argument("--codes", default="", help="comma-separated subset of codes")
    args = ap.parse_args()
    wanted = [name for name in CODES.values() if not args.codes or name in args.codes.split(",")]
    refs = {cid: RefLib(cid) for cid, name in CODES.items() if name in wanted}
    if args.time:
        return time_kernels(refs, args.time)
    results = []
    mism = 0
    t_start = time.time()
    todo = [c for c in cases() if c["code"] in wanted]
    if args.limit:
        todo = todo[:args.limit]
    for case in todo:
        ref = refs[case["lib"]]
        if case["kind"] == "XMS" and not xms_supported(ref):
            continue
        code = load_table(case["code"])
        llr = make_input(case, code.n)
        t0 = time.time()
        hard, app, msg, us = ref.decode(case["kind"], llr, case["W"], case["iters"])
        t1 = time.time()
        o = oracle.decode(code, case["kind"], llr, case["iters"], want_state=True)
        t2 = time.time()
        ok = (sha(o["hard"]) == sha(hard) and sha(o["app"]) == sha(app) and sha(o["msg"]) == sha(msg))
        mism += (not ok)
        results.append(dict(case, sha256={"hard": sha(hard), "app": sha(app), "msg": sha(msg)},
                            oracle_agreed=bool(ok)))
        print(case["code"], case["kind"], case["iters"], case["input"]["type"], "oracle", "OK" if ok else "MISMATCH",
              "ref %.2fs (kernel %.0f us) oracle %.2fs total %.0fs" % (t1 - t0, us, t2 - t1, time.time() - t_start),
              flush=True)
    doc = {"generator": "tests/golden/make_golden.py", "source": "reference kernels built by oracle/build_ref.sh",
           "cases": results}
    with open(args.out, "w") as f:
        json.dump(doc, f, indent=1)
    print("cases", len(results), "oracle mismatches", mism)
    return 0 if mism == 0 else 1


def time_kernels(refs, path):
    """Times the reference kernel alone on the 4000x2000 code: 4096 frames (-n 1024), 20 iterations."""
    code = load_table("4000x2000")
    ref = refs[4000]
    rate = code.n_info / code.n
    rows = []
    for W in (1024, 8192):
        llr = llr_gen.llr("awgn", 4 * W * code.n, 7, sigma=llr_gen.sigma_for(2.0, rate))
        for kind in KINDS:
            if kind == "2NMS":
                continue  # its early termination hangs on divergent barriers (see cases())
            ts = []
            for _ in range(4):
                _, _, _, us = ref.decode(kind, llr, W, 20, block=128, want_state=False)
                ts.append(us)
            us = float(np.median(ts[1:]))
            gbps = 4 * W * code.n_info / (us * 1e-6) / 1e9
            rows.append({"kind": kind, "W": W, "frames": 4 * W, "iters": 20, "kernel_us": us,
                         "info_gbps": gbps})
            print(rows[-1], flush=True)
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "w") as f:
        json.dump(rows, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
