#!/usr/bin/env python
"""Decoded info Gbit/s of the fixed-point LDPC decoder on B200 GPUs.

Default workload (the metric: learned-offset decoder vs plain OMS at equal FER):
  seeded regular (3,6) QC-LDPC, 8x16 base of Z=256 circulants (N=4096, K=2048,
  4-cycle free), random info bits through the systematic encoder, BPSK over AWGN
  at Eb/N0 = 2.25 dB, int8 LLRs quantised like the reference channel
  (q = trunc(clamp(8y, -31, 31)), awgn_channel/CChanel_AWGN_SIMD.cu:21-24),
  65536 frames per GPU, at most 10 layered iterations.
  value      : the deployed learned-offset decoder (LDPC_LEARNED with the per-iteration
               offsets in fast_ldpc_decoder_for_gpu_fixed_b200/trained/qc3x6_z256_T10_offsets.json,
               trained with every scale held at 1.0; --constants for another set, such as the
               offsets-and-scales set qc3x6_z256_T10.json,
               syndrome early stop per frame pair, each pair stopping at its first codeword
               iteration (LDPC_EARLY_SLACK_ANY); --early-unit word|frame and --slack for the
               other rules), kernel only, LLRs resident in HBM
  plain_oms  : the plain 8-bit OMS kernel (offset 1, 10 fixed iterations) on the same
               batch and GPU; vs_plain_oms = value / plain_oms.value
  oms_early_stop : plain OMS with the same early stop; early_stop_gain = its value /
               plain_oms, learned_gain = value / its value
  fer        : both decoders on 2^20 further frames at the same Eb/N0 (untimed)
  e2e        : the learned decoder through the reference-facing host call
               (ldpc_decode_host: pinned host LLRs in, 0/1 bytes out, copies timed);
               e2e_packed the same through ldpc_decode_host_ex with packed bits out
Other workloads: --workload oms (plain OMS, fixed iterations), --table NAME (a
reference H table, all-zero codeword), --workload ira (N=64800 IRA code, one frame
per CTA, early stop, at most 50 iterations, 2048 frames).

python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Multi-GPU: torchrun ... bench.py --gpus N (weak scaling: every rank decodes its own batch).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "qc(3,6) N=4096 K=2048 Z=256, 65536 frames, Eb/N0 %.2f dB: learned-offset int8 decoder with early stop " \
           "(max %d layered iterations) vs plain OMS offset 1, %d fixed iterations"
TRAINED = os.path.join(ROOT, "fast_ldpc_decoder_for_gpu_fixed_b200", "trained", "qc3x6_z256_T10_offsets.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=65536)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--kind", default="OMS")
    ap.add_argument("--pack", default="AUTO")
    ap.add_argument("--ebn0", type=float, default=None, help="default 2.25 dB (learned), 2.0 (oms, table), 1.4 (ira)")
    ap.add_argument("--workload", default="learned", choices=["learned", "oms", "ira", "batch"])
    ap.add_argument("--slack", default=None,
                    help="early-stop slack: an integer or 'any' (LDPC_EARLY_SLACK_ANY: every iteration a "
                         "candidate; default: the library's)")
    ap.add_argument("--per-frame", action="store_true",
                    help="early stop per frame with slot refill (LDPC_FLAG_EARLY_STOP_FRAMES); same as --early-unit frame")
    ap.add_argument("--early-unit", default="pairs", choices=["word", "pairs", "frame"],
                    help="frames that stop together under the early stop of the learned workload: the 4-frame word "
                         "(LDPC_FLAG_EARLY_STOP), each frame pair (LDPC_FLAG_EARLY_STOP_PAIRS, default) or each frame")
    ap.add_argument("--fer-frames", type=int, default=1 << 20)
    ap.add_argument("--no-sweep", dest="sweep", action="store_false",
                    help="skip the learned-vs-plain ratio over Eb/N0 1.5..2.5 dB")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-qc", action="store_true", help="use the level-scheduled kernel even for the QC code")
    ap.add_argument("--table", default=None,
                    help="decode a reference H table (e.g. 4000x2000) with the all-zero codeword instead of the QC workload")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample budget")
    ap.add_argument("--constants", default=TRAINED, help="trained LDPC_LEARNED constants (learned workload)")
    a = ap.parse_args()
    if a.table:
        a.workload = "oms"
    if a.slack is None and a.workload == "learned":
        a.slack = "any"  # the deployed decoder: every iteration a stop candidate (exact last-layer gate)
    if a.slack is not None:
        a.slack = (1 << 30) if str(a.slack).lower() == "any" else int(a.slack)
    if a.per_frame:
        a.early_unit = "frame"
    if a.ebn0 is None:
        a.ebn0 = {"learned": 2.25, "oms": 2.0, "ira": 1.4, "batch": 3.0}[a.workload]
    if a.workload == "batch":
        a.frames = 200000 if a.frames == 65536 else a.frames
        a.iters = 20 if a.iters == 10 else a.iters
    if a.workload == "ira":
        a.frames = min(a.frames, 2048) if a.frames != 65536 else 2048
        a.iters = 50 if a.iters == 10 else a.iters
    return a


class _AllZero:
    """Stands in for the encoder of a reference table: the all-zero codeword, k = N - checks
    information bits (the reference's own transmission, awgn_channel/CChanel_AWGN_SIMD.cu:21-22)."""

    def __init__(self, code):
        self.k = code.n_info

    def encode(self, info):
        return np.zeros((info.shape[0], self.n), dtype=np.uint8)


def make_workload(frames, ebn0, seed, rank=0, table=None, workload="learned"):
    """Codewords + quantised channel LLRs (int8, frame-major) for `frames` frames."""
    from fast_ldpc_decoder_for_gpu_fixed_b200.codes import Encoder, IRAEncoder, ira, load_table, qc_regular
    if table:
        code = load_table(table)
        enc = _AllZero(code)
        enc.n = code.n
    elif workload == "ira":
        code = ira()
        enc = IRAEncoder(code)
    else:
        code = qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
        enc = Encoder(code)
    rng = np.random.default_rng(seed + 7919 * rank)
    distinct = min(frames, 1024)
    cws = enc.encode(rng.integers(0, 2, size=(distinct, enc.k)))
    idx = np.arange(frames) % distinct
    rate = enc.k / code.n
    sigma = np.sqrt(10.0 ** (-(ebn0 + 10 * np.log10(rate)) / 10.0) / 2.0)
    llr = np.empty((frames, code.n), dtype=np.int8)
    step = 4096
    for f0 in range(0, frames, step):
        f1 = min(frames, f0 + step)
        y = (2.0 * cws[idx[f0:f1]].astype(np.float32) - 1.0) + sigma * rng.standard_normal((f1 - f0, code.n), dtype=np.float32)
        llr[f0:f1] = np.trunc(np.clip(8.0 * y, -31.0, 31.0)).astype(np.int8)
    return code, enc, cws, idx, llr, sigma


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples taken while the timed region runs."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.t.join(timeout=2)
        sm = [float(r[0]) for r in self.rows if r and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) > 4 + i and r[4 + i].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(code, llr, iters, kind, budget_s, info_bits):
    """The reference's kernel arithmetic restated on the host CPU (AVX2, all threads) on a
    bounded sample of the same batch, repeated until about `budget_s` seconds of CPU work;
    returns (Gbit/s, cores, sample description)."""
    from oracle import oracle
    cores = os.cpu_count() or 1
    probe = min(llr.shape[0], 1024) // 32 * 32   # the AVX2 port decodes 32-frame groups
    if probe == 0:
        return 0.0, cores, "no sample (fewer than 32 frames)"
    t = time.perf_counter()
    oracle.decode_batch(code, kind, llr[:probe], iters, nthreads=cores)
    dt = time.perf_counter() - t
    frames = int(min(llr.shape[0], max(probe, probe * budget_s / max(dt, 1e-6)))) // 32 * 32
    done, t = 0, time.perf_counter()
    while True:
        oracle.decode_batch(code, kind, llr[:frames], iters, nthreads=cores)
        done += frames
        dt = time.perf_counter() - t
        if dt >= budget_s or done >= 64 * frames:
            break
    return done * info_bits / dt / 1e9, cores, "%d frames (%d passes over %d of the batch's frames), %d iterations, %.1f s" % (
        done, done // frames, frames, iters, dt)


def run_reference(args):
    """Reference arm: the reference has no CPU decoder, so its fixed-point kernel arithmetic is
    timed as the CPU port (oracle/ldpc_oracle_batch.c) on the host cores, per step a bounded sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    code, enc, cws, idx, llr, sigma = make_workload(min(args.frames, 65536), args.ebn0, args.seed, 0, args.table,
                                                    args.workload)
    kind = "OMS" if args.workload == "learned" else args.kind   # the reference's best plain decoder
    per_step = max(1.0, 60.0 / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_baseline(code, llr, args.iters, kind, min(per_step, 2.0), enc.k)
    vals, samples = [], []
    cores = os.cpu_count() or 1
    for _ in range(args.steps):
        v, cores, s = cpu_baseline(code, llr, args.iters, kind, per_step, enc.k)
        vals.append(v)
        samples.append(s)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": "decoded info Gbit/s", "value": value, "unit": "Gbit/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": llr.shape[0] * enc.k / (value * 1e9) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
            "data": "synthetic (seeded QC codewords, AWGN)",
            "config": {"workload": workload_name(args), "l2": "host CPU run", "kind": kind},
            "cpu_baseline": dict({"value": value, "unit": "Gbit/s", "cores": cores, "kind": "port",
                                  "sample": samples[-1]}, **_cpu_info()),
            "e2e": {"value": value, "unit": "Gbit/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def batch_codes():
    """The mixed batch: four seeded irregular QC codes with a 24-column base (rates
    1/2, 2/3, 3/4, 5/6; Z from {27, 54, 81})."""
    from fast_ldpc_decoder_for_gpu_fixed_b200.codes import qc_irregular
    rng = np.random.default_rng(1201)
    zs = rng.choice([27, 54, 81], size=4)
    return [qc_irregular(z=int(z), rate=r, seed=1300 + i) for i, (z, r) in
            enumerate(zip(zs, ((1, 2), (2, 3), (3, 4), (5, 6))))]


def zipf_words(total_frames, n, s=1.2, seed=1201):
    """Per-code word counts (4 frames each): Zipf(s) shares over a seeded order."""
    rng = np.random.default_rng(seed + 1)
    p = 1.0 / np.arange(1, n + 1) ** s
    p = p[rng.permutation(n)] / p.sum()
    return [max(1, int(round(total_frames * x / 4))) for x in p]


def run_batch(args):
    """Config 3: one persistent, graph-captured, autotuned launch over the mixed batch."""
    import torch
    from fast_ldpc_decoder_for_gpu_fixed_b200 import Batch, Decoder, _lib
    from fast_ldpc_decoder_for_gpu_fixed_b200.learned import random_codewords, sigma_for
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    codes = batch_codes()
    words = zipf_words(args.frames, len(codes))
    st = torch.cuda.Stream()
    llrs, outs, its, cws = [], [], [], []
    for i, (c, w) in enumerate(zip(codes, words)):
        cw = torch.from_numpy(random_codewords(c, 64, 40 + i)).cuda()
        d = torch.empty(4 * w * c.n, dtype=torch.int8, device="cuda")
        _lib.check(_lib.lib().ldpc_channel_awgn(d.data_ptr(), 4 * w, c.n, sigma_for(args.ebn0, c.n_info / c.n),
                                                args.seed, i, cw.data_ptr(), 64, None))
        llrs.append(d)
        outs.append(torch.empty(4 * w * c.n, dtype=torch.uint8, device="cuda"))
        its.append(torch.zeros(w, dtype=torch.int32, device="cuda"))
        cws.append(cw)
    torch.cuda.synchronize()
    b = Batch(codes, args.kind, early_stop=True, graph=True)
    tune_ms = b.autotune(llrs, outs, words, args.iters, d_iters=its, stream=st)
    info = b.info()
    if info["per_code"]:
        info["code_kernels"] = [b.code_info(i) for i in range(len(codes))]

    def step():
        b.decode(llrs, outs, words, args.iters, d_iters=its, stream=st)

    with torch.cuda.stream(st):
        for _ in range(args.warmup):
            step()
    st.synchronize()
    fe = fr = 0
    it_tot = 0
    edge_updates = 0.0
    for c, w, o, it, cw in zip(codes, words, outs, its, cws):
        hard = o.view(4 * w, c.n)
        ref = cw[torch.arange(4 * w, device="cuda") % 64]
        fe += int(((hard != ref).sum(dim=1) > 0).sum())
        fr += 4 * w
        it_tot += int(it.sum())
        edge_updates += float(it.sum()) * 4 * c.e
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    with torch.cuda.stream(st):
        ms = _timed(step, args.steps, st, False)
    clocks = sampler.stop()
    ms_step = ms / args.steps
    info_bits = sum(4 * w * c.n_info for c, w in zip(codes, words))
    value = info_bits / (ms_step * 1e-3) / 1e9
    # the same frames as separate per-code launches (one decoder per code, default stream order)
    decs = [Decoder(c, args.kind, nb_frames=w, early_stop=True) for c, w in zip(codes, words)]

    def sep():
        for dcd, l, o, w in zip(decs, llrs, outs, words):
            dcd.decode_device(l, o, w, args.iters, stream=st)

    with torch.cuda.stream(st):
        for _ in range(args.warmup):
            sep()
        ms_sep = _timed(sep, args.steps, st, False)
    for dcd in decs:
        dcd.close()
    int_peak = _int_peak()
    achieved = 2.0 * edge_updates / (ms_step * 1e-3) / 1e12
    line = {"metric": "decoded info Gbit/s", "value": value, "unit": "Gbit/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8", "data": "synthetic (seeded codewords, AWGN, reference quantiser)",
            "config": {"workload": "mixed batch: %s, Zipf(1.2) frame counts %s (%d frames), %s with early stop, "
                       "max %d iterations, Eb/N0 %.2f dB, one persistent graph-captured launch" % (
                           ", ".join("%s N=%d" % (c.name, c.n) for c in codes), [4 * w for w in words],
                           4 * sum(words), args.kind, args.iters, args.ebn0, ),
                       "mean_iterations": it_tot / sum(words), "fer": fe / fr, "autotuned": info,
                       "autotune_ms": tune_ms, "l2": "inputs (%d MB) re-read each step" % (
                           sum(4 * w * c.n for c, w in zip(codes, words)) // 2**20)},
            "per_code_launches": {"value": info_bits / (ms_sep / args.steps * 1e-3) / 1e9, "unit": "Gbit/s",
                                  "ms_per_step": ms_sep / args.steps},
            "roofline": {"bound": "int", "achieved": achieved, "peak": int_peak, "unit": "Tops/s (int32 word-ops)",
                         "frac": achieved / int_peak, "traffic": None, "edge_updates_per_launch": edge_updates},
            "cpu_baseline": None, "e2e": None, "gpu_launches": args.steps, "clocks": clocks}
    print(json.dumps(line), flush=True)
    b.close()
    return 0


def workload_name(args):
    if args.workload == "learned":
        return WORKLOAD % (args.ebn0, args.iters, args.iters)
    if args.table:
        return "reference table %s, all-zero codeword, %s, %d iterations, %d frames, Eb/N0 %.2f dB" % (
            args.table, args.kind, args.iters, args.frames, args.ebn0)
    if args.workload == "ira":
        return "IRA N=64800 K=32400 (groups of 360, 1/5 degree 8), %s with early stop, max %d iterations, " \
               "%d frames, Eb/N0 %.2f dB" % (args.kind, args.iters, args.frames, args.ebn0)
    return "qc(3,6) N=4096 K=2048 Z=256 %s, %d layered iterations, %d frames, Eb/N0 %.2f dB" % (
        args.kind, args.iters, args.frames, args.ebn0)


def _timed(step, steps, stream, flush):
    """Device time (ms) of `steps` calls of step(), bracketed by CUDA events on `stream`;
    with `flush` the 126 MB L2 is overwritten (256 MB) between steps, outside the timed spans."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if flush:
        scratch = torch.empty(256 * 2**20, dtype=torch.uint8, device="cuda")
        total = 0.0
        for k in range(steps):
            scratch.fill_(k & 0xFF)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    import torch
    import torch.distributed as dist
    from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, _lib, replicas
    from fast_ldpc_decoder_for_gpu_fixed_b200.learned import evaluate, load_constants

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    code, enc, cws, idx, llr, sigma = make_workload(args.frames, args.ebn0, args.seed, rank, args.table,
                                                    args.workload)
    code.no_qc = args.no_qc
    words = args.frames // 4
    learned = args.workload == "learned"
    early = args.workload in ("learned", "ira")
    constants = load_constants(args.constants)[:2] if learned else None
    kind = "LEARNED" if learned else args.kind
    es = _early_mode(args) if early else False
    dec = Decoder(code, kind, nb_frames=words, pack=args.pack, early_stop=es)
    if constants is not None:
        dec.set_learned(*constants)
    if early and args.slack is not None:
        dec.set_early_stop(True, args.slack)
    info = dec.info()
    per_frame = info["path"] in (3, 5)  # iteration counts per frame
    stream = torch.cuda.current_stream()
    d_llr = torch.from_numpy(llr.reshape(-1)).cuda()
    d_out = torch.empty(args.frames * code.n, dtype=torch.uint8, device="cuda")
    d_its = torch.zeros(args.frames if per_frame else words, dtype=torch.int32, device="cuda")

    def step():
        dec.decode_device(d_llr, d_out, words, args.iters, _lib.OUT_BYTES, d_its, stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # error rates and iterations of this batch (not timed; every step decodes the same batch)
    hard = d_out.view(args.frames, code.n)
    ref_bits = torch.from_numpy(cws).cuda()[torch.from_numpy(idx).cuda()]
    err = (hard != ref_bits).sum(dim=1)
    fer = float((err > 0).float().mean())
    ber = float(err.sum()) / (args.frames * code.n)
    mean_iters = float(d_its.float().mean()) if early else float(args.iters)
    del ref_bits, err, hard

    flush = llr.nbytes < 2 * 126 * 2**20
    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    ms = _timed(step, args.steps, stream, flush)
    clocks = sampler.stop()
    launches = args.steps
    ms_max = replicas.max_over_ranks(ms, device="cuda")
    ms_step = ms_max / args.steps
    info_bits = args.frames * enc.k
    value = world * info_bits * args.steps / (ms_max * 1e-3) / 1e9

    # the plain 8-bit OMS kernel on the same batch and GPU (the metric's comparison)
    plain = None
    if learned:
        pdec = Decoder(code, "OMS", nb_frames=words, pack=args.pack)

        def pstep():
            pdec.decode_device(d_llr, d_out, words, args.iters, _lib.OUT_BYTES, None, stream)

        for _ in range(args.warmup):
            pstep()
        torch.cuda.synchronize()
        pms = replicas.max_over_ranks(_timed(pstep, args.steps, stream, flush), device="cuda")
        launches += args.steps
        hard = d_out.view(args.frames, code.n)
        ref_bits = torch.from_numpy(cws).cuda()[torch.from_numpy(idx).cuda()]
        perr = (hard != ref_bits).sum(dim=1)
        plain = {"value": world * info_bits * args.steps / (pms * 1e-3) / 1e9, "unit": "Gbit/s",
                 "ms_per_step": pms / args.steps, "kernel": "qc_register_messages" if pdec.info()["path"] == 1
                 else "level_scheduled", "iterations": args.iters, "batch_fer": float((perr > 0).float().mean()),
                 "batch_ber": float(perr.sum()) / (args.frames * code.n)}
        del ref_bits, perr, hard
        pdec.close()

    # plain OMS with the same syndrome early stop: splits vs_plain_oms into the early-stop
    # gain (oms_early_stop / plain_oms) and the learned constants' gain (value / oms_early_stop)
    oms_es = None
    if learned:
        edec = Decoder(code, "OMS", nb_frames=words, pack=args.pack, early_stop=es)
        if args.slack is not None:
            edec.set_early_stop(True, args.slack)
        e_its = torch.zeros(args.frames if per_frame else words, dtype=torch.int32, device="cuda")

        def estep():
            edec.decode_device(d_llr, d_out, words, args.iters, _lib.OUT_BYTES, e_its, stream)

        for _ in range(args.warmup):
            estep()
        torch.cuda.synchronize()
        ems = replicas.max_over_ranks(_timed(estep, args.steps, stream, flush), device="cuda")
        launches += args.steps
        oms_es = {"value": world * info_bits * args.steps / (ems * 1e-3) / 1e9, "unit": "Gbit/s",
                  "ms_per_step": ems / args.steps, "mean_iterations": float(e_its.float().mean()),
                  "early_stop": _early_name(args, per_frame)}
        edec.close()

    # equal-FER evidence on more frames (untimed)
    fer_cmp = None
    if learned and rank == 0 and args.fer_frames > 0:
        fl = evaluate(code, "LEARNED", args.iters, args.ebn0, args.fer_frames, constants=constants, early_stop=es,
                      slack=args.slack)
        fp = evaluate(code, "OMS", args.iters, args.ebn0, args.fer_frames)
        fe = evaluate(code, "OMS", args.iters, args.ebn0, args.fer_frames, early_stop=es, slack=args.slack)
        fer_cmp = {"frames": fl["frames"], "ebn0_db": args.ebn0,
                   "learned_early_stop": {"fer": fl["fer"], "frame_errors": fl["frame_errors"], "ber": fl["ber"],
                                          "mean_iters": fl["mean_iters"]},
                   "oms_early_stop": {"fer": fe["fer"], "frame_errors": fe["frame_errors"], "ber": fe["ber"],
                                      "mean_iters": fe["mean_iters"]},
                   "plain_oms": {"fer": fp["fer"], "frame_errors": fp["frame_errors"], "ber": fp["ber"]}}

    # the ratio across the config-2 Eb/N0 range (untimed by the caller: extra lines of evidence)
    sweep = None
    if learned and rank == 0 and args.sweep:
        sweep = _sweep(code, constants, args, stream)

    # roofline of the decode kernel (one launch per step), from the iterations it executed
    int_peak = _int_peak()
    # the algorithmic work of an edge-update (one frame, one edge, one iteration) is 8 int8
    # lane-ops, i.e. 2 int32 word-ops at 4 lanes per word, whatever the packing of the kernel
    pair_iters = None
    if per_frame:
        edge_updates = float(d_its.sum().item()) * code.e
    elif es == "pairs":
        # the iterations each pair ran: the same frames decoded with each pair doubled into a
        # word of its own (the pairs are independent, so its count is that pair's), untimed
        pair_iters = _pair_counts(code, kind, constants, d_llr, words, args, stream)
        word_max = torch.maximum(pair_iters[:words], pair_iters[words:])
        if not torch.equal(word_max, d_its):
            raise RuntimeError("per-pair iteration counts disagree with the word counts")
        edge_updates = float(pair_iters.sum().item()) * 2 * code.e
    else:
        edge_updates = float(d_its.sum().item()) * 4 * code.e if early else float(args.frames) * code.e * args.iters
    alg_ops = 2.0 * edge_updates
    achieved = alg_ops / (ms_step * 1e-3) / 1e12
    hbm_bytes = args.frames * code.n * 2  # int8 LLRs in + 0/1 bytes out
    peaks = _measured_peaks()

    e2e = e2e_packed = None
    if not args.no_e2e:
        e2e = _e2e(dec, llr, args, info_bits, world)
        e2e_packed = _e2e(dec, llr, args, info_bits, world, packed=True)

    cpu = None
    if rank == 0 and world == 1:
        ckind = "OMS" if learned else args.kind
        v, cores, sample = cpu_baseline(code, llr, min(args.iters, 10) if args.workload == "ira" else args.iters,
                                        ckind, args.cpu_seconds, enc.k)
        cpu = dict({"value": v, "unit": "Gbit/s", "cores": cores, "kind": "port", "sample": sample}, **_cpu_info())

    if rank == 0:
        kernel = {0: "level_scheduled", 1: "qc_register_messages", 2: "level_scheduled_2f",
                  3: "long_code_tma_staged_rows", 4: "qc_register_messages_2f",
                  5: "qc_register_messages_per_frame_refill", 6: "level_scheduled_flooding",
                  7: "qc_register_messages_2f_split_rows"}[info["path"]]
        workload = workload_name(args)
        line = {
            "metric": "decoded info Gbit/s", "value": value, "unit": "Gbit/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8",
            "data": "synthetic (seeded codewords, AWGN, reference quantiser)",
            "config": {"workload": workload, "kind": kind, "pack": info["pack"], "frames_per_gpu": args.frames,
                       "max_iterations": args.iters, "early_stop": _early_name(args, per_frame) if early else False, "mean_iterations": mean_iters,
                       "ebn0_db": args.ebn0, "batch_fer": fer, "batch_ber": ber,
                       "l2": ("inputs %d MB: L2 flushed (256 MB write) between steps, outside the timed spans" % (
                           llr.nbytes // 2**20)) if flush else
                       "inputs (%d MB) larger than the 126 MB L2; no flush" % (llr.nbytes // 2**20),
                       "parallelism": "replicas" if world > 1 else "1gpu", "threads_per_cta": info["threads"],
                       "smem_per_cta": info["smem"], "ctas_per_sm": info["ctas_per_sm"], "regs": info["regs"],
                       "kernel": kernel},
            "plain_oms": plain,
            "vs_plain_oms": value / plain["value"] if plain else None,
            "oms_early_stop": oms_es,
            "early_stop_gain": oms_es["value"] / plain["value"] if oms_es else None,
            "learned_gain": value / oms_es["value"] if oms_es else None,
            "fer": fer_cmp,
            "ebn0_sweep": sweep,
            "roofline": {"bound": "int", "achieved": achieved, "peak": int_peak, "unit": "Tops/s (int32 word-ops)",
                         "frac": achieved / int_peak, "traffic": _traffic(info["path"], args),
                         "peak_nominal": NOMINAL_INT_TOPS, "frac_nominal": achieved / NOMINAL_INT_TOPS,
                         "alg_ops_per_launch": alg_ops, "edge_updates_per_launch": edge_updates,
                         "mean_pair_iterations": float(pair_iters.float().mean()) if pair_iters is not None else None,
                         "ops_per_edge_update": 2.0,
                         "peak_source": "ldpc_probe_int_peak: best measured int32 lane-op rate (LOP3/IADD3 chains, "
                                        "all SMs; profiles/int_peak.md); peak_nominal: 148 SMs x 128 lanes x 1.965 GHz"},
            "roofline_hbm": {"achieved": hbm_bytes / (ms_step * 1e-3) / 1e9, "peak": peaks.get("hbm_gbs"),
                             "peak_source": peaks.get("source", "MEASURED_PEAKS.json"),
                             "unit": "GB/s", "frac": (hbm_bytes / (ms_step * 1e-3) / 1e9) / peaks["hbm_gbs"]
                             if peaks.get("hbm_gbs") else None, "alg_bytes_per_launch": hbm_bytes},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "e2e_packed": e2e_packed,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    dec.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _pair_counts(code, kind, constants, d_llr, words, args, stream):
    """Iterations run by each frame pair under LDPC_FLAG_EARLY_STOP_PAIRS: entry g (g < words)
    is pair 0 of word g, entry words + g its pair 1."""
    import torch
    from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, _lib
    l4 = d_llr.view(words, 4, code.n)
    dup = torch.cat([l4[:, [0, 1, 0, 1]], l4[:, [2, 3, 2, 3]]], 0).reshape(-1).contiguous()
    out = torch.empty(dup.numel(), dtype=torch.uint8, device="cuda")
    its = torch.zeros(2 * words, dtype=torch.int32, device="cuda")
    dec = Decoder(code, kind, nb_frames=2 * words, pack=args.pack, early_stop="pairs")
    if constants is not None:
        dec.set_learned(*constants)
    if args.slack is not None:
        dec.set_early_stop(True, args.slack)
    dec.decode_device(dup, out, 2 * words, args.iters, _lib.OUT_BYTES, its, stream)
    torch.cuda.synchronize()
    dec.close()
    return its


def _early_mode(args):
    """Decoder early_stop argument of the learned workload (the IRA workload's frame path
    stops per frame whatever it is given)."""
    if args.workload != "learned":
        return True
    return {"word": True, "pairs": "pairs", "frame": "frame"}[args.early_unit]


def _early_name(args, per_frame):
    if per_frame:
        return "per_frame"
    unit = "per_pair" if _early_mode(args) == "pairs" else "per_word"
    if args.slack is None:
        return unit
    # slack >= LDPC_EARLY_SLACK_ANY: every iteration a stop candidate
    return unit + (", every iteration a candidate" if args.slack >= (1 << 30) else ", slack %d" % args.slack)


def _sweep(code, constants, args, stream):
    """Learned decoder with early stop vs plain OMS (10 fixed iterations) at each Eb/N0 of the
    config-2 range: kernel Gbit/s of both on 65 536 channel frames, and their FER on 2^18 frames."""
    import torch
    from fast_ldpc_decoder_for_gpu_fixed_b200 import Decoder, _lib
    from fast_ldpc_decoder_for_gpu_fixed_b200.learned import evaluate, random_codewords, sigma_for
    words = args.frames // 4
    cw = torch.from_numpy(random_codewords(code, 64, 77)).cuda()
    llr = torch.empty(4 * words * code.n, dtype=torch.int8, device="cuda")
    out = torch.empty(4 * words * code.n, dtype=torch.uint8, device="cuda")
    es = _early_mode(args)
    its = torch.zeros(4 * words if es == "frame" else words, dtype=torch.int32, device="cuda")
    ldec = Decoder(code, "LEARNED", nb_frames=words, early_stop=es)
    ldec.set_learned(*constants)
    if args.slack is not None:
        ldec.set_early_stop(True, args.slack)
    pdec = Decoder(code, "OMS", nb_frames=words)
    rows = []
    for e in (1.5, 1.75, 2.0, 2.25, 2.5):
        _lib.check(_lib.lib().ldpc_channel_awgn(llr.data_ptr(), 4 * words, code.n, sigma_for(e, code.n_info / code.n),
                                                91, 0, cw.data_ptr(), 64, stream.cuda_stream))
        row = {"ebn0_db": e}
        for name, dec, d_its in (("learned_early_stop", ldec, its), ("plain_oms", pdec, None)):
            def st():
                dec.decode_device(llr, out, words, args.iters, _lib.OUT_BYTES, d_its, stream)
            for _ in range(2):
                st()
            ms = _timed(st, 10, stream, False) / 10
            r = evaluate(code, "LEARNED" if d_its is not None else "OMS", args.iters, e, 1 << 18,
                         constants=constants if d_its is not None else None, early_stop=es if d_its is not None else False,
                         slack=args.slack)
            row[name] = {"gbps": 4 * words * code.n_info / (ms * 1e-3) / 1e9, "fer": r["fer"],
                         "frame_errors": r["frame_errors"], "mean_iters": r["mean_iters"]}
        row["ratio"] = row["learned_early_stop"]["gbps"] / row["plain_oms"]["gbps"]
        rows.append(row)
    ldec.close()
    pdec.close()
    return rows


def _measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(p))
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def _int_peak():
    """INT32 lane-op peak of one B200 in T ops/s: the best measured issue rate of
    independent LOP3 / IADD3 chains on all SMs (ldpc_probe_int_peak; profiles/int_peak.md)."""
    from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib
    import ctypes
    v = ctypes.c_double()
    _lib.check(_lib.lib().ldpc_probe_int_peak(ctypes.byref(v), None))
    return v.value / 1e12


def _e2e(dec, llr, args, info_bits, world, packed=False):
    """Host-buffer decode through the reference-facing call (ldpc_decode_host: 0/1 bytes out,
    like the reference's decode()), or with packed=True through ldpc_decode_host_ex with
    LDPC_OUT_PACKED (n/8 bytes per frame back); copies inside the timed region."""
    import torch
    from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib
    n = llr.shape[1]
    out_bytes = args.frames * ((n + 7) // 8 if packed else n)
    h_in = torch.from_numpy(llr.reshape(-1)).pin_memory()
    h_out = torch.empty(out_bytes, dtype=torch.uint8).pin_memory()
    a_in, a_out = h_in.numpy(), h_out.numpy()
    steps = max(3, min(args.steps, 10))

    def call():
        if packed:
            dec.decode_host_ex(a_in, a_out, args.iters, out_format=_lib.OUT_PACKED)
        else:
            dec.decode_host(a_in, a_out, args.iters)

    for _ in range(2):
        call()
    t = time.perf_counter()
    for _ in range(steps):
        call()
    dt = time.perf_counter() - t
    chunks = min(8, max(1, (args.frames // 4) // 256))
    return {"value": world * info_bits * steps / dt / 1e9, "unit": "Gbit/s", "ms_per_step": dt * 1e3 / steps,
            "h2d_bytes_per_step": int(llr.size), "d2h_bytes_per_step": int(out_bytes),
            "output": "packed bits (ldpc_decode_host_ex)" if packed else "0/1 bytes (ldpc_decode_host)",
            "host_buffers": "pinned", "gpu_launches_per_step": chunks, "steps": steps}


# nominal INT32 rate of one B200: 148 SMs x 128 lanes x 1.965 GHz (T lane-ops/s)
NOMINAL_INT_TOPS = 148 * 128 * 1.965e9 / 1e12

# DRAM bytes (read + write) per frame of the dominant decode kernel, from one ncu capture
# of a smaller batch of the same workload, scaled here by the frames of a launch
# (profiles/decode_qc_exact_gate_qc3x6_n4096_32768f.md: 134.5 MB + 92.3 MB for
# 32 768 frames; the kernel streams each frame's LLRs once and writes its decisions once,
# so the traffic grows with the frames; path 3: profiles/decode_frame_ira_n64800_296f.md,
# 20.0 MB + 74.4 MB for 296 frames of 12 iterations, most of the message traffic in L2)
TRAFFIC_PER_FRAME = {1: (134.5e6 + 92.3e6) / 32768}


def _traffic(path, args):
    per = TRAFFIC_PER_FRAME.get(path) if args.workload == "learned" else None
    return None if per is None else per * args.frames


def _cpu_info():
    from oracle import oracle
    return {"nproc": os.cpu_count(), "cpu_model": oracle.cpu_model(), "isa": oracle.batch_isa()}

if __name__ == "__main__":
    sys.exit(main())
