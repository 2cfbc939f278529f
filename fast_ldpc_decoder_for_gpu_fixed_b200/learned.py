"""Learned min-sum: training of the LDPC_LEARNED constants on the GPU, their
quantisation, and FER/BER evaluation against plain OMS.

The reference (src/decoder_oms/CUDA_OMS_SIMD.cu:73-74) uses one fixed offset
(1) for every iteration.  LDPC_LEARNED replaces it by an offset and a scale per
iteration and per row group, c = clamp(floor(min * scale / 128) - offset, 0, 31).
They are trained here in FP32 by the project's own forward and backward kernels
(ldpc_train_step, csrc/train.cu) through the unrolled layered decoder, on frames
that the AWGN channel kernel (ldpc_channel_awgn) generates at Eb/N0 drawn
uniformly from a range.  The loss is the BCE of the soft outputs ("bit") or a
soft frame error rate ("frame": 1 - exp(-summed BCE) per frame), of the last
iteration or of every iteration ("all", which rewards early convergence).
Training runs in two phases: the real-valued relaxation, then
quantisation-aware steps whose forward pass is exactly the int8 decoder
(floored scale, integer offset), with straight-through gradients.
Finally the constants are frozen to int8 offsets and Q1.7 scales.

PyTorch only holds the buffers and applies Adam to the 4*T parameters; every
decoder pass is one of this library's kernels.
"""
import os

import numpy as np

from . import _lib
from .codes import Encoder, IRAEncoder
from .decoder import Decoder


def sigma_for(ebn0, rate):
    """Noise deviation of the channel at Eb/N0 (dB) and code rate (ldpc_sigma)."""
    return float(_lib.lib().ldpc_sigma(float(ebn0), float(rate), 0))


def random_codewords(code, count, seed):
    """``count`` codewords of random information bits (seeded), frame-major uint8."""
    rng = np.random.default_rng(seed)
    enc = IRAEncoder(code) if getattr(code, "ira_k", None) else Encoder(code)
    return enc.encode(rng.integers(0, 2, size=(count, enc.k)))


SCALE_STEP = 8   # Q1.7 scales on a 1/16 grid: what the fp16 (QC) kernels compute exactly
OFFSET_MAX = 31


def quantize(alpha, beta, scale_step=SCALE_STEP):
    """FP32 scales/offsets [T][2] -> (int8 offsets in [-31, 31], uint8 Q1.7 scales,
    multiples of ``scale_step``)."""
    alpha = np.asarray(alpha, dtype=np.float64)
    beta = np.asarray(beta, dtype=np.float64)
    off = np.clip(np.rint(beta), -OFFSET_MAX, OFFSET_MAX).astype(np.int8)
    top = 255 // scale_step * scale_step
    sc = np.clip(np.rint(alpha * 128.0 / scale_step) * scale_step, 0, top).astype(np.uint8)
    return off, sc


class Trainer:
    """Trains per-iteration, per-row-group scales and offsets for ``code``.

    Each step draws ``batch`` frames: ``batch // sub`` channel calls of ``sub``
    frames, each at its own Eb/N0 ~ U[ebn0], over ``n_codewords`` seeded random
    codewords (``sub`` must be a multiple of ``n_codewords``).  ``iters`` is the
    number of unrolled decoder iterations (at most 32).
    """

    def __init__(self, code, iters=10, batch=4096, sub=512, ebn0=(1.0, 3.0), lr=0.03, seed=1,
                 n_codewords=256, init_alpha=1.0, init_beta=1.0, weights="last", loss="bit", device="cuda",
                 train_scales=True):
        import torch
        if sub % n_codewords or batch % sub:
            raise ValueError("batch must be a multiple of sub, and sub a multiple of n_codewords")
        self.torch = torch
        self.code = code
        self.T = int(iters)
        self.batch = int(batch)
        self.sub = int(sub)
        self.ebn0 = tuple(ebn0)
        self.rate = code.n_info / code.n
        self.seed = int(seed)
        self.rng = np.random.default_rng(seed)
        self.dec = Decoder(code, "OMS", nb_frames=1)   # supplies the code's row schedule
        dev = torch.device(device)
        cw = random_codewords(code, n_codewords, seed + 7)
        self.d_cw = torch.from_numpy(cw).to(dev)
        self.n_cw = n_codewords
        self.d_bits = self.d_cw.repeat(batch // n_codewords, 1).contiguous()
        self.d_llr8 = torch.zeros(batch, code.n, dtype=torch.int8, device=dev)
        self.d_llr = torch.zeros(batch, code.n, dtype=torch.float32, device=dev)
        self.d_kappa = torch.zeros(batch, dtype=torch.float32, device=dev)
        self.d_stash = torch.empty(self.dec.train_stash_bytes(batch, self.T), dtype=torch.uint8, device=dev)
        self.d_loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.alpha = torch.full((self.T, 2), float(init_alpha), dtype=torch.float32, device=dev, requires_grad=True)
        self.beta = torch.full((self.T, 2), float(init_beta), dtype=torch.float32, device=dev, requires_grad=True)
        self.alpha.grad = torch.zeros_like(self.alpha)
        self.beta.grad = torch.zeros_like(self.beta)
        # train_scales=False: the scales stay at init_alpha (1.0: a learned-offset decoder, whose
        # deployed kernel computes min - offset like OMS) and only the offsets are trained
        self.train_scales = bool(train_scales)
        self.opt = torch.optim.Adam([self.alpha, self.beta] if self.train_scales else [self.beta], lr=lr)
        # loss weight per iteration: "last" (the final soft output only) or "all"
        # (every iteration's soft output, which rewards early convergence)
        if isinstance(weights, str):
            w = np.zeros(self.T, dtype=np.float32)
            if weights == "last":
                w[-1] = 1.0
            elif weights == "all":
                w[:] = 1.0 / self.T
            else:
                raise ValueError("weights: 'last', 'all' or an array of %d floats" % self.T)
        else:
            w = np.asarray(weights, dtype=np.float32).reshape(self.T)
        self.d_weights = torch.from_numpy(w).to(dev)
        if loss not in ("bit", "frame"):
            raise ValueError("loss: 'bit' (mean BCE) or 'frame' (soft frame error rate)")
        self.frame_loss = loss == "frame"
        self.calls = 0
        self.history = []

    def _frames(self):
        """Fills the LLR batch from the channel kernel; kappa = 2/sigma^2 / 8 per frame."""
        for j in range(self.batch // self.sub):
            e = float(self.rng.uniform(*self.ebn0))
            s = sigma_for(e, self.rate)
            _lib.check(_lib.lib().ldpc_channel_awgn(
                self.d_llr8[j * self.sub:(j + 1) * self.sub].data_ptr(), self.sub, self.code.n, s,
                self.seed, self.calls, self.d_cw.data_ptr(), self.n_cw,
                self.torch.cuda.current_stream().cuda_stream))
            self.calls += 1
            self.d_kappa[j * self.sub:(j + 1) * self.sub] = 1.0 / (4.0 * s * s)
        self.d_llr.copy_(self.d_llr8)

    def _used(self, quantized):
        if not quantized:
            return self.alpha.detach(), self.beta.detach()
        q = 128.0 / SCALE_STEP
        return (self.torch.round(self.alpha.detach() * q) / q).contiguous(), \
            self.torch.round(self.beta.detach()).contiguous()

    def step(self, quantized=False):
        """One training step; returns the loss as a device tensor (no sync)."""
        self._frames()
        a, b = self._used(quantized)
        self.alpha.grad.zero_()
        self.beta.grad.zero_()
        self.d_loss.zero_()
        self.dec.train_step(self.d_llr, self.d_kappa, self.batch, self.T, a, b, self.d_loss,
                            d_bits=self.d_bits, quantized=quantized, d_grad_alpha=self.alpha.grad,
                            d_grad_beta=self.beta.grad, d_stash=self.d_stash, d_weights=self.d_weights,
                            frame_loss=self.frame_loss, stream=self.torch.cuda.current_stream())
        self.opt.step()
        with self.torch.no_grad():
            self.alpha.clamp_(0.0, (255 // SCALE_STEP * SCALE_STEP) / 128.0)
            self.beta.clamp_(-8.0, float(OFFSET_MAX))
        return self.d_loss.clone()

    def train(self, frames, qat_fraction=0.3, log_every=16):
        """Trains on ``frames`` frames in total; the last ``qat_fraction`` of the
        steps run the quantized forward pass.  Returns the loss history."""
        steps = max(1, int(frames) // self.batch)
        q0 = int(round(steps * (1.0 - qat_fraction)))
        pending = []
        for i in range(steps):
            pending.append((i, self.step(quantized=i >= q0)))
            if len(pending) >= log_every or i == steps - 1:
                for k, l in pending:
                    self.history.append((k, float(l.item())))
                pending = []
        return self.history

    def validation_loss(self, ebn0, quantized=True, seed=99):
        """Loss of the current constants on one fixed batch at ``ebn0`` dB
        (forward pass only; comparable across calls)."""
        s = sigma_for(ebn0, self.rate)
        _lib.check(_lib.lib().ldpc_channel_awgn(self.d_llr8.data_ptr(), self.batch, self.code.n, s, seed, 0,
                                                self.d_cw.data_ptr(), self.n_cw,
                                                self.torch.cuda.current_stream().cuda_stream))
        self.d_llr.copy_(self.d_llr8)
        self.d_kappa.fill_(1.0 / (4.0 * s * s))
        a, b = self._used(quantized)
        self.d_loss.zero_()
        self.dec.train_step(self.d_llr, self.d_kappa, self.batch, self.T, a, b, self.d_loss, d_bits=self.d_bits,
                            quantized=quantized, d_weights=self.d_weights, frame_loss=self.frame_loss,
                            stream=self.torch.cuda.current_stream())
        return float(self.d_loss.item())

    def constants(self):
        """The frozen (int8 offsets, uint8 Q1.7 scales), [T][2] each."""
        return quantize(self.alpha.detach().cpu().numpy(), self.beta.detach().cpu().numpy())

    def close(self):
        self.dec.close()


def evaluate(code, kind, iters, ebn0, frames, seed=11, constants=None, n_codewords=256, words_per_call=4096,
             pack="AUTO", early_stop=False, slack=None):
    """Frame and bit error rates and mean iterations of the int8 decoder ``kind``
    (with LDPC_LEARNED ``constants`` = (offsets, scales)) at ``ebn0`` dB over at
    least ``frames`` frames of seeded random codewords: channel kernel, decode
    with per-word iteration counts, error-count kernel.  Errors are counted over
    all n bits.  ``early_stop="frame"``: the per-frame early stop, and mean_iters is
    per frame.  ``slack``: the early stop's slack (ldpc_decoder_set_early_stop; None: the
    library's default).  Returns dict(frames, bit_errors, frame_errors, fer, ber, mean_iters)."""
    import torch
    words = min(words_per_call, max(1, (frames + 3) // 4))
    dec = Decoder(code, kind, nb_frames=words, pack=pack, early_stop=early_stop)
    if constants is not None:
        dec.set_learned(*constants)
    if early_stop and slack is not None:
        dec.set_early_stop(True, slack)
    cw = torch.from_numpy(random_codewords(code, n_codewords, seed + 3)).cuda()
    llr = torch.empty(4 * words * code.n, dtype=torch.int8, device="cuda")
    hard = torch.empty(4 * words * code.n, dtype=torch.uint8, device="cuda")
    per_frame = early_stop == "frame"  # iteration counts per frame, not per word
    its = torch.zeros(4 * words if per_frame else words, dtype=torch.int32, device="cuda")
    it_sum = torch.zeros(1, dtype=torch.int64, device="cuda")
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    s = sigma_for(ebn0, code.n_info / code.n)
    st = torch.cuda.current_stream()
    calls = (frames + 4 * words - 1) // (4 * words)
    for c in range(calls):
        _lib.check(_lib.lib().ldpc_channel_awgn(llr.data_ptr(), 4 * words, code.n, s, seed, c, cw.data_ptr(),
                                                n_codewords, st.cuda_stream))
        dec.decode_device(llr, hard, words, iters, d_iters=its, stream=st)
        _lib.check(_lib.lib().ldpc_count_errors(hard.data_ptr(), 4 * words, code.n, code.n, cw.data_ptr(),
                                                n_codewords, counts.data_ptr(), st.cuda_stream))
        it_sum += its.sum()
    torch.cuda.synchronize()
    dec.close()
    f, be, fe = (int(x) for x in counts.cpu().tolist())
    return {"frames": f, "bit_errors": be, "frame_errors": fe, "fer": fe / f, "ber": be / (f * code.n),
            "mean_iters": float(it_sum.item()) / (calls * its.numel())}


def save_constants(path, offsets, scales, **meta):
    """Writes frozen constants ([T][2] int8 offsets, uint8 Q1.7 scales) and metadata as JSON."""
    import json
    doc = dict(meta)
    doc["offsets"] = np.asarray(offsets, dtype=np.int8).tolist()
    doc["scales"] = np.asarray(scales, dtype=np.uint8).tolist()
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)


def load_constants(path):
    """(offsets, scales, metadata) from a file written by ``save_constants``."""
    import json
    with open(path) as f:
        doc = json.load(f)
    return np.asarray(doc["offsets"], dtype=np.int8), np.asarray(doc["scales"], dtype=np.uint8), doc


TRAINED_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "trained")


def _code_by_name(name):
    from .codes import load_table, qc_regular
    if name == "qc3x6_z256":
        return qc_regular(z=256, mb=8, nb=16, wc=3, seed=2024, name="qc3x6_z256")
    return load_table(name)


def main(argv=None):
    """python -m fast_ldpc_decoder_for_gpu_fixed_b200.learned --code qc3x6_z256 --out FILE:
    trains, evaluates against plain OMS and writes the frozen constants."""
    import argparse
    import time
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--code", default="qc3x6_z256")
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--frames", type=int, default=2_000_000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--ebn0", type=float, nargs=2, default=(1.0, 3.0))
    ap.add_argument("--loss", default="bit", choices=("bit", "frame"))
    ap.add_argument("--weights", default="all", choices=("all", "last"))
    ap.add_argument("--init", default="oms", choices=("oms", "ms"))
    ap.add_argument("--qat", type=float, default=1.0, help="fraction of the steps with the quantised forward pass")
    ap.add_argument("--lr", type=float, default=0.01)
    ap.add_argument("--offsets-only", action="store_true",
                    help="keep every scale at 1.0 and train the offsets only (a learned-offset decoder)")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--eval-ebn0", type=float, nargs="*", default=(1.75, 2.0, 2.25))
    ap.add_argument("--eval-frames", type=int, default=262144)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    code = _code_by_name(a.code)
    tr = Trainer(code, iters=a.iters, batch=a.batch, lr=a.lr, seed=a.seed, weights=a.weights, loss=a.loss,
                 init_alpha=1.0, init_beta=1.0 if a.init == "oms" else 0.0, ebn0=tuple(a.ebn0),
                 train_scales=not a.offsets_only)
    v0 = tr.validation_loss(2.0)
    t0 = time.time()
    tr.train(a.frames, qat_fraction=a.qat)
    dt = time.time() - t0
    v1 = tr.validation_loss(2.0)
    off, sc = tr.constants()
    tr.close()
    evals = []
    for e in a.eval_ebn0:
        row = {"ebn0_db": e}
        for name, kind, c in (("oms", "OMS", None), ("learned", "LEARNED", (off, sc))):
            r = evaluate(code, kind, a.iters, e, a.eval_frames, constants=c, early_stop=True)
            row[name] = {"fer": r["fer"], "frame_errors": r["frame_errors"], "ber": r["ber"],
                         "mean_iters": r["mean_iters"]}
        evals.append(row)
    meta = {"code": a.code, "iterations": a.iters, "frames": a.frames, "batch": a.batch, "ebn0_db": list(a.ebn0),
            "loss": a.loss, "weights": a.weights, "init": a.init, "qat_fraction": a.qat, "lr": a.lr, "seed": a.seed,
            "offsets_only": bool(a.offsets_only),
            "train_seconds": round(dt, 2), "validation_loss_2db": [v0, v1],
            "evaluation": evals, "evaluation_frames": a.eval_frames}
    import json
    print(json.dumps(meta), flush=True)
    if a.out:
        save_constants(a.out, off, sc, **meta)
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
