"""FP64 CPU model of the learned min-sum training pass (test infrastructure).

Restates, in numpy over a batch of frames, the forward and backward passes
that ``fast_ldpc_decoder_for_gpu_fixed_b200/csrc/train.cu`` runs on the GPU:
the row-layered min-sum decoder of ``oracle/ldpc_oracle.c`` (decode_word:
saturating t = APP - message, |t| capped at 127, parity signs with a positive
value meaning bit 1, the 31 clip) with real-valued per-iteration,
per-row-group scale alpha and offset beta:

    c(x) = clamp(alpha * x - beta, 0, 31)         (quantized: floor(alpha * x) - beta)

and the loss sum_t w[t] * mean BCE(sigmoid(kappa_f * APP after iteration t),
transmitted bits) (no weights: the last iteration only), or the soft frame
error rate sum_t w[t] * mean_f (1 - exp(-S_f(t))), S_f the frame's summed BCE.  The backward pass is
the exact reverse of the row sequence, straight-through for min, sign, the
saturations and the floor.  Rows are taken in table order; the GPU's level
order gives the same result because rows of one level share no variable.

``forward_dtype=np.float32`` runs the forward pass in FP32 with one rounding
per operation, which is what the GPU kernel does, so its APPs and decisions
match the kernel bit for bit; the loss and the backward pass stay FP64.

The reference decoders (src/decoder_oms/CUDA_OMS_SIMD.cu:40-134) have no
learned constants, so this model has no reference counterpart beyond the int8
update it generalises: with alpha = 1, beta = 1 and integer LLRs its quantized
forward pass is the XMS decoder; with alpha = s/128 and integer beta it is
LDPC_LEARNED.  Only the tests import this module.
"""
import numpy as np


def _rows(code):
    rp = code.row_ptr
    return [(code.cols[rp[r]:rp[r + 1]], int(code.row_class[r])) for r in range(code.m)]


def _pre(alpha, beta, x, quantized):
    p = alpha * x
    return (np.floor(p) if quantized else p) - beta


def _bce(z, b):
    return np.maximum(z, 0) + np.log1p(np.exp(-np.abs(z))) - b * z


def forward_backward(code, llr, bits, kappa, alpha, beta, quantized=False, backward=True, weights=None,
                     forward_dtype=np.float64, frame_loss=False):
    """llr [F][n] (float), bits [F][n] 0/1 or None, kappa [F], alpha/beta [T][2],
    weights [T] or None.  Returns (loss, app [F][n], d_alpha [T][2], d_beta [T][2]).
    Loss per weighted iteration: mean_f S_f / n, or with ``frame_loss``
    mean_f (1 - exp(-S_f)), S_f the frame's summed bit BCE."""
    ft = forward_dtype
    llr = np.asarray(llr, dtype=ft)
    F, n = llr.shape
    alpha = np.asarray(alpha, dtype=np.float64).reshape(-1, 2)
    beta = np.asarray(beta, dtype=np.float64).reshape(-1, 2)
    T = alpha.shape[0]
    w = np.zeros(T) if weights is None else np.asarray(weights, dtype=np.float64)
    if weights is None:
        w[-1] = 1.0
    rows = _rows(code)
    b = np.zeros((F, n)) if bits is None else np.asarray(bits, dtype=np.float64)
    kappa = np.asarray(kappa, dtype=np.float64).reshape(F, 1)
    count = float(F * n)
    ar = np.arange(F)
    a = llr.copy()
    msg = [np.zeros((F, len(c)), dtype=ft) for c, _ in rows]
    stash, apps, S_all = [], [], []
    loss = 0.0
    for t in range(T):
        st_t = []
        for r, (cols, g) in enumerate(rows):
            d = len(cols)
            al, be = ft(alpha[t, g]), ft(beta[t, g])
            tv = np.clip(a[:, cols] - msg[r], ft(-128), ft(127))
            mag = np.minimum(np.abs(tv), ft(127))
            pos = tv > 0
            order = np.argsort(mag, axis=1, kind="stable")
            i1, i2 = order[:, 0], order[:, 1]
            m1, m2 = mag[ar, i1], mag[ar, i2]
            par = np.logical_xor.reduce(pos, axis=1)
            c1 = np.clip(_pre(al, be, m2, quantized), ft(0), ft(31))
            c2 = np.clip(_pre(al, be, m1, quantized), ft(0), ft(31))
            c = np.repeat(c2[:, None], d, axis=1)
            c[ar, i1] = c1
            m = np.where(par[:, None] ^ pos, c, -c)
            msg[r] = m
            a[:, cols] = np.clip(tv + m, ft(-128), ft(127))
            st_t.append((m1.astype(np.float64), m2.astype(np.float64), i1, i2, pos, par))
        stash.append(st_t)
        apps.append(a.astype(np.float64))
        if w[t] != 0.0:
            S = np.sum(_bce(kappa * apps[t], b), axis=1)
            S_all.append(S)
            loss += w[t] * float(np.mean(1.0 - np.exp(-S)) if frame_loss else np.sum(S) / count)
        else:
            S_all.append(None)
    app = apps[-1].copy()
    if not backward:
        return loss, app, None, None
    ga = np.zeros((F, n))
    gmsg = [np.zeros((F, len(c))) for c, _ in rows]
    d_alpha = np.zeros((T, 2))
    d_beta = np.zeros((T, 2))
    for t in range(T - 1, -1, -1):
        if w[t] != 0.0:
            z = kappa * apps[t]
            coef = np.exp(-S_all[t])[:, None] / F if frame_loss else 1.0 / count
            ga += w[t] * coef * kappa * (1.0 / (1.0 + np.exp(-z)) - b)
        for r in range(len(rows) - 1, -1, -1):
            cols, g = rows[r]
            m1, m2, i1, i2, pos, par = stash[t][r]
            al, be = alpha[t, g], beta[t, g]
            gav = ga[:, cols]
            gm = gav + gmsg[r]
            s = np.where(par[:, None] ^ pos, gm, -gm)
            gc1 = s[ar, i1]
            gc2 = s.sum(axis=1) - gc1
            y1 = _pre(ft(al), ft(be), m2.astype(ft), quantized)
            y2 = _pre(ft(al), ft(be), m1.astype(ft), quantized)
            k1 = (y1 > 0) & (y1 < 31)
            k2 = (y2 > 0) & (y2 < 31)
            d_alpha[t, g] += np.sum(np.where(k1, m2 * gc1, 0.0)) + np.sum(np.where(k2, m1 * gc2, 0.0))
            d_beta[t, g] -= np.sum(np.where(k1, gc1, 0.0)) + np.sum(np.where(k2, gc2, 0.0))
            gm2 = np.where(k1, al * gc1, 0.0)
            gm1 = np.where(k2, al * gc2, 0.0)
            gt = gav.copy()
            gt[ar, i1] += np.where(pos[ar, i1], gm1, -gm1)
            gt[ar, i2] += np.where(pos[ar, i2], gm2, -gm2)
            ga[:, cols] = gt
            gmsg[r] = -gt
    return loss, app, d_alpha, d_beta
