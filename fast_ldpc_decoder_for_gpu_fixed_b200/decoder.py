"""Decoder objects over the C ABI, and Python mirrors of the reference's plugin classes.

The reference's decoder plugins (``src/decoder_template/CGPUDecoder.h:19-35``)
are C++ classes built against one compile-time H matrix:

    CGPUDecoder(size_t nb_frames, size_t n, size_t k, size_t m);
    virtual void initialize() = 0;
    virtual void decode(float var_nodes[_N], int Rprime_fix[_N], int nombre_iterations) = 0;

with subclasses CGPU_Decoder_MS_SIMD, _OMS_SIMD, _NMS_SIMD, _2NMS_SIMD and
CGPU_Decoder_MS_SIMD_v2 (``-xMS``), chosen in ``src/main.cpp:213-228``.
``nb_frames`` counts 32-bit lanes (4 codewords each); ``decode`` takes the
frame-major int8 LLRs of 4*nb_frames codewords (typed float* in the reference)
and writes frame-major 0/1 bytes (typed int*).  The classes below keep those
names, arguments and meanings; the H matrix is the module's selected code
(``select_code``, default "4000x2000" like ``src/matrix/code.h:1``), and
errors raise ``LdpcError`` instead of the reference's exit(0).
The C++ equivalents of these classes are in ``cpp/CGPUDecoder.h``.
"""
import ctypes

import numpy as np

from . import _lib
from .codes import Code, load_table


class NativeCode:
    """An ldpc_code handle (H matrix + level schedule) built from a ``Code``."""

    def __init__(self, code):
        self.code = code
        h = ctypes.c_void_p()
        if getattr(code, "shifts", None) is not None and not getattr(code, "no_qc", False):
            sh = np.where(code.base > 0, code.shifts, -1).astype(np.int32)
            _lib.check(_lib.lib().ldpc_code_create_qc(ctypes.byref(h), int(code.z), sh.shape[0], sh.shape[1],
                                                      sh.ctypes.data))
        else:
            _lib.check(_lib.lib().ldpc_code_create(
                ctypes.byref(h), code.n, code.m, code.row_ptr.ctypes.data, code.cols.ctypes.data,
                code.row_class.ctypes.data))
        self.handle = h

    def info(self):
        a = (ctypes.c_int * 8)()
        _lib.check(_lib.lib().ldpc_code_info(self.handle, a))
        keys = ("n", "checks", "edges", "dmax", "levels", "widest_level", "n_info")
        return dict(zip(keys, list(a)))

    def close(self):
        if self.handle:
            _lib.lib().ldpc_code_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(x):
    """Raw address of a numpy array, a torch tensor, an int or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError("cannot take the address of %r" % type(x))


class Decoder:
    """One ldpc_decoder: ``kind`` in MS/OMS/NMS/2NMS/XMS/LEARNED, ``nb_frames`` 32-bit
    lanes (4*nb_frames codewords per call), ``pack`` in AUTO/SIMD4/F16X2/I8;
    ``early_stop`` sets LDPC_FLAG_EARLY_STOP (syndrome early stop per word), or with
    ``early_stop="frame"`` LDPC_FLAG_EARLY_STOP_FRAMES (per frame, finished frames'
    slots refilled; iteration counts per frame), ``early_stop="pairs"``
    LDPC_FLAG_EARLY_STOP_PAIRS (each frame pair of a word on its own); ``flooding`` sets
    LDPC_FLAG_FLOODING."""

    def __init__(self, code, kind="OMS", nb_frames=1024, pack="AUTO", early_stop=False, flooding=False):
        if isinstance(code, str):
            code = load_table(code)
        self.code = code if isinstance(code, Code) else code.code
        self.native = code if isinstance(code, NativeCode) else NativeCode(self.code)
        self.kind = kind.upper()
        self.nb_frames = int(nb_frames)
        h = ctypes.c_void_p()
        if early_stop == "frame":
            flags = _lib.FLAG_EARLY_STOP_FRAMES
        elif early_stop == "pairs":
            flags = _lib.FLAG_EARLY_STOP_PAIRS
        else:
            flags = _lib.FLAG_EARLY_STOP if early_stop else 0
        if flooding:
            flags |= _lib.FLAG_FLOODING
        _lib.check(_lib.lib().ldpc_decoder_create(
            ctypes.byref(h), self.native.handle, _lib.KINDS[self.kind], self.nb_frames,
            _lib.PACKS[pack.upper()], flags))
        self.handle = h
        self.early_stop = bool(early_stop)
        self.per_frame = early_stop == "frame"
        self.pairs = early_stop == "pairs"
        self.early_slack = _lib.EARLY_STOP_DEFAULT_SLACK

    def info(self):
        a = (ctypes.c_int * 8)()
        _lib.check(_lib.lib().ldpc_decoder_info(self.handle, a))
        keys = ("kind", "pack", "nb_frames", "threads", "smem", "ctas_per_sm", "regs", "path")
        return dict(zip(keys, list(a)))

    def set_early_stop(self, enabled=True, slack=_lib.EARLY_STOP_DEFAULT_SLACK):
        """Syndrome early stop on/off and its slack (ldpc_decoder_set_early_stop)."""
        _lib.check(_lib.lib().ldpc_decoder_set_early_stop(self.handle, int(bool(enabled)), int(slack)))
        self.early_stop = bool(enabled)
        self.early_slack = int(slack)

    def status(self):
        """1 when a kernel of this decoder gave up waiting on a bulk copy since the last
        call (ldpc_decoder_status), else 0."""
        st = ctypes.c_int(0)
        _lib.check(_lib.lib().ldpc_decoder_status(self.handle, ctypes.byref(st)))
        return st.value

    def set_learned(self, offsets, scales):
        """LDPC_LEARNED constants: [n_iters][2] int8 offsets and uint8 Q1.7 scales."""
        off = np.ascontiguousarray(offsets, dtype=np.int8).reshape(-1, 2)
        sc = np.ascontiguousarray(scales, dtype=np.uint8).reshape(-1, 2)
        _lib.check(_lib.lib().ldpc_decoder_set_learned(self.handle, off.shape[0], off.ctypes.data, sc.ctypes.data))

    def decode_host(self, llr, hard, iters):
        """Synchronous host-buffer decode of all 4*nb_frames codewords (numpy arrays)."""
        n_bytes = 4 * self.nb_frames * self.code.n
        if llr.nbytes < n_bytes or hard.nbytes < n_bytes:
            raise ValueError("buffers must hold %d bytes" % n_bytes)
        if not (llr.flags.c_contiguous and hard.flags.c_contiguous and hard.flags.writeable):
            raise ValueError("buffers must be C-contiguous (and hard writeable)")
        _lib.check(_lib.lib().ldpc_decode_host(self.handle, _ptr(llr), _ptr(hard), int(iters)))
        return hard

    def decode_host_ex(self, llr, out, iters, out_format=_lib.OUT_BYTES, iters_out=None, syndrome_ok=None):
        """Host-buffer decode of all 4*nb_frames codewords with packed output and the
        per-word iteration counts / per-frame syndrome flags (ldpc_decode_host_ex)."""
        n_bytes = 4 * self.nb_frames * self.code.n
        o_bytes = 4 * self.nb_frames * ((self.code.n + 7) // 8 if out_format == _lib.OUT_PACKED else self.code.n)
        if llr.nbytes < n_bytes or out.nbytes < o_bytes:
            raise ValueError("buffers must hold %d and %d bytes" % (n_bytes, o_bytes))
        if syndrome_ok is not None and syndrome_ok.nbytes < 4 * self.nb_frames:
            raise ValueError("syndrome_ok must hold %d bytes" % (4 * self.nb_frames))
        _lib.check(_lib.lib().ldpc_decode_host_ex(self.handle, _ptr(llr), _ptr(out), int(iters), int(out_format),
                                                  _ptr(iters_out), _ptr(syndrome_ok)))
        return out

    def decode_device(self, d_llr, d_out, n_words, iters, out_format=_lib.OUT_BYTES, d_iters=None, stream=None,
                      d_syndrome=None):
        """Asynchronous device-buffer decode of 4*n_words codewords on ``stream`` (a raw
        cudaStream_t value, a torch stream or None for the legacy default stream);
        ``d_syndrome`` (4*n_words bytes) receives the per-frame syndrome flags."""
        st = getattr(stream, "cuda_stream", stream)
        _lib.check(_lib.lib().ldpc_decode_device(self.handle, _ptr(d_llr), _ptr(d_out), int(n_words), int(iters),
                                                 int(out_format), _ptr(d_iters), _ptr(d_syndrome), st))

    def decode_device_state(self, d_llr, d_hard, n_words, iters, d_iters=None, d_app=None, d_msg=None,
                            stream=None):
        st = getattr(stream, "cuda_stream", stream)
        _lib.check(_lib.lib().ldpc_decode_device_state(self.handle, _ptr(d_llr), _ptr(d_hard), int(n_words),
                                                       int(iters), _ptr(d_iters), _ptr(d_app), _ptr(d_msg), st))

    def simulate(self, n_words, iters, sigma, seed, offset, d_counts, d_codewords=None, n_codewords=0,
                 n_vars=None, d_hard=None, stream=None):
        """Fused channel + decode + error count of 4*n_words frames (device buffers)."""
        st = getattr(stream, "cuda_stream", stream)
        nv = self.code.n_info if n_vars is None else n_vars
        _lib.check(_lib.lib().ldpc_simulate(self.handle, int(n_words), int(iters), float(sigma), int(seed),
                                            int(offset), _ptr(d_codewords), int(n_codewords), int(nv),
                                            _ptr(d_counts), _ptr(d_hard), st))

    def train_stash_bytes(self, frames, iters):
        """Device bytes of the stash ``train_step`` needs for a backward pass."""
        return int(_lib.lib().ldpc_train_stash_bytes(self.handle, int(frames), int(iters)))

    def train_step(self, d_llr, d_kappa, frames, iters, d_alpha, d_beta, d_loss, d_bits=None, quantized=False,
                   d_grad_alpha=None, d_grad_beta=None, d_stash=None, d_app=None, d_weights=None,
                   frame_loss=False, stream=None):
        """FP32 forward (and, with gradient buffers and a stash, backward) pass of the
        learned min-sum decoder over ``frames`` frames (device buffers; see
        ldpc_train_step in include/ldpc_b200.h)."""
        st = getattr(stream, "cuda_stream", stream)
        flags = (_lib.TRAIN_QUANTIZED if quantized else 0) | (_lib.TRAIN_FRAME_LOSS if frame_loss else 0)
        _lib.check(_lib.lib().ldpc_train_step(
            self.handle, _ptr(d_llr), _ptr(d_bits), _ptr(d_kappa), int(frames), int(iters), flags,
            _ptr(d_alpha), _ptr(d_beta), _ptr(d_weights), _ptr(d_grad_alpha), _ptr(d_grad_beta), _ptr(d_loss),
            _ptr(d_stash), _ptr(d_app), st))

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib().ldpc_decoder_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several codes decoded by one persistent kernel (ldpc_batch_*).  ``codes``: a
    list of ``Code``; ``graph``: capture launches in a CUDA graph; buffers are
    lists (one torch CUDA tensor per code)."""

    def __init__(self, codes, kind="OMS", pack="AUTO", early_stop=False, graph=False):
        self.codes = [c if isinstance(c, Code) else c.code for c in codes]
        self.natives = [NativeCode(c) for c in self.codes]
        self.kind = kind.upper()
        arr = (ctypes.c_void_p * len(codes))(*[nc.handle.value for nc in self.natives])
        h = ctypes.c_void_p()
        if early_stop == "frame":
            flags = _lib.FLAG_EARLY_STOP_FRAMES
        else:
            flags = _lib.FLAG_EARLY_STOP if early_stop else 0
        flags |= _lib.BATCH_GRAPH if graph else 0
        _lib.check(_lib.lib().ldpc_batch_create(ctypes.byref(h), arr, len(codes), _lib.KINDS[self.kind],
                                                _lib.PACKS[pack.upper()], flags))
        self.handle = h

    @staticmethod
    def _arrays(d_llr, d_out, n_words, d_iters):
        n = len(d_llr)
        llr = (ctypes.c_void_p * n)(*[_ptr(x) for x in d_llr])
        out = (ctypes.c_void_p * n)(*[_ptr(x) for x in d_out])
        words = (ctypes.c_size_t * n)(*[int(w) for w in n_words])
        its = (ctypes.c_void_p * n)(*[_ptr(x) for x in d_iters]) if d_iters is not None else None
        return llr, out, words, its

    def decode(self, d_llr, d_out, n_words, iters, out_format=_lib.OUT_BYTES, d_iters=None, stream=None,
               d_syndrome=None):
        st = getattr(stream, "cuda_stream", stream)
        llr, out, words, its = self._arrays(d_llr, d_out, n_words, d_iters)
        syn = (ctypes.c_void_p * len(d_llr))(*[_ptr(x) for x in d_syndrome]) if d_syndrome is not None else None
        _lib.check(_lib.lib().ldpc_batch_decode(self.handle, llr, out, words, int(iters), int(out_format), its, syn,
                                                st))

    def autotune(self, d_llr, d_out, n_words, iters, d_iters=None, stream=None):
        """Picks the fastest packing / CTA width / residency on these inputs; returns ms per decode."""
        st = getattr(stream, "cuda_stream", stream)
        llr, out, words, its = self._arrays(d_llr, d_out, n_words, d_iters)
        best = ctypes.c_double()
        _lib.check(_lib.lib().ldpc_batch_autotune(self.handle, llr, out, words, int(iters), its,
                                                  ctypes.byref(best), st))
        return best.value

    def configure(self, per_code=False, pack="SIMD4", threads=128, ctas_per_sm=0):
        """The strategy by hand (ldpc_batch_configure)."""
        _lib.check(_lib.lib().ldpc_batch_configure(self.handle, int(bool(per_code)), _lib.PACKS[pack.upper()],
                                                   int(threads), int(ctas_per_sm)))

    def status(self):
        """1 when a kernel of this decoder gave up waiting on a bulk copy since the last
        call (ldpc_decoder_status), else 0."""
        st = ctypes.c_int(0)
        _lib.check(_lib.lib().ldpc_decoder_status(self.handle, ctypes.byref(st)))
        return st.value

    def set_learned(self, offsets, scales):
        off = np.ascontiguousarray(offsets, dtype=np.int8).reshape(-1, 2)
        sc = np.ascontiguousarray(scales, dtype=np.uint8).reshape(-1, 2)
        _lib.check(_lib.lib().ldpc_batch_set_learned(self.handle, off.shape[0], off.ctypes.data, sc.ctypes.data))

    def set_early_stop(self, enabled=True, slack=_lib.EARLY_STOP_DEFAULT_SLACK):
        _lib.check(_lib.lib().ldpc_batch_set_early_stop(self.handle, int(bool(enabled)), int(slack)))

    def set_code_kernel(self, candidates):
        """Per-code kernels (ldpc_batch_set_code_kernel): one candidate number per code
        (0 SIMD4, 1 F16X2, 2 I8 level kernels, 3 QC register kernel, 4 flooding)."""
        for i, c in enumerate(candidates):
            self.set_code_kernel_one(i, c)

    def set_code_kernel_one(self, i, candidate):
        """Code i's per-code kernel (ldpc_batch_set_code_kernel)."""
        _lib.check(_lib.lib().ldpc_batch_set_code_kernel(self.handle, int(i), int(candidate)))

    def code_info(self, i):
        """The per-code strategy's kernel of code i (ldpc_batch_code_info)."""
        a = (ctypes.c_int * 5)()
        _lib.check(_lib.lib().ldpc_batch_code_info(self.handle, int(i), a))
        names = {0: "SIMD4", 1: "F16X2", 2: "I8", 3: "QC", 4: "FLOODING", 5: "QC_SPLIT"}
        return {"candidate": names.get(a[0], a[0]), "path": a[1], "threads": a[2], "smem": a[3],
                "ctas_per_sm": a[4]}

    def info(self):
        a = (ctypes.c_int * 9)()
        _lib.check(_lib.lib().ldpc_batch_info(self.handle, a))
        keys = ("kind", "pack", "threads", "smem", "ctas_per_sm", "grid", "graph", "codes", "per_code")
        return dict(zip(keys, list(a)))

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib().ldpc_batch_destroy(self.handle)
            self.handle = None
        for nc in getattr(self, "natives", []):
            nc.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# reference-compatible plugin classes
# ---------------------------------------------------------------------------

_selected = {"code": None, "name": "4000x2000"}


def select_code(code):
    """Selects the H matrix the plugin classes use (the reference's src/matrix/code.h)."""
    if isinstance(code, str):
        _selected["name"], _selected["code"] = code, None
    else:
        _selected["name"], _selected["code"] = code.name, code


def selected_code():
    if _selected["code"] is None:
        _selected["code"] = load_table(_selected["name"])
    return _selected["code"]


class CGPUDecoder:
    """Mirror of decoder_template/CGPUDecoder.h:19-35 (abstract; use a subclass)."""
    KIND = None

    def __init__(self, nb_frames, n, k, m, pack="AUTO"):
        code = selected_code()
        if (n, k, m) != (code.n, code.m, code.e):
            raise ValueError("decoder built for (N,K,M)=(%d,%d,%d) but the selected code is (%d,%d,%d)"
                             % (n, k, m, code.n, code.m, code.e))
        if self.KIND is None:
            raise TypeError("CGPUDecoder is abstract")
        self.nb_frames = int(nb_frames)
        self.sz_nodes = n * self.nb_frames
        self.sz_checks = k * self.nb_frames
        self.sz_msgs = m * self.nb_frames
        self._dec = Decoder(code, self.KIND, self.nb_frames, pack)

    def initialize(self):
        pass

    def decode(self, var_nodes, Rprime_fix, nombre_iterations):
        """var_nodes: 4*nb_frames*N int8 LLRs (any dtype, read as bytes);
        Rprime_fix: writable buffer of the same byte size receiving 0/1 bytes."""
        llr = np.ascontiguousarray(var_nodes).view(np.int8).reshape(-1)
        out = Rprime_fix.view(np.uint8).reshape(-1)
        self._dec.decode_host(llr, out, nombre_iterations)

    def close(self):
        self._dec.close()


class CGPU_Decoder_MS_SIMD(CGPUDecoder):
    """-MS / -fMS (decoder_ms/CGPU_Decoder_MS_SIMD.cu)."""
    KIND = "MS"


class CGPU_Decoder_OMS_SIMD(CGPUDecoder):
    """-OMS (decoder_oms/CGPU_Decoder_OMS_SIMD.cu)."""
    KIND = "OMS"


class CGPU_Decoder_NMS_SIMD(CGPUDecoder):
    """-NMS (decoder_nms/CGPU_Decoder_NMS_SIMD.cu)."""
    KIND = "NMS"


class CGPU_Decoder_2NMS_SIMD(CGPUDecoder):
    """-2NMS (decoder_2nms/CGPU_Decoder_2NMS_SIMD.cu)."""
    KIND = "2NMS"


class CGPU_Decoder_MS_SIMD_v2(CGPUDecoder):
    """-xMS (decoder_oms_v2/CGPU_Decoder_MS_SIMD_v2.cu): input already word-interleaved."""
    KIND = "XMS"


PLUGINS = {"fMS": CGPU_Decoder_MS_SIMD, "MS": CGPU_Decoder_MS_SIMD, "OMS": CGPU_Decoder_OMS_SIMD,
           "NMS": CGPU_Decoder_NMS_SIMD, "2NMS": CGPU_Decoder_2NMS_SIMD, "xMS": CGPU_Decoder_MS_SIMD_v2}
