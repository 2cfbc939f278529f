"""B200-native (sm_100a) fixed-point LDPC decoding engine.

Drop-in for the decoder plugins of blegal/Fast_LDPC_decoder_for_GPU_fixed:
hand-written CUDA kernels behind a C ABI (include/ldpc_b200.h,
libldpc_b200.so), with Python (``decoder``) and C++ (``cpp/CGPUDecoder.h``)
mirrors of the reference's ``CGPUDecoder`` classes.
"""
from .codes import Code, load_table, reference_tables  # noqa: F401
from ._lib import LdpcError, KINDS, PACKS  # noqa: F401
from .decoder import (Batch, Decoder, NativeCode, CGPUDecoder, CGPU_Decoder_MS_SIMD, CGPU_Decoder_OMS_SIMD,  # noqa: F401
                      CGPU_Decoder_NMS_SIMD, CGPU_Decoder_2NMS_SIMD, CGPU_Decoder_MS_SIMD_v2, PLUGINS,
                      select_code, selected_code)
