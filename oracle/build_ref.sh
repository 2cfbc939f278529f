#!/bin/bash
# Builds the reference's own GPU kernels, unmodified, from the reference
# sources where they lie, into oracle/_ref/libref_<code>.so (git-ignored).
# Test infrastructure only: oracle/make_golden.py runs these on a B200 to pin
# the CPU oracle.  The reference selects its H matrix at compile time through
# src/matrix/code.h (`#define CODE 4000`), so each code gets a shadow tree
# oracle/_ref/src_<code>/ made of symbolic links into the reference plus a
# generated matrix/code.h; no reference file is copied or edited.
#
# usage: oracle/build_ref.sh [--if-present] [code ...]
#   (default codes: those of tests/golden/make_golden.py; the reference's src directory
#   is $REF_SRC, by default where this machine keeps the reference tree; --if-present
#   exits 0 quietly when it is absent, as on machines that only run the built files)
set -euo pipefail
IF_PRESENT=0
if [ "${1:-}" = "--if-present" ]; then IF_PRESENT=1; shift; fi
REF=${REF_SRC:-/root/reference/src}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
NVCC=${NVCC:-nvcc}
if [ ! -d "$REF" ]; then
    [ $IF_PRESENT = 1 ] && exit 0
    echo "reference sources not found at $REF (set REF_SRC)" >&2
    exit 1
fi
mkdir -p "$OUT"

dir_of() {
    case $1 in
        576) echo 576x288 ;; 816) echo 816x408 ;; 1024) echo 1024x518 ;;
        1200) echo 1200x600 ;; 1944) echo 1944x972 ;; 2048) echo 2048x384 ;;
        2304) echo 2304x1152 ;; 4000) echo 4000x2000 ;; 4896) echo 4896x2448 ;;
        8000) echo 8000x4000 ;; 9972) echo 9972x4986 ;; 20000) echo 20000x10000 ;;
        64800) echo 64800x32400 ;; 64801) echo 64800x21600 ;;
        *) echo "unknown code $1" >&2; return 1 ;;
    esac
}

CODES=("$@")
[ ${#CODES[@]} -gt 0 ] || CODES=(4000 576 1944 2304 816)

for CODE in "${CODES[@]}"; do
    D=$(dir_of "$CODE")
    S=$OUT/src_$CODE
    mkdir -p "$S/matrix"
    # Real directories holding one symbolic link per file (cp -rs), never a link to a
    # whole directory: the kernels include "../../matrix/constantes_gpu.h", and through
    # a directory link that path resolves inside the reference tree, whose own
    # matrix/code.h (CODE 4000) would then select the table instead of this tree's.
    for d in decoder_ms decoder_oms decoder_nms decoder_2nms decoder_oms_v2 transpose; do
        rm -rf "$S/$d"
        cp -rs "$REF/$d" "$S/$d"
    done
    ln -sf "$REF/matrix/constantes_gpu.h" "$S/matrix/constantes_gpu.h"
    ln -sf "$REF/matrix/constantes_decoder.cpp" "$S/matrix/constantes_decoder.cpp"
    ln -sfn "$REF/matrix/$D" "$S/matrix/$D"
    echo "#define CODE $CODE" > "$S/matrix/code.h"
    # every unit must see this tree's table: the kernels' array bounds carry _N
    WANT=${D%%x*}
    for u in decoder_ms/cuda/CUDA_MS_SIMD.cu decoder_oms/cuda/CUDA_OMS_SIMD.cu decoder_nms/cuda/CUDA_NMS_SIMD.cu \
             decoder_2nms/cuda/CUDA_2NMS_SIMD.cu decoder_oms_v2/cuda/CUDA_OMS_SIMD_v2.cu; do
        GOT=$($NVCC -E -w -I"$S" "$S/$u" 2>/dev/null | grep -o 'var_nodes\[[0-9]*\]' | head -1 | tr -dc 0-9)
        if [ "$GOT" != "$WANT" ]; then
            echo "$u sees _N=$GOT, expected $WANT for $D: the shadow tree leaks another table" >&2
            exit 1
        fi
    done
    LIB=$OUT/libref_$CODE.so
    if [ -f "$LIB" ] && [ "$LIB" -nt "$HERE/ref_harness.cu" ] && [ "$LIB" -nt "$0" ]; then
        echo "up to date: $LIB"
        continue
    fi
    echo "building $LIB"
    $NVCC -O3 -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fPIC \
        -w -I"$S" -o "$LIB" \
        "$HERE/ref_harness.cu" \
        "$S/decoder_ms/cuda/CUDA_MS_SIMD.cu" \
        "$S/decoder_oms/cuda/CUDA_OMS_SIMD.cu" \
        "$S/decoder_nms/cuda/CUDA_NMS_SIMD.cu" \
        "$S/decoder_2nms/cuda/CUDA_2NMS_SIMD.cu" \
        "$S/decoder_oms_v2/cuda/CUDA_OMS_SIMD_v2.cu" \
        "$S/transpose/GPU_Transpose_uint8.cu" \
        "$S/matrix/constantes_decoder.cpp"
done
