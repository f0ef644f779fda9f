#!/bin/sh
# Builds the reference's own tensor-core SP2 (PROGRESS src/sp2_tensorcore/src: the
# FP16 hi + lo cuBLAS driver prg_sp2_tensorcore) from its sources where they lie, into
# oracle/_ref/libprg_sp2_tc.so.  Test infrastructure: the GPU tests and bench.py load it
# as the prior art to check against and to race; nothing of it enters libsp2b.
#
# The sources are compiled unchanged, with the flag their C entry needs
# (SP2TCFortran: extern "C" prg_sp2_tensorcore) and their own #defines (DIAG_OFF: the
# spectral bounds h1 = -27.55, hN = 25.00 written in the source; NO_REFINEMENT: D is the
# final FP32 iterate).  cuBLAS and cuSOLVER come from the CUDA toolkit.
#
# Usage: oracle/build_ref.sh <path of the PROGRESS checkout>
set -e
REF="$1"
if [ -z "$REF" ] || [ ! -d "$REF/src/sp2_tensorcore/src" ]; then
  echo "usage: $0 <PROGRESS source tree>" >&2
  exit 2
fi
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
mkdir -p "$OUT"
SRC="$REF/src/sp2_tensorcore/src"
NVCC="${CUDA_HOME:-/usr/local/cuda}/bin/nvcc"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -shared -Xcompiler -fPIC \
  -DSP2TCFortran -I"$SRC" \
  "$SRC/prg_sp2_tensorcore.cu" "$SRC/tcore_hp_emulator.cu" "$SRC/linalg_tools.cu" \
  -o "$OUT/libprg_sp2_tc.so" -lcublas -lcusolver
echo "$OUT/libprg_sp2_tc.so"
