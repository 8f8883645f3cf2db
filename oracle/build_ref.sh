#!/usr/bin/env bash
# Build recipe for the checker's reference binaries (TEST INFRASTRUCTURE ONLY).
#
# Compiles the reference's own sources where they lie (the tree named by the FDK_REFERENCE
# environment variable) through the small extern "C" harnesses in this folder, and
# writes every output under oracle/_ref/ (git-ignored; it travels to the GPU box
# with the rest of the tree).  Nothing from the reference tree is copied into the
# repository.  The reference's own build system (VisualGDB makefiles) is not used.
#
# Two build-time adjustments:
#  1. common/type.h:3144 needs the `template` disambiguator under g++ (MSVC accepts
#     `x.FilterX<D>(...)` on a dependent expression).  A sed-fixed copy is generated
#     into oracle/_ref/gen/ and force-included first; its include guard (__Type_H)
#     turns every later `#include "../common/type.h"` of the original into a no-op.
#  2. CUDA 12 removed texture/surface references; ref_texture_shim.h declares
#     stand-ins for the binding helpers the tested kernels never call.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${FDK_REFERENCE:-}"
OUT="$HERE/_ref"
if [ -z "$REF" ] || [ ! -f "$REF/common/type.h" ]; then
    echo "build_ref: FDK_REFERENCE does not name a reference tree ('$REF'); skipping" >&2
    exit 0
fi
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
mkdir -p "$OUT/gen"
sed 's/FilterZ<D>(kernel)\.FilterX<D>(kernel)\.FilterY<D>(kernel)/FilterZ<D>(kernel).template FilterX<D>(kernel).template FilterY<D>(kernel)/' \
    "$REF/common/type.h" > "$OUT/gen/type_fixed.h"
grep -q 'template FilterX<D>' "$OUT/gen/type_fixed.h"

# CPU: Parameter/filter/cos table/matrices, Bourke row filter, 3dct CPU FDK.
# x86-64-v3 (AVX2+FMA) so the library runs on the GPU box's host CPU too.
g++ -std=gnu++11 -O3 -march=x86-64-v3 -fopenmp -fPIC -shared -w \
    -include "$OUT/gen/type_fixed.h" -I"$REF" \
    "$HERE/ref_cpu_harness.cpp" -o "$OUT/libref_cpu.so"

# GPU: cudaFdkBP via BackProjectionFDK, and the cuFFT filter plugin, for sm_100a.
NVFLAGS=(-std=c++14 -O3 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC,-fopenmp -shared -w
         -include "$HERE/ref_texture_shim.h" -include "$OUT/gen/type_fixed.h" -I"$REF"
         -Xlinker -rpath,/usr/local/cuda/lib64)
"$NVCC" "${NVFLAGS[@]}" "$HERE/ref_gpu_harness.cu" -o "$OUT/libref_gpu_bp.so"
"$NVCC" "${NVFLAGS[@]}" "$HERE/ref_gpu_filter_harness.cu" -lcufft -o "$OUT/libref_gpu_filter.so"
echo "build_ref: wrote $OUT"
