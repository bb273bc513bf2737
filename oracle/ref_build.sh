#!/bin/bash
# Builds the reference's own CUDA solver (cuda_simulation.cu + cuda_tool.cu, unmodified,
# compiled where they lie under /root/reference) together with this directory's harness
# into oracle/_ref/libsnowref.so, for sm_100a.  Test infrastructure: the reference run is
# the pin of the CPU oracle.  Where the reference sources are absent the script skips,
# and the library built earlier is used.  The reference project is a Visual Studio build with OpenGL headers
# on its include path; two type-only stand-ins written here (GL/gl.h with the GL scalar
# typedefs, and nothing else) let nvcc parse those headers.  The build mirrors the
# reference's project settings: fast math and relocatable device code.
set -e
REF=${REF:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
[ -d "$REF" ] || { echo "reference sources not present; skipping"; exit 0; }
mkdir -p "$OUT/stub/GL"
cat > "$OUT/stub/GL/gl.h" <<'H'
#ifndef SNOWREF_STUB_GL_H
#define SNOWREF_STUB_GL_H
typedef unsigned int GLenum;
typedef unsigned int GLuint;
#endif
H
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
COMMON=(-std=c++17 -gencode arch=compute_100a,code=sm_100a -O2 -rdc=true -DGLEW_NO_GLU -D__forceinline=inline
        -Xcompiler -fPIC -shared -I"$OUT/stub" -I"$REF" -I"$REF/include" -I"$REF/include/cuda_common"
        "$REF/cuda_simulation.cu" "$REF/cuda_tool.cu" "$HERE/ref_harness.cu")
# 1. as the reference project builds it (FastMath, SnowSimulation.vcxproj:151-154)
"$NVCC" "${COMMON[@]}" -use_fast_math -o "$OUT/libsnowref.so"
# 2. the same sources with IEEE arithmetic and no contraction: every float operation is
#    then the one the CPU oracle performs, so deterministic stages compare bit for bit
"$NVCC" "${COMMON[@]}" -fmad=false -prec-div=true -prec-sqrt=true -ftz=false -o "$OUT/libsnowref_ieee.so"
echo "built $OUT/libsnowref.so $OUT/libsnowref_ieee.so"
