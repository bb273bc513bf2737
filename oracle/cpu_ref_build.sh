#!/bin/bash
# Builds the reference's CPU neighbour search and constraint solver (NeighborSearch.cpp,
# ConstraintSolver.cpp, Constraints.cpp and the Particle/Collider files they link against,
# unmodified, compiled where they lie under /root/reference) with this directory's
# cpu_ref_harness.cpp into oracle/_ref/libsnowcpuref.so.  Measurement infrastructure: the
# library times the reference's own CPU code for the reported CPU baselines.  Where the
# reference sources are absent the script skips, and the library built earlier is used.
# Shims, as the reference's Visual Studio project has on its include path: the GL scalar
# typedefs (type names only) for the OpenGL headers, `std::floorf` (NeighborSearch.cpp
# calls it; libstdc++ only declares ::floorf) and MSVC's __forceinline.
set -e
REF=${REF:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
[ -d "$REF" ] || { echo "reference sources not present; skipping"; exit 0; }
mkdir -p "$OUT/stub/GL" "$OUT/cpu_obj"
cat > "$OUT/stub/GL/gl.h" <<'H'
#ifndef SNOWREF_STUB_GL_H
#define SNOWREF_STUB_GL_H
typedef unsigned int GLenum;
typedef unsigned int GLuint;
#endif
H
cat > "$OUT/stub/floorf_std.h" <<'H'
#pragma once
#include <cmath>
namespace std { using ::floorf; }
H
CUDA=${CUDA_HOME:-/usr/local/cuda}
FLAGS=(-std=c++17 -O2 -fPIC -fopenmp -w -include "$OUT/stub/floorf_std.h" -DGLEW_NO_GLU -D__forceinline=inline
       -I"$OUT/stub" -I"$REF" -I"$REF/include" -I"$REF/include/cuda_common" -I"$CUDA/include")
OBJS=()
for f in NeighborSearch ConstraintSolver Constraints Particle Collider CollisionDetection; do
    g++ "${FLAGS[@]}" -c "$REF/$f.cpp" -o "$OUT/cpu_obj/$f.o"
    OBJS+=("$OUT/cpu_obj/$f.o")
done
g++ "${FLAGS[@]}" -c "$HERE/cpu_ref_harness.cpp" -o "$OUT/cpu_obj/harness.o"
g++ -shared -fopenmp -Wl,--no-undefined -o "$OUT/libsnowcpuref.so" "$OUT/cpu_obj/harness.o" "${OBJS[@]}" \
    -L"$CUDA/lib64" -Wl,-rpath,"$CUDA/lib64" -lcudart
echo "built $OUT/libsnowcpuref.so"
