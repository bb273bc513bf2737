#!/bin/bash
# Checks the C++ shim snowsimulation_b200/shim/cuda_simulation_b200.cpp, which gives
# libsnowb200 the reference's cuda_simulation.cuh signatures, against the reference
# itself: the shim is compiled with the reference's own headers where they lie under
# /root/reference (its static_asserts compare the reference's struct sizes with the C ABI's)
# and linked, with no undefined symbol left, against libsnowb200.so and the reference's
# Particle/Collider sources (ParticleSet::setSize and its constructors); then
# shim_caller.cpp, which calls every entry point through the reference's declarations, is
# linked against it with no undefined symbol left; last, the C++ host driver
# snowsimulation_b200/shim/snow_host.cpp is built on the same objects.  Outputs go to
# oracle/_ref/shim/ only.  Where the reference sources are absent the script skips.
# Shims, as in cpu_ref_build.sh: GL scalar typedefs, std::floorf, MSVC's __forceinline.
set -e
REF=${REF:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(dirname "$HERE")"
OUT="$HERE/_ref/shim"
[ -d "$REF" ] || { echo "reference sources not present; skipping"; exit 0; }
[ -f "$ROOT/snowsimulation_b200/libsnowb200.so" ] || { echo "libsnowb200.so not built"; exit 1; }
mkdir -p "$OUT/stub/GL"
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
FLAGS=(-std=c++17 -O2 -fPIC -w -include "$OUT/stub/floorf_std.h" -DGLEW_NO_GLU -D__forceinline=inline
       -I"$OUT/stub" -I"$REF" -I"$REF/include" -I"$REF/include/cuda_common" -I"$CUDA/include" -I"$ROOT/include")
OBJS=()
for f in Particle Collider CollisionDetection; do
    g++ "${FLAGS[@]}" -c "$REF/$f.cpp" -o "$OUT/$f.o"
    OBJS+=("$OUT/$f.o")
done
g++ "${FLAGS[@]}" -c "$ROOT/snowsimulation_b200/shim/cuda_simulation_b200.cpp" -o "$OUT/shim.o"
g++ -shared -Wl,--no-undefined -o "$OUT/libshimcheck.so" "$OUT/shim.o" "${OBJS[@]}" \
    -L"$ROOT/snowsimulation_b200" -lsnowb200 -L"$CUDA/lib64" -lcudart
# every entry point, called through the reference's declarations, resolves in the shim
g++ "${FLAGS[@]}" -c "$HERE/shim_caller.cpp" -o "$OUT/caller.o"
g++ -shared -Wl,--no-undefined -o "$OUT/libshimcaller.so" "$OUT/caller.o" -L"$OUT" -lshimcheck \
    -L"$ROOT/snowsimulation_b200" -lsnowb200 -L"$CUDA/lib64" -lcudart
# the C++ host driver (snowsimulation_b200/shim/snow_host.cpp): the reference's host call
# sequence on the reference's types, linked with the shim in place of cuda_simulation.cu
g++ "${FLAGS[@]}" -c "$ROOT/snowsimulation_b200/shim/snow_host.cpp" -o "$OUT/snow_host.o"
g++ -o "$OUT/snow_host" "$OUT/snow_host.o" "$OUT/shim.o" "${OBJS[@]}" \
    -L"$ROOT/snowsimulation_b200" -lsnowb200 -L"$CUDA/lib64" -lcudart \
    -Wl,-rpath,'$ORIGIN/../../../snowsimulation_b200' -Wl,-rpath,"$CUDA/lib64"
echo "shim ok: $OUT/libshimcheck.so $OUT/snow_host"
