#!/usr/bin/env bash
# Test build of the six MEX gateways (top_gpu_on_matlab_b200/mex/*.cpp)
# against the MEX stand-in in oracle/mexshim, one shared library per gateway
# (tests/_mexgw/lib<Name>.so, git-ignored), linked to libtopgpu.so.  A MATLAB
# installation builds the same sources with mexcuda instead.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/.." && pwd)
SRC="$ROOT/top_gpu_on_matlab_b200/mex"
SHIM="$ROOT/oracle/mexshim"
OUT="$HERE/_mexgw"
CXX=${CXX:-g++}
mkdir -p "$OUT"
for name in Gathering_inplace Scattering_inplace scatter_accum3_inplace \
            assembleKs_level2_inplace assembleKs_higherLevel_inplace assembleKs_level2_superEle_inplace; do
    lib="$OUT/lib$name.so"
    if [ -f "$lib" ] && [ "$lib" -nt "$SRC/$name.cpp" ] && [ "$lib" -nt "$SRC/topgpu_mex.h" ] && \
       [ "$lib" -nt "$SHIM/mexshim.cpp" ]; then continue; fi
    "$CXX" -O2 -std=c++17 -fPIC -shared -Wall -Werror -I"$SHIM" -I"$ROOT/include" -o "$lib" \
        "$SRC/$name.cpp" "$SHIM/mexshim.cpp" -L"$ROOT/top_gpu_on_matlab_b200" -ltopgpu \
        -Wl,-rpath,"\$ORIGIN/../../top_gpu_on_matlab_b200"
done
