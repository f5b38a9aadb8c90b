#!/usr/bin/env bash
# Compile the reference's six CUDA MEX kernels, unmodified and in place, for
# sm_100a against the test-only MEX stand-in (oracle/mexshim).  Output:
# oracle/_ref/lib<Name>.so (git-ignored; travels with the repository to the
# GPU box).  Usage: oracle/ref_build.sh /path/to/TOP_GPU_on_matlab
set -euo pipefail
REF=${1:?usage: ref_build.sh <reference checkout>}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
mkdir -p "$OUT"
for name in Gathering_inplace Scattering_inplace scatter_accum3_inplace \
            assembleKs_level2_inplace assembleKs_higherLevel_inplace assembleKs_level2_superEle_inplace; do
    src="$REF/$name.cu"
    lib="$OUT/lib$name.so"
    if [ -f "$lib" ] && [ "$lib" -nt "$src" ] && [ "$lib" -nt "$HERE/mexshim/mexshim.cpp" ]; then continue; fi
    "$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Xcompiler -fPIC -shared \
        -I"$HERE/mexshim" -o "$lib" "$src" "$HERE/mexshim/mexshim.cpp"
done
