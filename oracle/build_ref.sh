#!/usr/bin/env bash
# Builds the reference-side checkers into oracle/_ref/ straight from the
# reference's own source files (no use of its CMake build):
#
#   _ref/libref_host.so  host number theory (primes, NTT tables, RNS constants)
#                        of the vendored PhantomFHE, compiled by g++, behind
#                        the extern "C" face in ref_host_shim.cpp
#   _ref/ref_golden      the reference GPU evaluator (all PhantomFHE .cu files,
#                        the moai:: adapter ckks_evaluator_parallel.cu and the
#                        shared-a files FmtSwitch.cu, ShRotate.cu and
#                        SharedABatchOps.cu) for sm_100a, linked with the
#                        golden-vector and timing harness ref_golden.cu
#
# The outputs are test infrastructure.  Run where the reference tree exists;
# elsewhere the script does nothing.  Set SHMOAI_REF_GPU=0 to skip the
# (slow, ~minutes) GPU build.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
# the reference tree: $SHMOAI_REFERENCE, else a checkout named "reference" beside the repository
REF=${SHMOAI_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}
OUT=$HERE/_ref
PH=$REF/thirdparty/phantom-fhe
if [ ! -d "$PH" ]; then
    echo "build_ref: reference tree not found at $REF, nothing to build"
    exit 0
fi
mkdir -p "$OUT/obj"
CUDA_INC=/usr/local/cuda/include

if [ ! -f "$OUT/libref_host.so" ] || [ "$HERE/ref_host_shim.cpp" -nt "$OUT/libref_host.so" ]; then
    g++ -std=c++17 -O2 -fPIC -shared -I"$PH/include" -I"$PH/include/util" -I"$CUDA_INC" \
        -x c++ "$PH/src/util/ntt.cu" "$PH/src/util/numth.cu" "$PH/src/util/uintarith.cu" \
        "$PH/src/util/uintarithmod.cu" "$PH/src/util/uintarithsmallmod.cu" "$PH/src/util/globals.cu" \
        "$PH/src/util/rns.cu" "$PH/src/modulus.cu" \
        -x none "$HERE/ref_host_shim.cpp" -o "$OUT/libref_host.so"
    echo "build_ref: built $OUT/libref_host.so"
fi

if [ "${SHMOAI_REF_GPU:-1}" = "0" ]; then exit 0; fi
if [ -f "$OUT/ref_golden" ] && [ "$OUT/ref_golden" -nt "$HERE/ref_golden.cu" ]; then exit 0; fi

NVFLAGS=(-std=c++17 -O3 -rdc=true -Xcompiler -fPIC,-fopenmp --default-stream per-thread -DPHANTOM_USE_CUDA_PTX
         -gencode arch=compute_100a,code=sm_100a -I"$PH/include" -I"$REF/src/include/source"
         -I"$REF/src/include/source/bootstrapping" -w)
BOOT=$REF/src/include/source/bootstrapping
SRCS=("$PH"/src/*.cu "$PH"/src/ntt/*.cu "$PH"/src/util/*.cu "$REF/src/include/source/ckks_evaluator_parallel.cu"
      "$BOOT/FmtSwitch.cu" "$BOOT/ShRotate.cu" "$BOOT/SharedABatchOps.cu")
pids=()
for src in "${SRCS[@]}"; do
    rel=${src#"$REF"/}
    obj="$OUT/obj/$(echo "$rel" | tr '/' '_').o"
    if [ ! -f "$obj" ] || [ "$src" -nt "$obj" ]; then
        nvcc "${NVFLAGS[@]}" -c "$src" -o "$obj" &
        pids+=($!)
        if [ "${#pids[@]}" -ge "$(nproc)" ]; then wait "${pids[0]}"; pids=("${pids[@]:1}"); fi
    fi
done
for p in "${pids[@]}"; do wait "$p"; done
nvcc "${NVFLAGS[@]}" -c "$HERE/ref_golden.cu" -o "$OUT/obj/ref_golden.o"
nvcc -gencode arch=compute_100a,code=sm_100a -rdc=true -Xcompiler -fopenmp "$OUT"/obj/*.o -o "$OUT/ref_golden"
echo "build_ref: built $OUT/ref_golden"
