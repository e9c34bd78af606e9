#!/usr/bin/env bash
# Builds the reference's own GPU application (PeriodSearch period_search_BOINC,
# CUDA FP64) unchanged, against this project's BOINC stub, so that it can run
# standalone on a B200 as a second oracle and as the speed bar for the fit.
#
#   REF=<reference tree> oracle/refapp/build.sh
#
# Outputs (test infrastructure, never linked into the product):
#   oracle/_ref/refapp_sm100a   native sm_100a SASS
#   oracle/_ref/refapp_lto100   the reference Makefile's own sm_100 entry:
#                               compute_100 with code=[lto_100,sm_100]
#   oracle/_ref/refapp_b200shim the reference's host program on this
#                               project's engine (libps_b200.so must exist)
# Both use the reference Makefile's device flags (--use_fast_math,
# --maxrregcount=32, -rdc=true, --extra-device-vectorization, -O3).
#
# The one change: the reference caps MAX_N_FAC at 400 (constants.h), below
# the 512 facets of an nrows=8 object.  The sources are compiled from a
# temporary build copy in which that single constant reads 512; it only sizes
# static arrays.  The copy is deleted after the build, so no reference source
# stays in this tree.  The reference's own Makefile is not run.
set -euo pipefail
: "${REF:?set REF to the reference source tree}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$(cd "$HERE/.." && pwd)/_ref"
NVCC="${NVCC:-nvcc}"
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
mkdir -p "$OUT"

COMMON=(--forward-unknown-opts -mcmodel=medium -O3 -lineinfo --use_fast_math
        --extra-device-vectorization "--ptxas-options=-O3 --register-usage-level 0"
        --maxrregcount=32 -rdc=true)
HOSTFLAGS="-O3 -I$HERE/boinc_stub -I$CUDA_HOME/include"
HOST_C=(trifac areanorm sphfunc ellfit ludcmp lubksb covsrt memory dot_product)

build_variant() {
    local name="$1"; shift
    local gencode=("$@")
    local work="$OUT/.build_$name"
    rm -rf "$work"
    mkdir -p "$work"
    trap 'rm -rf "$work"' RETURN
    cp "$REF"/*.cu "$REF"/*.cuh "$REF"/*.h "$REF"/*.c "$REF"/*.cpp "$work"/
    sed -i 's/^#define MAX_N_FAC[[:space:]]\+400\b/#define MAX_N_FAC           512/' "$work/constants.h"
    grep -q '^#define MAX_N_FAC[[:space:]]\+512' "$work/constants.h"
    (
        cd "$work"
        for u in start_CUDA Start ComputeCapability; do
            "$NVCC" "${COMMON[@]}" "${gencode[@]}" --compiler-options="$HOSTFLAGS" -c "$u.cu" -o "$u.o" &
        done
        for c in "${HOST_C[@]}"; do
            g++ -O3 -mcmodel=medium -w -c -x c++ "$c.c" -o "$c.o" &
        done
        g++ $HOSTFLAGS -mcmodel=medium -w -c period_search_BOINC.cpp -o period_search_BOINC.o &
        g++ -O2 -I"$HERE/boinc_stub" -c "$HERE/boinc_stub.cpp" -o boinc_stub.o &
        wait
        for o in start_CUDA Start ComputeCapability period_search_BOINC boinc_stub "${HOST_C[@]}"; do
            test -s "$o.o"
        done
        "$NVCC" "${COMMON[@]}" "${gencode[@]}" -dlink -o pscuda.device-link.o \
            start_CUDA.o Start.o ComputeCapability.o
        g++ -o "$OUT/refapp_$name" period_search_BOINC.o start_CUDA.o Start.o ComputeCapability.o \
            pscuda.device-link.o boinc_stub.o "${HOST_C[@]/%/.o}" \
            -L"$CUDA_HOME/lib64" -lcudadevrt -lcudart_static -L"$CUDA_HOME/lib64/stubs" -lcuda \
            -lrt -pthread -ldl -lm
    )
    echo "built $OUT/refapp_$name"
}

# The reference's own host program (period_search_BOINC.cpp and its setup
# sources, unchanged) with start_CUDA.cu replaced by this project's binding
# ps_claude_opt_b200/host/start_b200.cpp, linked against libps_b200.so: the
# drop-in, built exactly as INTEGRATION.md tells a maintainer to.
build_shim() {
    local work="$OUT/.build_b200shim"
    local repo lib
    repo="$(cd "$HERE/../.." && pwd)"
    lib="$repo/ps_claude_opt_b200/_lib"
    test -f "$lib/libps_b200.so" || { echo "build libps_b200.so first"; return 1; }
    rm -rf "$work"
    mkdir -p "$work"
    trap 'rm -rf "$work"' RETURN
    cp "$REF"/*.h "$REF"/*.c "$REF"/*.cpp "$work"/
    sed -i 's/^#define MAX_N_FAC[[:space:]]\+400\b/#define MAX_N_FAC           512/' "$work/constants.h"
    (
        cd "$work"
        for c in "${HOST_C[@]}"; do
            g++ -O3 -mcmodel=medium -w -c -x c++ "$c.c" -o "$c.o" &
        done
        g++ $HOSTFLAGS -mcmodel=medium -w -c period_search_BOINC.cpp -o period_search_BOINC.o &
        g++ -O2 -I"$HERE/boinc_stub" -c "$HERE/boinc_stub.cpp" -o boinc_stub.o &
        g++ -O2 -std=c++17 -Wall -Wextra -I. -I"$HERE/boinc_stub" -I"$repo/include" \
            -c "$repo/ps_claude_opt_b200/host/start_b200.cpp" -o start_b200.o &
        wait
        for o in period_search_BOINC boinc_stub start_b200 "${HOST_C[@]}"; do
            test -s "$o.o"
        done
        g++ -o "$OUT/refapp_b200shim" period_search_BOINC.o start_b200.o boinc_stub.o "${HOST_C[@]/%/.o}" \
            -L"$lib" -lps_b200 -Wl,-rpath,"\$ORIGIN/../../ps_claude_opt_b200/_lib" \
            -L"$CUDA_HOME/lib64" -lcudart -lm -pthread
    )
    echo "built $OUT/refapp_b200shim"
}

build_variant sm100a -gencode arch=compute_100a,code=sm_100a &
build_variant lto100 "--generate-code=arch=compute_100,code=[lto_100,sm_100]" &
build_shim &
wait
test -x "$OUT/refapp_sm100a"
test -x "$OUT/refapp_lto100"
test -x "$OUT/refapp_b200shim"
