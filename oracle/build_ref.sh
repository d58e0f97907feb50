#!/bin/bash
# Test infrastructure: compiles the reference's own CUDA update (read in place from the
# reference checkout, never copied) together with oracle/ref_harness.cu into
# oracle/_ref/libref_k3dom.so and oracle/_ref/libref_dsphdmib.so.
#  - oracle/ref_shim provides glm/vec3.hpp (GLM is not installed) and a curand_kernel.h that
#    serves the library's Philox draws;
#  - -include thrust/sort.h supplies the include commented out at src/common/dom.cu:16;
#  - -fmad=false makes every float operation round once, as the library's _rn code does;
#  - -DNDEBUG compiles out the reference's device asserts (no trap on a shared GPU).
set -euo pipefail
REF=${K3DOM_REFERENCE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -d "$REF/src" ]; then
    echo "reference checkout not found at $REF (set K3DOM_REFERENCE)" >&2
    if [ "${1:-}" = "--if-present" ]; then exit 0; fi
    exit 1
fi
NVCC=${NVCC:-nvcc}
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -fmad=false --expt-extended-lambda
       -Xcompiler -fPIC -DNDEBUG -I"$HERE/ref_shim" -I"$REF/include" -include thrust/sort.h -shared -cudart static)
COMMON=("$REF"/src/common/dom.cu "$REF"/src/common/kernel/*.cu)
"$NVCC" "${FLAGS[@]}" -o "$OUT/libref_k3dom.so" "${COMMON[@]}" "$REF"/src/k3dom/dom.cu \
    "$REF"/src/k3dom/kernel/mass_update.cu "$HERE/ref_harness.cu" &
P1=$!
"$NVCC" "${FLAGS[@]}" -DREF_DS -o "$OUT/libref_dsphdmib.so" "${COMMON[@]}" "$REF"/src/dsphdmib/dom.cu \
    "$REF"/src/dsphdmib/kernel/*.cu "$HERE/ref_harness.cu" &
P2=$!
wait $P1
wait $P2
echo "built $OUT/libref_k3dom.so $OUT/libref_dsphdmib.so"
