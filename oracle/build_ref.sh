#!/usr/bin/env bash
# Builds oracle/_ref/libcrp_ref.so from the reference's own sources, where they
# lie, plus the stand-in headers in oracle/ref_stubs and the harness in
# oracle/ref_harness.inc.  Test infrastructure only; nothing in
# the product links it.  Output goes to oracle/_ref/ only.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $CRP_REFERENCE, else /root/reference (where the
#   read-only reference checkout lives on the build machine).  The root used is
#   written to oracle/_ref/reference_root for the tests that read the
#   reference's own files.  Exits 0 without building when the tree is absent.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref="${1:-${CRP_REFERENCE:-/root/reference}}"
out="$here/_ref"
if [[ ! -f "$ref/src/bubble_CUDA.cu" ]]; then
  echo "build_ref: no reference tree at $ref; skipping"
  exit 0
fi
mkdir -p "$out/stubs"
echo "$ref" > "$out/reference_root"
# Forwarding headers: the reference's quoted includes resolve through these to
# its inc/ directory, while its <thrust/...> includes keep resolving to CUDA's.
for h in bubbles.h bubble_CUDA.h bubble_CUDA_kernel.cuh output_styles.h SphDataType.h; do
  echo "#include \"$ref/inc/$h\"" > "$out/stubs/$h"
done
cat > "$out/ref_main.cu" <<EOF
#include "$here/ref_prelude.h"
#include "$ref/src/bubble_CUDA.cu"
#include "$here/ref_harness.inc"
EOF
echo "#include \"$ref/src/output_styles.cpp\"" > "$out/ref_output.cu"
echo "#include \"$ref/src/SphDataType.cpp\"" > "$out/ref_sph.cpp"

NVCC="${NVCC:-nvcc}"
inc=(-I"$out/stubs" -I"$here/ref_stubs")
arch=(-gencode arch=compute_100a,code=sm_100a)
# save_ascii (src/output_styles.cpp:139-341) has no return statement; GCC 13
# turns the end of such a function into a trap even at -O0, so that unit is
# built with -fno-unreachable-traps.
"$NVCC" -std=c++17 "${arch[@]}" "${inc[@]}" -w -Xcompiler -fPIC -Xcompiler -O2 -c "$out/ref_main.cu" -o "$out/ref_main.o"
"$NVCC" -std=c++17 "${arch[@]}" "${inc[@]}" -w -Xcompiler -fPIC -Xcompiler -O0 -Xcompiler -fno-unreachable-traps -c "$out/ref_output.cu" -o "$out/ref_output.o"
g++ -std=c++17 -fPIC -O0 -w "${inc[@]}" -c "$out/ref_sph.cpp" -o "$out/ref_sph.o"
"$NVCC" -shared "${arch[@]}" -o "$out/libcrp_ref.so" "$out/ref_main.o" "$out/ref_output.o" "$out/ref_sph.o" -lpthread
echo "build_ref: built $out/libcrp_ref.so"
