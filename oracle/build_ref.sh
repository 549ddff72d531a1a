#!/usr/bin/env bash
# Builds the reference's own sources and tests where they lie into
# oracle/_ref/.  The read-only reference tree is $REF; by default the
# directory named "reference" beside this repository's root.  Checker only:
# nothing in the product links these.
#
#   _ref/ref_<w>/      the reference's compilable code with its own tests:
#                      host CRT + limits (g++), and the stage kernels
#                      zero_pad / crt_gpu / carry_prop (nvcc, sm_100a)
#   _ref/compat_<w>/   the reference's tests compiled unmodified against
#                      this repository's compatible headers (include/) and
#                      linked with libbirdwing + the compat sources
#   _ref/libref_stage_hybrid.so  the reference's crt_gpu.cu + carry_prop.cu
#                      (LIMB_BITS=64) behind oracle/ref_stage_shim.cu
#
# <w> is 32, hybrid (LIMB_BITS=64) or native (LIMB_BITS=64 NATIVE_HOST_LIMBS).
# GPU-NTT (the reference's NTT library) is absent, so src/gpu_ntt.cu,
# src/host_multiply.cpp and tests/test_pipeline_crt.cpp are not buildable.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT="$(dirname "$HERE")"
REF="${REF:-$(dirname "$ROOT")/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-nvcc}"
ARCH="-gencode arch=compute_100a,code=sm_100a"
GMPLIB="$(ls /usr/lib/x86_64-linux-gnu/libgmp.so.10 2>/dev/null || echo -lgmp)"
[ -d "$REF/src" ] || { echo "reference tree not found at $REF"; exit 0; }
mkdir -p "$OUT"

declare -A WFLAGS=( [32]="-DLIMB_BITS=32" [hybrid]="-DLIMB_BITS=64"
                    [native]="-DLIMB_BITS=64 -DNATIVE_HOST_LIMBS" )
COMPAT="$ROOT/birdwing_b200/csrc/compat"
LIB="$ROOT/birdwing_b200"

for w in 32 hybrid native; do
  F="${WFLAGS[$w]}"
  # ---- the reference itself
  R="$OUT/ref_$w"; mkdir -p "$R"
  g++ -std=c++17 -O2 $F -I"$REF/include" "$REF/tests/test_crt.cpp" "$REF/src/crt.cpp" \
      "$REF/src/crt_utils.cpp" -o "$R/test_crt"
  g++ -std=c++17 -O2 $F -I"$REF/include" "$REF/tests/test_ntt_limits.cpp" \
      "$REF/src/ntt_limits.cpp" -o "$R/test_ntt_limits"
  $NVCC -std=c++17 -O2 $ARCH $F -I"$REF/include" "$REF/tests/test_zero_pad.cu" \
      "$REF/src/zero_pad.cu" -o "$R/test_zero_pad"
  $NVCC -std=c++17 -O2 $ARCH $F -I"$REF/include" "$REF/tests/test_crt_gpu.cu" \
      "$REF/src/crt_gpu.cu" "$REF/src/crt_utils.cpp" -o "$R/test_crt_gpu"
  $NVCC -std=c++17 -O2 $ARCH $F -I"$REF/include" "$REF/tests/test_carry_prop.cu" \
      "$REF/src/carry_prop.cu" -o "$R/test_carry_prop"

  # ---- the reference's tests against this repository's headers + library
  C="$OUT/compat_$w"; mkdir -p "$C/obj"
  INC="-I$ROOT/include -I$HERE/gmp_shim"
  LINK="-L$LIB -lbirdwing -Xlinker -rpath -Xlinker $LIB -Xlinker $GMPLIB"
  OBJS=""
  for s in gpu_ntt.cu host_multiply.cpp crt.cpp ntt_limits.cpp crt_gpu.cu carry_prop.cu zero_pad.cu; do
    $NVCC -std=c++17 -O2 $ARCH $F $INC -c "$COMPAT/$s" -o "$C/obj/${s%.*}.o"
    OBJS="$OBJS $C/obj/${s%.*}.o"
  done
  for t in test_zero_pad.cu test_crt_gpu.cu test_carry_prop.cu test_crt.cpp \
           test_gpu_ntt_smoke.cu test_full_multiply.cpp test_pointwise_mul.cu; do
    $NVCC -std=c++17 -O2 $ARCH $F $INC "$REF/tests/$t" $OBJS $LINK -o "$C/${t%.*}"
  done
  g++ -std=c++17 -O2 $F -I"$ROOT/include" "$REF/tests/test_ntt_limits.cpp" \
      "$COMPAT/ntt_limits.cpp" -o "$C/test_ntt_limits"
done

# ---- the reference's stage kernels behind a C shim, for parity tests
$NVCC -std=c++17 -O2 $ARCH -DLIMB_BITS=64 -Xcompiler -fPIC -shared -I"$REF/include" \
    "$HERE/ref_stage_shim.cu" "$REF/src/crt_gpu.cu" "$REF/src/carry_prop.cu" \
    "$REF/src/crt_utils.cpp" -o "$OUT/libref_stage_hybrid.so"
echo "reference builds in $OUT"
