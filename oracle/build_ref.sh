#!/usr/bin/env bash
# Compiles the reference's own VTI GPU path from its sources where they lie
# in the reference tree ($REF, read-only; nothing is copied) into oracle/_ref/:
#   ref3d : lib/vti-fwi-3d/gpu 3D modeling, gradient, RTM (+ the host glue they link)
#   ref2d : lib/vti-fwi-2d synthetic_f / modeling_f / objFuncGradient_f / GNhessian_f / rtm_f
#   ref_randb : lib/random-boundary's generator (CPU)
# linked with the small harnesses oracle/ref_driver{3d,2d}.cpp. Outputs go only
# to oracle/_ref/ (git-ignored). The binaries run on a GPU host to produce the
# golden fixtures under tests/golden/ (tests/golden/make_golden.py).
# The reference targets sm_70; it is rebuilt unmodified for sm_100a.
set -euo pipefail
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -d "$REF/lib" ]; then
  echo "reference tree not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT/obj3d" "$OUT/obj2d"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
L3="$REF/lib/vti-fwi-3d/gpu"
L2="$REF/lib/vti-fwi-2d"
IO="$REF/lib/io"
INC="-I$L3 -I$L2 -I$IO"
FLAGS="-O3 -std=c++14 $ARCH -Xcompiler -fopenmp -w"

build_objs() {  # dir outdir files...
  local src=$1 od=$2; shift 2
  for f in "$@"; do
    local o="$od/$(basename "$f").o"
    if [ ! -f "$o" ] || [ "$src/$f" -nt "$o" ]; then
      "$NVCC" $FLAGS $INC -x cu -c "$src/$f" -o "$o"
    fi
  done
}

# 3D path (objFuncGradient3d_f.cu, modelData3d_f.cu and what they link)
build_objs "$L3" "$OUT/obj3d" objFuncGradient3d_f.cu modelData3d_f.cu rtm3d_f.cu kernel3d.cu \
  injectRecord3d.cu abc3d.cu memcpy3d.cu boundary.cpp agc.cpp cluster.cpp
build_objs "$L2" "$OUT/obj3d" conversions.cpp check.cpp
build_objs "$IO" "$OUT/obj3d" myio.cpp
"$NVCC" $FLAGS -x cu -c "$HERE/ref_driver3d.cpp" -o "$OUT/obj3d/ref_driver3d.o"
"$NVCC" $ARCH -Xcompiler -fopenmp -o "$OUT/ref3d" "$OUT"/obj3d/*.o -lpthread

# 2D path (synthetic_f.cu, modeling_f.cu)
build_objs "$L2" "$OUT/obj2d" kernels.cu synthetic_f.cu modeling_f.cu objFuncGradient_f.cu \
  hessian_f.cu rtm_f.cu odcig_f.cu check.cpp conversions.cpp
build_objs "$IO" "$OUT/obj2d" myio.cpp
"$NVCC" $FLAGS -x cu -c "$HERE/ref_driver2d.cpp" -o "$OUT/obj2d/ref_driver2d.o"
"$NVCC" $ARCH -Xcompiler -fopenmp -o "$OUT/ref2d" "$OUT"/obj2d/*.o
# random-boundary generator (host code, lib/random-boundary/randomBound.h)
g++ -O2 -std=c++14 -w -I"$REF/lib/random-boundary" "$HERE/ref_randb.cpp" -o "$OUT/ref_randb"
echo "built $OUT/ref3d $OUT/ref2d $OUT/ref_randb"
