#!/usr/bin/env bash
# Links the reference's own FWI / RTM executables against the drop-in shim
# instead of the reference's GPU objects, to show that a caller of the
# reference needs nothing else: its objects compile from the reference tree
# with the reference's own headers (wave3d.h, wave.h) and every entry they
# call resolves in libvti_wave.so (+ libvti_b200.so). Nothing is run.
#   fwi3d-lbfgsc     lib/vti-fwi-3d/gpu/fwi3d-lbfgsc.cu (3D L-BFGS FWI, objFuncGradientVEpsDel)
#   rtm3d-cij-shot   lib/vti-fwi-3d/gpu/rtm3d-cij-shot.cu (rtmCij3d_f)
#   fwi-lbfgs-c-param lib/vti-fwi-2d/fwi-lbfgs-c-param.cu with its host glue
#                    objFuncGradient.cu (the 2D parameterisations over objFuncGradient_f)
# Host-only helpers come from the reference tree as its Makefiles list them
# (chapter2/Makefile:85, chapter5/Makefile:152): myio, check, conversions,
# init, lbfgs_c, la, lsearch. Outputs go to oracle/_ref/callers/ only.
set -euo pipefail
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
PKG="$HERE/../thesis-source-code_b200/vtib200"
OUT="$HERE/_ref/callers"
if [ ! -d "$REF/lib" ]; then
  echo "reference tree not found at $REF; skipping" >&2
  exit 0
fi
if [ ! -f "$PKG/libvti_wave.so" ]; then
  echo "libvti_wave.so not built" >&2
  exit 1
fi
mkdir -p "$OUT"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
L3="$REF/lib/vti-fwi-3d/gpu"
L2="$REF/lib/vti-fwi-2d"
IO="$REF/lib/io"
LB="$REF/lib/lbfgs"
LS="$REF/lib/LinearSolver"
INC="-I$L3 -I$L2 -I$IO -I$LB -I$LS"
cxx() {  # source object
  case "$1" in
    *.cu) "$NVCC" -O1 -std=c++14 -gencode arch=compute_100a,code=sm_100a -x cu -Xcompiler -fopenmp \
            -w $INC -c "$1" -o "$2" ;;
    *) g++ -O1 -std=c++14 -fopenmp -w $INC -c "$1" -o "$2" ;;
  esac
}
for f in "$IO/myio.cpp" "$L2/check.cpp" "$L2/conversions.cpp" "$L2/init.cpp" \
         "$LB/lbfgs_c.cpp" "$LB/la.cpp" "$LB/lsearch.cpp" \
         "$L3/fwi3d-lbfgsc.cu" "$L3/rtm3d-cij-shot.cu" "$L2/fwi-lbfgs-c-param.cu" \
         "$L2/objFuncGradient.cu"; do
  cxx "$f" "$OUT/$(basename "$f").o"
done
# the .cu objects carry the CUDA runtime's registration calls (no kernels)
CUDART=$(dirname "$(ldd "$PKG/libvti_b200.so" | awk '/libcudart/ {print $3}')")
LINK=(-L"$PKG" -lvti_wave -lvti_b200 -L"$CUDART" -l:libcudart.so.12 -Wl,-rpath,"$PKG"
      -Wl,-rpath,"$CUDART" -fopenmp -lpthread)
H="$OUT/myio.cpp.o $OUT/check.cpp.o $OUT/conversions.cpp.o"
LBF="$OUT/lbfgs_c.cpp.o $OUT/la.cpp.o $OUT/lsearch.cpp.o"
g++ -o "$OUT/fwi3d-lbfgsc" "$OUT/fwi3d-lbfgsc.cu.o" $H $LBF "${LINK[@]}"
g++ -o "$OUT/rtm3d-cij-shot" "$OUT/rtm3d-cij-shot.cu.o" $H "${LINK[@]}"
g++ -o "$OUT/fwi-lbfgs-c-param" "$OUT/fwi-lbfgs-c-param.cu.o" "$OUT/objFuncGradient.cu.o" \
  "$OUT/init.cpp.o" $H $LBF "${LINK[@]}"
echo "linked $OUT/fwi3d-lbfgsc $OUT/rtm3d-cij-shot $OUT/fwi-lbfgs-c-param"
