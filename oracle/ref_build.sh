#!/usr/bin/env bash
# Compiles the reference's own CUDA forward and gradient routines from their
# sources under the mounted reference tree into oracle/_ref/ (test
# infrastructure: parity against the reference binary on a GPU box).
#   libfkref_{fwd,grad}_dx0p035.so  the sources as they are (h = 0.035)
#   libfkref_{fwd,grad}_dx0p025.so  the parameter include switched to a
#       generated copy of the header with h = 0.025, the way the reference
#       selects parameter sets (sed of the include, fk_forward_Et_mono_PARAMETERS.cu:13-20)
#
# Where the reference tree is: the first argument, else FKADJ_REFERENCE_DIR,
# else the mount point of this build's container.  The chosen directory is
# recorded in oracle/_ref/source_dir for the tests that read the reference's
# data files.  With FKADJ_REF_OPTIONAL=1 a missing tree is not an error (the
# build then simply has no reference binary).
set -euo pipefail
REF=${1:-${FKADJ_REFERENCE_DIR:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
SRC=$REF/src/cuda
if [ ! -d "$SRC" ]; then
  if [ "${FKADJ_REF_OPTIONAL:-0}" = 1 ]; then echo "reference sources not found at $SRC; oracle/_ref not built"; exit 0; fi
  echo "reference sources not found at $SRC" >&2; exit 1
fi
mkdir -p "$OUT/src"
printf '%s\n' "$REF" > "$OUT/source_dir"
NVCC=${NVCC:-nvcc}
FLAGS="-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Xcompiler -fPIC -shared --cudart static -ccbin g++ -w"
build() {  # $1 tag  $2 cu-file  $3 define  $4 include-dir-for-cu
  "$NVCC" $FLAGS -D$3 -I"$HERE/ref_shim" -I"$4" -o "$OUT/libfkref_$1.so" "$2" "$HERE/ref_shim/ref_capi.cpp"
}
stamp=$OUT/.built
if [ -f "$stamp" ] && [ "$stamp" -nt "$HERE/ref_build.sh" ] && [ "$stamp" -nt "$HERE/ref_shim/ref_capi.cpp" ]; then
  exit 0
fi
# unmodified sources, h = 0.035
build fwd_dx0p035 "$SRC/fk_forward_Et_mono_PARAMETERS.cu" FKREF_FORWARD "$SRC"
build grad_dx0p035 "$SRC/fk_grad_Et_mono_PARAMETERS.cu" FKREF_GRAD "$SRC"
# h = 0.025 variant: generated header + include line switched in a copy
sed 's/constexpr double h = 0.035;/constexpr double h = 0.025;/' \
    "$SRC/fk_parameters_00_05_alpha_0p8_dx_0p035.h" > "$OUT/src/fk_parameters_dx_0p025.h"
grep -q 'h = 0.025' "$OUT/src/fk_parameters_dx_0p025.h"
for f in fk_forward_Et_mono_PARAMETERS fk_grad_Et_mono_PARAMETERS; do
  sed -e 's/#include "fk_parameters_00_05_alpha_0p8_dx_0p035.h"/#include "fk_parameters_dx_0p025.h"/' \
      "$SRC/$f.cu" > "$OUT/src/$f.cu"
done
build fwd_dx0p025 "$OUT/src/fk_forward_Et_mono_PARAMETERS.cu" FKREF_FORWARD "$SRC"
build grad_dx0p025 "$OUT/src/fk_grad_Et_mono_PARAMETERS.cu" FKREF_GRAD "$SRC"
touch "$stamp"
echo "reference built into $OUT"
