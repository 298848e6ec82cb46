#!/bin/bash
# Builds the REFERENCE implementation's CPU code, from its own sources where they lie,
# into oracle/_ref/ as shared libraries driven by oracle/ref_harness.c. Test
# infrastructure only (pins the CPU oracle; CPU baseline of the benchmark).
#
#   libref_cpu8a_{d,s}.so  default CPU path: sibling-blocking M2L (CPU8A)
#   libref_cpu9a_{d,s}.so  ij-blocking CPU M2L (CPU9A, the aux_CPU9* family)
#   libref_cpu8a_{d,s}_{r4,force}.so  the 1/r^4 (ONEOVERR4) and x / r^3 (LAPLACIANFORCE) builds
#   libref_cpu8a_ascii_d.so  the ENABLE_ASCII_IO build (operator files as text)
#   libref_dropin_*.so  the same code with the pass objects taken from the B200 library
#
# Flags follow the reference's own recipes (www.sh:23-36, zzz.sh:209-212) with gcc,
# -fcommon (bbfmm.h defines globals in a header) and gettimeofday timers. BLAS/LAPACK
# (?gesvd, ?gemm, ?dot) come from the OpenBLAS that ships inside the opencv wheel of
# this image. Usage: oracle/build_ref.sh [reference-dir]; without an argument the
# directory comes from BBFMM_REFERENCE_DIR, else the reference checkout's location in the
# build container. Exit code 2: no reference sources there (nothing built).
set -euo pipefail
REF=${1:-${BBFMM_REFERENCE_DIR:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
[ -f "$REF/bbfmm.c" ] || { echo "reference sources not found in $REF" >&2; exit 2; }
PY=${PYTHON:-python}
SITE=$($PY -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')
BL="$SITE/opencv_python_headless.libs"
BLAS=$(cd "$BL" && ls libopenblas*.so 2>/dev/null | head -1)
[ -n "$BLAS" ] || { echo "no OpenBLAS found under $BL" >&2; exit 3; }
mkdir -p "$OUT"
SRCS="bbfmm.c options.c checks.c opts.c envs.c output.c timer.c elapsed.c anotherFMMCompute.c
      anotherFMMInteraction.c anotherDownwardPassX.c anotherDownwardPass.c anotherUpwardPass.c
      anotherFMMDistribute.c anotherInteractionList.c anotherNearField.c m2l_aux.c
      auxAnotherFMMInteraction.c anotherBuildFMMHierachy.c xdot.c atransx.c m2l_aux_cpu.c"
KDEF=-DLAPLACIAN  # the kernel of the build (bbfmm.c:109-144)
build() {  # $1 = output name, rest = extra defines
  local name=$1; shift
  local objdir="$OUT/obj_$name"
  mkdir -p "$objdir"
  local objs=""
  for s in $SRCS; do
    gcc -std=gnu99 -O3 -fopenmp -fcommon -fPIC -w $KDEF -DFAST_HOST_CODE \
        -DENABLE_GETTIMEOFDAY "$@" -I"$REF" -c "$REF/$s" -o "$objdir/${s%.c}.o" &
    objs="$objs $objdir/${s%.c}.o"
  done
  gcc -std=gnu99 -O3 -fopenmp -fcommon -fPIC -w $KDEF -DFAST_HOST_CODE "$@" -I"$REF" \
      -c "$HERE/ref_harness.c" -o "$objdir/ref_harness.o" &
  wait
  gcc -shared -fopenmp -o "$OUT/$name.so" $objs "$objdir/ref_harness.o" \
      -L"$BL" -l:"$BLAS" -Wl,--disable-new-dtags,-rpath,"$BL" -lm
  rm -rf "$objdir"
}
build libref_cpu8a_d -DCPU8 -DCPU8A
build libref_cpu8a_s -DCPU8 -DCPU8A -DSINGLE
build libref_cpu9a_d -DCPU9 -DCPU9A
build libref_cpu9a_s -DCPU9 -DCPU9A -DSINGLE
KDEF=-DONEOVERR4 build libref_cpu8a_d_r4 -DCPU8 -DCPU8A  # the 1/r^4 kernel (homogeneity 4)
KDEF=-DONEOVERR4 build libref_cpu8a_s_r4 -DCPU8 -DCPU8A -DSINGLE
KDEF=-DLAPLACIANFORCE build libref_cpu8a_d_force -DCPU8 -DCPU8A  # x / r^3 (homogeneity 2)
KDEF=-DLAPLACIANFORCE build libref_cpu8a_s_force -DCPU8 -DCPU8A -DSINGLE
build libref_cpu8a_ascii_d -DCPU8 -DCPU8A -DENABLE_ASCII_IO  # operator files as text (.out)
KDEF=-DLAPLACIAN
# Drop-in build: the reference's own code with its pass objects (anotherFMMCompute,
# anotherUpwardPass, anotherFMMInteraction, anotherDownwardPass[X], anotherNearField) left
# out and resolved from the B200 library's reference-name shims instead.
LIBDIR="$HERE/../bbfmm_b200/lib"
if [ -f "$LIBDIR/libbbfmm_b200_ref_d.so" ]; then
  DROP="anotherFMMCompute.c anotherFMMInteraction.c anotherDownwardPassX.c anotherDownwardPass.c
        anotherUpwardPass.c anotherNearField.c"
  # d, s, the 1/r^4 kernel (ONEOVERR4, double) and x / r^3 (LAPLACIANFORCE, double)
  for var in d s d_r4 d_force; do
    prec=${var%%_*}; kdef=-DLAPLACIAN
    [ $var = d_r4 ] && kdef=-DONEOVERR4
    [ $var = d_force ] && kdef=-DLAPLACIANFORCE
    def=""; [ $prec = s ] && def="-DSINGLE"
    objdir="$OUT/obj_dropin_$var"; mkdir -p "$objdir"; objs=""
    for src in $SRCS; do
      case " $(echo $DROP) " in *" $src "*) continue;; esac
      gcc -std=gnu99 -O3 -fopenmp -fcommon -fPIC -w $kdef -DFAST_HOST_CODE -DENABLE_GETTIMEOFDAY \
          -DCPU8 -DCPU8A $def -I"$REF" -c "$REF/$src" -o "$objdir/${src%.c}.o" &
      objs="$objs $objdir/${src%.c}.o"
    done
    gcc -std=gnu99 -O3 -fopenmp -fcommon -fPIC -w $kdef -DFAST_HOST_CODE -DCPU8 -DCPU8A $def -I"$REF" \
        -c "$HERE/ref_harness.c" -o "$objdir/ref_harness.o" &
    wait
    gcc -shared -fopenmp -o "$OUT/libref_dropin_$var.so" $objs "$objdir/ref_harness.o" \
        -L"$LIBDIR" -l:libbbfmm_b200_ref_$prec.so -Wl,--disable-new-dtags,-rpath,'$ORIGIN/../../bbfmm_b200/lib' \
        -L"$BL" -l:"$BLAS" -Wl,-rpath,"$BL" -lm
    rm -rf "$objdir"
  done
fi
echo "built reference CPU libraries in $OUT"
