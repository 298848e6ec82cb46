#!/bin/bash
# Builds the REFERENCE implementation's GPU program (main.cu: its own octree, M2L scheme 0-3
# on the GPU via m2l_drv, postm2l and passes on the host, the `direct` near-field kernel) for
# sm_100a from its own sources, into oracle/_ref/gpu/ref_gpu_{d,s}_scheme{0..3}. Baseline /
# checker only: it times the reference's own kernels (timer_m2l_kernel, time_direct_kernel)
# on a B200. The build writes objects beside the sources, so it runs in a copy of the tree;
# cutil.h, from an SDK that no longer exists, is replaced by a one-line stub. Flags follow the
# reference's cumake_gcc.sh with the CUDA 4.6 tilings it selects for sm_20 (CUDA_ARCH=20 only
# picks the 8x1 (d) / 8x2 (s) register tiling of the ij-blocking kernel; the code is compiled
# for sm_100a).
#
# Usage: oracle/build_ref_gpu.sh [reference-dir] ["schemes"] ["precisions"]; without a
# directory it comes from BBFMM_REFERENCE_DIR, else the reference checkout's location in the
# build container. Exit code 2: no reference sources there.
set -euo pipefail
REF=${1:-${BBFMM_REFERENCE_DIR:-/root/reference}}
SCHEMES=${2:-"0 1 2 3"}
PRECS=${3:-"d s"}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref/gpu"
[ -f "$REF/main.cu" ] || { echo "reference sources not found in $REF" >&2; exit 2; }
PY=${PYTHON:-python}
SITE=$($PY -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')
BL="$SITE/opencv_python_headless.libs"
BLAS=$(cd "$BL" && ls libopenblas*.so 2>/dev/null | head -1)
[ -n "$BLAS" ] || { echo "no OpenBLAS found under $BL" >&2; exit 3; }
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
mkdir -p "$OUT"
one() {  # $1 = d|s, $2 = scheme
  local prec=$1 scheme=$2 def=""
  [ "$prec" = s ] && def="-DSINGLE"
  local W
  W=$(mktemp -d)
  cp -r "$REF/." "$W/"
  mkdir -p "$W/stub"
  echo '#define CUDA_SAFE_CALL(call) (call)' > "$W/stub/cutil.h"
  (cd "$W" && make -s -f Makefile.cuda CC=gcc NVCC="$NVCC" CUEXE=cuda.out CPU_CLOCK_GHZ=2.0 \
      OPTS="-std=gnu99 -O3 -fopenmp -fcommon -w -DLAPLACIAN -DFAST_HOST_CODE $def" \
      OPTS_ELAPSED=-DENABLE_GETTIMEOFDAY OMP="-lgomp -lpthread" \
      LIBS="$BL/$BLAS -Xlinker -rpath,$BL -lm" \
      CUOPTS="-O3 -w -DCUDA -DLAPLACIAN $def -DCUDA_VER46 -DCUDA_VER46Q -DFAST_HOST_CODE -DSCHEME=$scheme \
              -DLEVEL_SWITCH_IJ=2 -DNUM_ROW_GROUPS_IJ=4 -DDIRECT_NUM_THREADS_PER_BLOCK=64 -DDIRECT_SHARE_SIZE=64 \
              -gencode arch=compute_100a,code=sm_100a -DCUDA_ARCH=20 -Xcompiler -fopenmp,-fcommon" \
      CUINCLUDES="-I. -Istub" CULIBS="-lcudart" CULDFLAGS="-Xlinker -rpath-link=$BL" \
      > "$W/build.log" 2>&1) || { tail -30 "$W/build.log" >&2; rm -rf "$W"; return 1; }
  cp "$W/cuda.out" "$OUT/ref_gpu_${prec}_scheme${scheme}"
  rm -rf "$W"
}
pids=""
for p in $PRECS; do
  for s in $SCHEMES; do
    one "$p" "$s" &
    pids="$pids $!"
  done
done
rc=0
for p in $pids; do wait "$p" || rc=1; done
[ $rc = 0 ] && echo "built reference GPU programs in $OUT"
exit $rc
