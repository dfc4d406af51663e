#!/usr/bin/env bash
# Test infrastructure and measured baseline only: build the reference's own GPU fluid-solver kernel
# (CUFLU_FluidSolver_MHM with its gamma-law EoS), unmodified, for sm_100a.
#
# oracle/ref_gpu.cu includes the reference sources where they lie (never copied) and adds the
# launch of CUAPI_Asyn_FluidSolver; one shared library per compile-time variant under oracle/_ref/.
# Flags: the reference's GB200 build (configs/nano4_gnu-arm_GB200.config: NVCCFLAG_COM -O3,
# NVCCFLAG_FLU -Xptxas -dlcm=ca -prec-div=false -ftz=true) with the register caps src/configure.py
# sets for compute capability 10.x (--maxrregcount=128 in FP32, 192 with FLOAT8), and sm_100a code.
#
# usage: oracle/build_ref_gpu.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $GAMER_REFERENCE_ROOT, else to the read-only reference checkout of the
#   build container (/root/reference).  Without a reference tree the prebuilt libraries are kept.
set -euo pipefail
REF=${1:-${GAMER_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
mkdir -p "$OUT"
if [ ! -d "$REF/src" ]; then
  echo "build_ref_gpu.sh: reference tree $REF not found; keeping existing oracle/_ref" >&2
  exit 0
fi

BASE="-gencode arch=compute_100a,code=sm_100a -O3 -Xptxas -dlcm=ca -prec-div=false -ftz=true
      -Xcompiler -fPIC -shared -Xcompiler -fvisibility=hidden -w -Xptxas -v
      -I$REF/include -I$REF/src/Model_Hydro/GPU_Hydro
      -DGPU -DGPU_COMPUTE_CAPABILITY=1000 -DMODEL=HYDRO -DEOS=EOS_GAMMA -DNCOMP_PASSIVE_USER=0
      -DPATCH_SIZE=8 -DNLEVEL=10 -DMAX_PATCH=1000000 -DSERIAL -DRANDOM_NUMBER=RNG_GNU_EXT"
INC="-DGREF_GPU_MHM=\"$REF/src/Model_Hydro/GPU_Hydro/CUFLU_FluidSolver_MHM.cu\"
     -DGREF_GPU_EOS=\"$REF/src/EoS/Gamma/GPU_EoS_Gamma.cu\""

# name : flags
VARIANTS=(
  "mhm_plm_hllc:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLC"
  "mhm_ppm_roe:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=ROE"
)

build_one() {
  local name=$1 flags=$2 prec=$3 pflag=$4
  local so="$OUT/libgrefgpu_${name}_${prec}.so"
  # shellcheck disable=SC2086
  $NVCC $BASE $INC $flags $pflag "$HERE/ref_gpu.cu" -o "$so.tmp" > "$OUT/libgrefgpu_${name}_${prec}.ptxas.txt" 2>&1 \
    && mv "$so.tmp" "$so" || { cat "$OUT/libgrefgpu_${name}_${prec}.ptxas.txt" >&2; return 1; }
  echo "built $so"
}

pids=()
for v in "${VARIANTS[@]}"; do
  name=${v%%:*}; flags=${v#*:}
  build_one "$name" "$flags" fp32 "--maxrregcount=128" &
  pids+=($!)
  build_one "$name" "$flags" fp64 "-DFLOAT8 --maxrregcount=192" &
  pids+=($!)
done
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
exit $rc
