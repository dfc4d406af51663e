#!/usr/bin/env bash
# Test infrastructure only: build the reference CPU fluid solver, unmodified, as the oracle.
#
# Compiles the reference's own sources (read in place, never copied) together with
# oracle/ref_stub.cpp into one shared library per compile-time variant under oracle/_ref/.
# The reference selects scheme / reconstruction / Riemann solver / precision / MHD / dual energy
# at compile time (src/configure.py), so every variant is a separate library.
#
# usage: oracle/build_ref.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $GAMER_REFERENCE_ROOT, else to the read-only reference checkout of the
#   build container (/root/reference).  Without a reference tree the prebuilt oracle/_ref is kept.
#   GREF_ONLY=<bash glob> builds only the variants whose name matches (e.g. GREF_ONLY='ctu_*_mhd').
set -euo pipefail
REF=${1:-${GAMER_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -d "$REF/src" ]; then
  echo "build_ref.sh: reference tree $REF not found; keeping existing oracle/_ref" >&2
  exit 0
fi

SRC=(
  "$REF/src/Fluid/CPU_FluidSolver.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_MHM.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_CTU.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_DataReconstruction.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_ComputeFlux.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_FullStepUpdate.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_FluUtility.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_DualEnergy.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_ConstrainedTransport.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_RiemannSolver_HLLC.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_RiemannSolver_HLLE.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_RiemannSolver_HLLD.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_RiemannSolver_Roe.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_Shared_RiemannSolver_Exact.cpp"
  "$REF/src/Model_Hydro/CPU_Hydro/CPU_dtSolver_HydroCFL.cpp"
  "$REF/src/EoS/Gamma/CPU_EoS_Gamma.cpp"
  "$HERE/ref_stub.cpp"
)

BASE="-O3 -fopenmp -ffp-contract=off -fPIC -shared -fvisibility=hidden -Wl,-Bsymbolic -w
      -I$REF/include -DMODEL=HYDRO -DEOS=EOS_GAMMA -DNCOMP_PASSIVE_USER=0 -DPATCH_SIZE=8
      -DNLEVEL=10 -DMAX_PATCH=1000000 -DSERIAL -DOPENMP -DRANDOM_NUMBER=RNG_GNU_EXT"

# name : flags
VARIANTS=(
  "mhm_plm_hllc:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLC"
  "mhm_plm_roe:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=ROE"
  "mhm_plm_hlle:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLE"
  "mhm_ppm_roe:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=ROE"
  "mhm_plm_exact:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=EXACT"
  "mhm_ppm_exact:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=EXACT"
  "mhm_plm_exact_de:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=EXACT -DDUAL_ENERGY=DE_ENPY"
  "mhm_ppm_exact_de:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=EXACT -DDUAL_ENERGY=DE_ENPY"
  "mhm_ppm_hllc:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=HLLC"
  "mhm_plm_hllc_de:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY"
  "mhm_plm_hllc_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLC -DCHAR_RECONSTRUCTION"
  "mhm_plm_roe_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=ROE -DCHAR_RECONSTRUCTION"
  "mhm_plm_hlle_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLE -DCHAR_RECONSTRUCTION"
  "mhm_ppm_hllc_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=HLLC -DCHAR_RECONSTRUCTION"
  "mhm_ppm_roe_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=ROE -DCHAR_RECONSTRUCTION"
  "mhm_plm_exact_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=EXACT -DCHAR_RECONSTRUCTION"
  "mhm_ppm_exact_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=EXACT -DCHAR_RECONSTRUCTION"
  "mhm_ppm_hllc_de_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY -DCHAR_RECONSTRUCTION"
  "mhm_ppm_roe_de:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=ROE -DDUAL_ENERGY=DE_ENPY"
  "mhmrp_plm_hllc:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLC"
  "mhmrp_plm_roe:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=ROE"
  "mhmrp_plm_hlle:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLE"
  "mhmrp_plm_hllc_de:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY"
  "mhmrp_ppm_hllc:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLC"
  "mhmrp_ppm_roe:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=ROE"
  "mhmrp_ppm_hlle:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLE"
  "mhmrp_ppm_hllc_de:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY"
  "mhmrp_ppm_hllc_char:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLC -DCHAR_RECONSTRUCTION"
  "mhmrp_ppm_roe_char:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=ROE -DCHAR_RECONSTRUCTION"
  "mhmrp_ppm_hllc_de_char:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY -DCHAR_RECONSTRUCTION"
  "mhmrp_plm_hllc_char:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLC -DCHAR_RECONSTRUCTION"
  "mhmrp_plm_roe_char:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=ROE -DCHAR_RECONSTRUCTION"
  "mhmrp_plm_hllc_de_char:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY -DCHAR_RECONSTRUCTION"
  "mhm_plm_hllc_p2:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLC -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "mhmrp_plm_hllc_p2:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLC -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "mhmrp_plm_roe_p2_de:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=ROE -DDUAL_ENERGY=DE_ENPY -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "mhmrp_plm_hllc_p2_char:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLC -DCHAR_RECONSTRUCTION -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "mhmrp_ppm_hllc_p2_char:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLC -DCHAR_RECONSTRUCTION -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "mhm_ppm_roe_p2_de_char:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=ROE -DDUAL_ENERGY=DE_ENPY -DCHAR_RECONSTRUCTION -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "mhmrp_ppm_hllc_p2:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLC -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "mhmrp_ppm_hlle_p2_de:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLE -DDUAL_ENERGY=DE_ENPY -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "mhm_plm_hllc_p2_de:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "ctu_plm_hllc:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLC"
  "ctu_plm_hlle:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLE"
  "ctu_plm_roe:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=ROE"
  "ctu_plm_exact:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=EXACT"
  "ctu_plm_hllc_de:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY"
  "ctu_plm_roe_de:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=ROE -DDUAL_ENERGY=DE_ENPY"
  "ctu_plm_hllc_p2:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLC -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "ctu_plm_roe_p2:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=ROE -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "ctu_plm_hllc_p2_de:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "ctu_ppm_hllc:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=HLLC"
  "ctu_ppm_roe:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=ROE"
  "ctu_ppm_hlle:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=HLLE"
  "ctu_ppm_exact:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=EXACT"
  "ctu_ppm_hllc_de:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY"
  "ctu_ppm_hllc_char:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=HLLC -DCHAR_RECONSTRUCTION"
  "ctu_ppm_hllc_p2:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=HLLC -UNCOMP_PASSIVE_USER -DNCOMP_PASSIVE_USER=2"
  "ctu_plm_hllc_char:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLC -DCHAR_RECONSTRUCTION"
  "ctu_plm_roe_char:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=ROE -DCHAR_RECONSTRUCTION"
  "ctu_plm_exact_char:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=EXACT -DCHAR_RECONSTRUCTION"
  "ctu_plm_hllc_de_char:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLC -DDUAL_ENERGY=DE_ENPY -DCHAR_RECONSTRUCTION"
  "ctu_plm_hlld_mhd:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLD -DMHD"
  "ctu_plm_hlld_char_mhd:-DFLU_SCHEME=CTU -DLR_SCHEME=PLM -DRSOLVER=HLLD -DMHD -DCHAR_RECONSTRUCTION"
  "ctu_ppm_hlld_mhd:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=HLLD -DMHD"
  "ctu_ppm_hlld_char_mhd:-DFLU_SCHEME=CTU -DLR_SCHEME=PPM -DRSOLVER=HLLD -DMHD -DCHAR_RECONSTRUCTION"
  "mhmrp_plm_hlld_mhd:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLD -DMHD"
  "mhm_plm_hlld_mhd:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLD -DMHD"
  "mhm_plm_hlld_char_mhd:-DFLU_SCHEME=MHM -DLR_SCHEME=PLM -DRSOLVER=HLLD -DMHD -DCHAR_RECONSTRUCTION"
  "mhm_ppm_hlld_mhd:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=HLLD -DMHD"
  "mhm_ppm_hlld_char_mhd:-DFLU_SCHEME=MHM -DLR_SCHEME=PPM -DRSOLVER=HLLD -DMHD -DCHAR_RECONSTRUCTION"
  "mhmrp_plm_hlld_char_mhd:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PLM -DRSOLVER=HLLD -DMHD -DCHAR_RECONSTRUCTION"
  "mhmrp_ppm_hlld_mhd:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLD -DMHD"
  "mhmrp_ppm_hlld_char_mhd:-DFLU_SCHEME=MHM_RP -DLR_SCHEME=PPM -DRSOLVER=HLLD -DMHD -DCHAR_RECONSTRUCTION"
)

# hydro MHM variants also carry CorrectUnphysical() of src/Fluid/Flu_Close.cpp (oracle/ref_close.cpp
# includes that file where it lies), Flu_FixUp_Flux() (oracle/ref_fixup.cpp) and the spatial
# interpolation Interpolate() with its schemes (oracle/ref_interp.cpp includes Interpolate.cpp)
CLOSE_SRC=(
  "$HERE/ref_close.cpp"
  "$HERE/ref_fixup.cpp"
  "$HERE/ref_interp.cpp"
  "$REF/src/Fluid/Flu_FixUp_Flux.cpp"
  "$REF/src/Auxiliary/Aux_IsFinite.cpp"
  "$REF/src/Tables/Table_02.cpp"
  "$REF/src/Interpolation/Int_MinMod1D.cpp"
  "$REF/src/Interpolation/Int_MinMod3D.cpp"
  "$REF/src/Interpolation/Int_vanLeer.cpp"
  "$REF/src/Interpolation/Int_CQuadratic.cpp"
  "$REF/src/Interpolation/Int_Quadratic.cpp"
  "$REF/src/Interpolation/Int_CQuartic.cpp"
  "$REF/src/Interpolation/Int_Quartic.cpp"
)

# the CTU+MHD variant carries the MHD branches of the same close consumers: CorrectUnphysical(),
# Flu_FixUp_Flux() with the magnetic energy, and MHD_FixUp_Electric()
MHD_CLOSE_SRC=(
  "$HERE/ref_close.cpp"
  "$HERE/ref_fixup.cpp"
  "$REF/src/Fluid/Flu_FixUp_Flux.cpp"
  "$REF/src/Model_Hydro/MHD_FixUp_Electric.cpp"
  "$REF/src/Model_Hydro/MHD_GetCellCenteredBInPatch.cpp"
  "$REF/src/Auxiliary/Aux_IsFinite.cpp"
  "$REF/src/Tables/Table_02.cpp"
  "$REF/src/Tables/Table_SiblingSharingSameEdge.cpp"
)

build_one() {
  local name=$1 flags=$2 prec=$3 pflag=$4
  local so="$OUT/libgref_${name}_${prec}.so"
  local extra=()
  if [[ $name == *_mhd ]]; then
    extra=("${MHD_CLOSE_SRC[@]}" "-DGREF_FLU_CLOSE=\"$REF/src/Fluid/Flu_Close.cpp\"" -Wl,--no-undefined)
  elif [[ $name == mhm_* ]]; then
    extra=("${CLOSE_SRC[@]}" "-DGREF_FLU_CLOSE=\"$REF/src/Fluid/Flu_Close.cpp\""
           "-DGREF_INTERPOLATE=\"$REF/src/Interpolation/Interpolate.cpp\"" -Wl,--no-undefined)
  fi
  # shellcheck disable=SC2086
  g++ $BASE $flags $pflag "${SRC[@]}" "${extra[@]}" -o "$so.tmp" && mv "$so.tmp" "$so"
  echo "built $so"
}

pids=()
for v in "${VARIANTS[@]}"; do
  name=${v%%:*}; flags=${v#*:}
  # shellcheck disable=SC2053
  [[ -n ${GREF_ONLY:-} && $name != $GREF_ONLY ]] && continue
  build_one "$name" "$flags" fp32 "" &
  pids+=($!)
  build_one "$name" "$flags" fp64 "-DFLOAT8" &
  pids+=($!)
done
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
exit $rc
