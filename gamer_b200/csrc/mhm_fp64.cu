// Instantiations of the MHM kernel for the P_FP64 policy (PLM/PPM x HLLC/HLLE/Roe x 5/6 variables).
#include "mhm_launch.cuh"
GB_MHM_REGISTRY( mhm_lookup_fp64, double, P_FP64, GB_MHM_NO_REG_PICK )
