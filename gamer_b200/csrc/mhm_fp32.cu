// Instantiations of the MHM kernel for the P_FP32 policy (PLM/PPM x HLLC/HLLE/Roe x 5/6 variables).
#include "mhm_launch.cuh"
GB_MHM_REGISTRY( mhm_lookup_fp32, float, P_FP32, GB_MHM_REG_PICK )
