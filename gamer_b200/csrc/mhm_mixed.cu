// Instantiations of the MHM kernel for the P_MIXED policy (PLM/PPM x HLLC/HLLE/Roe x 5/6 variables).
#include "mhm_launch.cuh"
GB_MHM_REGISTRY( mhm_lookup_mixed, float, P_MIXED, GB_MHM_REG_PICK )
