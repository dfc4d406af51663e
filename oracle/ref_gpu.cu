// Test infrastructure and measured baseline only: the reference's own GPU kernel
// CUFLU_FluidSolver_MHM (src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_MHM.cpp:265, reached through
// src/Model_Hydro/GPU_Hydro/CUFLU_FluidSolver_MHM.cu) and its gamma-law EoS
// (src/EoS/Gamma/GPU_EoS_Gamma.cu), compiled unmodified for sm_100a from the reference tree, where
// they lie, by oracle/build_ref_gpu.sh into oracle/_ref/libgrefgpu_<variant>_<prec>.so.  The product
// never links or loads it: the bench times it beside this repository's solver on the same device
// arrays, and a GPU test checks it against the reference CPU solver.
//
// What this file adds is the launch the reference's CUAPI_Asyn_FluidSolver performs
// (src/GPU_API/CUAPI_Asyn_FluidSolver.cu:557-575): the global-memory scratch of
// CUAPI_MemAllocate_Fluid (src/GPU_API/CUAPI_MemAllocate_Fluid.cu:116-120, 242-249), the EoS
// constants and device function pointers of CUAPI_SetConstMemory_EoS / EoS_Init_Gamma, one CTA of
// FLU_BLOCK_SIZE_X threads per patch group.
#define DEFINE_GLOBAL
#include "CUFLU.h"
#include GREF_GPU_MHM
#include GREF_GPU_EOS

#include <cstdarg>
#include <cstdio>
#include <cstdlib>

// the reference reports CUDA errors through Aux_Error (include/CUDA_CheckError.h); here a failed
// set-up call is printed and the process ends, as in the reference
void Aux_Error( const char *File, const int Line, const char *Func, const char *Format, ... )
{
   va_list ap;
   va_start( ap, Format );
   fprintf( stderr, "grefgpu: %s:%d %s: ", File, Line, Func );
   vfprintf( stderr, Format, ap );
   va_end( ap );
   exit( 1 );
}

namespace {

EoS_t  g_eos;
bool   g_eos_ready = false;
double g_gamma     = 0.0;
real  *g_privar = NULL, *g_fcvar = NULL, *g_fcflux = NULL, *g_slope = NULL;
long   g_npg_alloc = 0;

// the reference's per-patch-group scratch (CUAPI_MemAllocate_Fluid.cu:116-120)
int ensure_scratch( const long npg )
{
   if ( npg <= g_npg_alloc )  return 0;
   cudaFree( g_privar );  cudaFree( g_fcvar );  cudaFree( g_fcflux );  cudaFree( g_slope );
   g_privar = g_fcvar = g_fcflux = g_slope = NULL;
   g_npg_alloc = 0;
   if ( cudaMalloc( (void**)&g_privar, sizeof(real)*npg*NCOMP_LR*CUBE(FLU_NXT) ) != cudaSuccess ||
        cudaMalloc( (void**)&g_fcvar,  sizeof(real)*npg*6*NCOMP_TOTAL_PLUS_MAG*CUBE(N_FC_VAR) ) != cudaSuccess ||
        cudaMalloc( (void**)&g_fcflux, sizeof(real)*npg*3*NCOMP_TOTAL_PLUS_MAG*CUBE(N_FC_FLUX) ) != cudaSuccess )
      return 1;
#  if ( LR_SCHEME == PPM )
   if ( cudaMalloc( (void**)&g_slope, sizeof(real)*npg*3*NCOMP_LR*CUBE(N_SLOPE_PPM) ) != cudaSuccess )   return 1;
#  endif
   g_npg_alloc = npg;
   return 0;
}

// EoS_SetAuxArray_Gamma (src/EoS/Gamma/CPU_EoS_Gamma.cpp:54-65, OPT__UNIT off, MOLECULAR_WEIGHT 0.6),
// copied to constant memory as CUAPI_SetConstMemory_EoS does, and the device function pointers of
// EoS_SetGPUFunc_Gamma
int ensure_eos( const double gamma )
{
   if ( g_eos_ready  &&  gamma == g_gamma )  return 0;
   double flt[EOS_NAUX_MAX] = { 0.0 };
   int    in[EOS_NAUX_MAX]  = { 0 };
   flt[0] = gamma;
   flt[1] = gamma - 1.0;
   flt[2] = 1.0/( gamma - 1.0 );
   flt[3] = 1.0/gamma;
   flt[4] = 0.6;
   flt[5] = 1.0/flt[4];
   real *table[EOS_NTABLE_MAX] = { NULL };
   if ( cudaMemcpyToSymbol( c_EoS_AuxArray_Flt, flt, sizeof(flt) ) != cudaSuccess ||
        cudaMemcpyToSymbol( c_EoS_AuxArray_Int, in, sizeof(in) ) != cudaSuccess ||
        cudaMemcpyToSymbol( c_EoS_Table, table, sizeof(table) ) != cudaSuccess ||
        cudaGetSymbolAddress( (void**)&g_eos.AuxArrayDevPtr_Flt, c_EoS_AuxArray_Flt ) != cudaSuccess ||
        cudaGetSymbolAddress( (void**)&g_eos.AuxArrayDevPtr_Int, c_EoS_AuxArray_Int ) != cudaSuccess ||
        cudaGetSymbolAddress( (void**)&g_eos.Table, c_EoS_Table ) != cudaSuccess )
      return 1;
   g_eos.GuessHTilde_FuncPtr = NULL;
   g_eos.HTilde2Temp_FuncPtr = NULL;
   g_eos.Temp2HTilde_FuncPtr = NULL;
   EoS_SetGPUFunc_Gamma( g_eos.DensEint2Pres_FuncPtr, g_eos.DensPres2Eint_FuncPtr, g_eos.DensPres2CSqr_FuncPtr,
                         g_eos.DensEint2Temp_FuncPtr, g_eos.DensTemp2Pres_FuncPtr, g_eos.DensEint2Entr_FuncPtr,
                         g_eos.General_FuncPtr );
   g_gamma = gamma;
   g_eos_ready = true;
   return 0;
}

} // namespace

extern "C" {

// info[0] FLU_NXT, [1] NCOMP_TOTAL, [2] sizeof(real), [3] FLU_BLOCK_SIZE_X, [4] patch-group scratch
// bytes (the global-memory round trips of the reference kernel)
__attribute__((visibility("default")))
int grefgpu_info( long *info )
{
   info[0] = FLU_NXT;
   info[1] = NCOMP_TOTAL;
   info[2] = sizeof(real);
   info[3] = FLU_BLOCK_SIZE_X;
   info[4] = (long)sizeof(real)*( NCOMP_LR*CUBE(FLU_NXT) + 6*NCOMP_TOTAL_PLUS_MAG*CUBE(N_FC_VAR) +
                                  3*NCOMP_TOTAL_PLUS_MAG*CUBE(N_FC_FLUX) );
   return 0;
}

// One launch of CUFLU_FluidSolver_MHM over npg patch groups of DEVICE arrays on `stream`, as
// CUAPI_Asyn_FluidSolver issues it (CUAPI_Asyn_FluidSolver.cu:557-575): in [npg][NCOMP][FLU_NXT^3],
// out [npg][NCOMP][16^3], flux [npg][9][NCOMP][16^2] (NULL when store_flux == 0), de [npg][16^3]
// (dual energy only).  Returns 0, or 1 when the scratch or the launch failed.
__attribute__((visibility("default")))
int grefgpu_solve( const void *in, void *out, void *flux, char *de, const int npg, const double dt, const double dh,
                   const int store_flux, const int lr_limiter, const double minmod_coeff, const int minmod_maxiter,
                   const double min_dens, const double min_pres, const double min_eint, const double de_switch,
                   const double gamma, void *stream )
{
   if ( npg <= 0 )  return 0;
   if ( ensure_eos( gamma ) != 0  ||  ensure_scratch( npg ) != 0 )  { cudaGetLastError();  return 1; }
#  ifdef DUAL_ENERGY
   const long PassiveFloor = BIDX( DUAL );
#  else
   const long PassiveFloor = 0L;
#  endif
   MicroPhy_t MicroPhy;
   MicroPhy.useless = false;
   typedef real FluIn_t  [NCOMP_TOTAL][ CUBE(FLU_NXT) ];
   typedef real FluOut_t [NCOMP_TOTAL][ CUBE(PS2) ];
   typedef real Flux_t   [9][NCOMP_TOTAL][ SQR(PS2) ];
   typedef char DE_t     [ CUBE(PS2) ];
   typedef real PriVar_t [NCOMP_LR][ CUBE(FLU_NXT) ];
   typedef real Slope_t  [3][NCOMP_LR][ CUBE(N_SLOPE_PPM) ];
   typedef real FCVar_t  [6][NCOMP_TOTAL_PLUS_MAG][ CUBE(N_FC_VAR) ];
   typedef real FCFlux_t [3][NCOMP_TOTAL_PLUS_MAG][ CUBE(N_FC_FLUX) ];
   CUFLU_FluidSolver_MHM <<< npg, FLU_BLOCK_SIZE_X, 0, (cudaStream_t)stream >>>
      ( (const FluIn_t*)in, (FluOut_t*)out, NULL, NULL, (DE_t*)de, (Flux_t*)flux, NULL, NULL, NULL,
        (PriVar_t*)g_privar, (Slope_t*)g_slope, (FCVar_t*)g_fcvar, (FCFlux_t*)g_fcflux, NULL, NULL,
        (real)dt, (real)dh, store_flux != 0, false, (LR_Limiter_t)lr_limiter, (real)minmod_coeff, minmod_maxiter,
        0.0, false, EXT_ACC_NONE, NULL, (real)min_dens, (real)min_pres, (real)min_eint, (real)de_switch,
        PassiveFloor, false, 0, false, 0, false, (real)0.0, g_eos, MicroPhy );
   return ( cudaGetLastError() == cudaSuccess ) ? 0 : 1;
}

} // extern "C"
