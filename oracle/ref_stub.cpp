// Test infrastructure only: the C entry point of the reference-solver oracle.
//
// This file is compiled together with the UNMODIFIED reference sources
//    src/Fluid/CPU_FluidSolver.cpp
//    src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_{MHM,CTU}.cpp
//    src/Model_Hydro/CPU_Hydro/CPU_Shared_*.cpp
//    src/EoS/Gamma/CPU_EoS_Gamma.cpp
// into one shared library per compile-time variant (oracle/build_ref.sh).  It defines the
// handful of globals that those files expect from the rest of GAMER (they live in
// src/Main/Main.cpp:300-334 and src/Init/Init_MemAllocate_Fluid.cpp:91 in the reference) and
// exports two plain C functions used by the tests and by the CPU baseline leg of bench.py:
//
//    gref_info(int info[GREF_NINFO])   compile-time layout of this variant
//    gref_solve(...)                   one call of CPU_FluidSolver() (src/Fluid/CPU_FluidSolver.cpp:210)
//    gref_dt(...)                      one call of CPU_dtSolver_HydroCFL()
//                                      (src/Model_Hydro/CPU_Hydro/CPU_dtSolver_HydroCFL.cpp:57)
//
// Nothing in the product links this file.

#include "GAMER.h"
#include "CUFLU.h"
#include <omp.h>

// ---- globals normally defined by src/Main/Main.cpp -------------------------------------------
double GAMMA = 5.0/3.0, MOLECULAR_WEIGHT = 0.6, MU_NORM = 1.0, UNIT_E = 1.0, UNIT_M = 1.0;
bool   OPT__UNIT = false;

double EoS_AuxArray_Flt[EOS_NAUX_MAX];
int    EoS_AuxArray_Int[EOS_NAUX_MAX];
EoS_GUESS_t   EoS_GuessHTilde_CPUPtr   = NULL;
EoS_H2TEM_t   EoS_HTilde2Temp_CPUPtr   = NULL;
EoS_TEM2H_t   EoS_Temp2HTilde_CPUPtr   = NULL;
EoS_DE2P_t    EoS_DensEint2Pres_CPUPtr = NULL;
EoS_DP2E_t    EoS_DensPres2Eint_CPUPtr = NULL;
EoS_DP2C_t    EoS_DensPres2CSqr_CPUPtr = NULL;
EoS_DE2T_t    EoS_DensEint2Temp_CPUPtr = NULL;
EoS_DT2P_t    EoS_DensTemp2Pres_CPUPtr = NULL;
EoS_DE2S_t    EoS_DensEint2Entr_CPUPtr = NULL;
EoS_GENE_t    EoS_General_CPUPtr       = NULL;
EoS_t EoS;

// ---- solver scratch normally allocated by src/Init/Init_MemAllocate_Fluid.cpp ------------------
real (*h_PriVar)      [NCOMP_LR            ][ CUBE(FLU_NXT)     ] = NULL;
real (*h_Slope_PPM)[3][NCOMP_LR            ][ CUBE(N_SLOPE_PPM) ] = NULL;
real (*h_FC_Var)   [6][NCOMP_TOTAL_PLUS_MAG][ CUBE(N_FC_VAR)    ] = NULL;
real (*h_FC_Flux)  [3][NCOMP_TOTAL_PLUS_MAG][ CUBE(N_FC_FLUX)   ] = NULL;
#ifdef MHD
real (*h_FC_Mag_Half)[NCOMP_MAG][ FLU_NXT_P1*SQR(FLU_NXT) ] = NULL;
real (*h_EC_Ele     )[NCOMP_MAG][ CUBE(N_EC_ELE)          ] = NULL;
#endif

void EoS_Init_Gamma();
void CPU_dtSolver_HydroCFL( real g_dt_Array[], const real g_Flu_Array[][FLU_NIN_T][ CUBE(PS1) ],
                            const real g_Mag_Array[][NCOMP_MAG][ PS1P1*SQR(PS1) ], const int NPG,
                            const real dh, const real Safety, const real MinPres,
                            const long PassiveFloor, const EoS_t EoS, const MicroPhy_t MicroPhy );

// the EoS set-up of Init_GAMER (EoS_Init + the CPU function pointers) for an ideal gas of GAMMA = gamma
static void SetEoS( const double gamma )
{
   GAMMA = gamma;
   EoS_Init_Gamma();
   EoS.AuxArrayDevPtr_Flt    = EoS_AuxArray_Flt;
   EoS.AuxArrayDevPtr_Int    = EoS_AuxArray_Int;
   EoS.DensEint2Pres_FuncPtr = EoS_DensEint2Pres_CPUPtr;
   EoS.DensPres2Eint_FuncPtr = EoS_DensPres2Eint_CPUPtr;
   EoS.DensPres2CSqr_FuncPtr = EoS_DensPres2CSqr_CPUPtr;
   EoS.DensEint2Temp_FuncPtr = EoS_DensEint2Temp_CPUPtr;
   EoS.DensTemp2Pres_FuncPtr = EoS_DensTemp2Pres_CPUPtr;
   EoS.DensEint2Entr_FuncPtr = EoS_DensEint2Entr_CPUPtr;
   EoS.GuessHTilde_FuncPtr   = EoS_GuessHTilde_CPUPtr;
   EoS.HTilde2Temp_FuncPtr   = EoS_HTilde2Temp_CPUPtr;
   EoS.Temp2HTilde_FuncPtr   = EoS_Temp2HTilde_CPUPtr;
   EoS.General_FuncPtr       = EoS_General_CPUPtr;
   EoS.Table                 = NULL;
}

#define GREF_NINFO 12
#define GREF_CHUNK 32   // patch groups per CPU_FluidSolver() call: bounds the scratch memory

static int g_ScratchNPG = 0;

static void AllocScratch( const int NPG )
{
   if ( NPG <= g_ScratchNPG )  return;
   delete [] h_PriVar;   delete [] h_Slope_PPM;   delete [] h_FC_Var;   delete [] h_FC_Flux;
   h_PriVar    = new real [NPG   ][NCOMP_LR            ][ CUBE(FLU_NXT)     ];
   h_Slope_PPM = new real [NPG][3][NCOMP_LR            ][ CUBE(N_SLOPE_PPM) ];
   h_FC_Var    = new real [NPG][6][NCOMP_TOTAL_PLUS_MAG][ CUBE(N_FC_VAR)    ];
   h_FC_Flux   = new real [NPG][3][NCOMP_TOTAL_PLUS_MAG][ CUBE(N_FC_FLUX)   ];
#  ifdef MHD
   delete [] h_FC_Mag_Half;   delete [] h_EC_Ele;
   h_FC_Mag_Half = new real [NPG][NCOMP_MAG][ FLU_NXT_P1*SQR(FLU_NXT) ];
   h_EC_Ele      = new real [NPG][NCOMP_MAG][ CUBE(N_EC_ELE)          ];
#  endif
   g_ScratchNPG = NPG;
}

extern "C" {

// info[]: 0 FLU_NXT, 1 NCOMP_TOTAL, 2 sizeof(real), 3 MHD, 4 FLU_SCHEME, 5 LR_SCHEME, 6 RSOLVER,
//         7 DUAL_ENERGY, 8 FLU_GHOST_SIZE, 9 PS2, 10 NCOMP_MAG, 11 NCOMP_ELE
__attribute__((visibility("default")))
int gref_info( int info[GREF_NINFO] )
{
   info[0]  = FLU_NXT;
   info[1]  = NCOMP_TOTAL;
   info[2]  = (int)sizeof(real);
#  ifdef MHD
   info[3]  = 1;
#  else
   info[3]  = 0;
#  endif
   info[4]  = FLU_SCHEME;
   info[5]  = LR_SCHEME;
   info[6]  = RSOLVER;
#  ifdef DUAL_ENERGY
   info[7]  = DUAL_ENERGY;
#  else
   info[7]  = 0;
#  endif
   info[8]  = FLU_GHOST_SIZE;
   info[9]  = PS2;
   info[10] = NCOMP_MAG;
   info[11] = NCOMP_ELE;
   return 0;
}

// Run-time options of the next gref_solve calls that the plain interface leaves at GAMER's defaults:
// PassiveFloor (use_default != 0: the dual-energy field when DUAL_ENERGY is on), NormPassive/NormIdx,
// FracPassive/FracIdx and JeansMinPres/JeansMinPres_Coeff (src/Fluid/CPU_FluidSolver.cpp:210-232).
static int  g_floor_default = 1;
static long g_passive_floor = 0L;
static int  g_nnorm = 0, g_norm_idx[8];
static int  g_nfrac = 0, g_frac_idx[8];
static int  g_jeans = 0;
static double g_jeans_coeff = 0.0;

__attribute__((visibility("default")))
int gref_set_options( const int floor_default, const long passive_floor, const int nnorm, const int *norm_idx,
                      const int nfrac, const int *frac_idx, const int jeans, const double jeans_coeff )
{
   if ( nnorm < 0 || nnorm > 8 || nfrac < 0 || nfrac > 8 )  return 1;
   g_floor_default = floor_default;
   g_passive_floor = passive_floor;
   g_nnorm = nnorm;
   for (int v=0; v<nnorm; v++)   g_norm_idx[v] = norm_idx[v];
   g_nfrac = nfrac;
   for (int v=0; v<nfrac; v++)   g_frac_idx[v] = frac_idx[v];
   g_jeans = jeans;
   g_jeans_coeff = jeans_coeff;
   return 0;
}

// Advance NPG patch groups by dt with CPU_FluidSolver().  Array shapes follow the reference:
//    flu_in [NPG][NCOMP_TOTAL][FLU_NXT^3]            flu_out[NPG][NCOMP_TOTAL][PS2^3]
//    mag_in [NPG][3][(FLU_NXT+1)*FLU_NXT^2]          mag_out[NPG][3][(PS2+1)*PS2^2]      (MHD)
//    de_out [NPG][PS2^3]  (char)                     flux   [NPG][9][NCOMP_TOTAL][PS2^2]
//    ele    [NPG][9][NCOMP_ELE][(PS2+1)*PS2]          (MHD)
// Unused arrays may be NULL.  Returns 0.
__attribute__((visibility("default")))
int gref_solve( const void *flu_in, void *flu_out, const void *mag_in, void *mag_out, char *de_out,
                void *flux, void *ele, const int NPG, const double dt, const double dh,
                const int store_flux, const int store_ele, const int lr_limiter,
                const double minmod_coeff, const int minmod_maxiter,
                const double min_dens, const double min_pres, const double min_eint,
                const double de_switch, const double gamma, const int nthreads )
{
   SetEoS( gamma );

   if ( nthreads > 0 )  omp_set_num_threads( nthreads );
   omp_set_schedule( omp_sched_static, 0 );

   const int Chunk = ( NPG < GREF_CHUNK ) ? NPG : GREF_CHUNK;
   AllocScratch( Chunk );

   typedef real FluIn_t  [FLU_NIN ][ CUBE(FLU_NXT) ];
   typedef real FluOut_t [FLU_NOUT][ CUBE(PS2) ];
   typedef real MagIn_t  [NCOMP_MAG][ FLU_NXT_P1*SQR(FLU_NXT) ];
   typedef real MagOut_t [NCOMP_MAG][ PS2P1*SQR(PS2) ];
   typedef char DE_t     [ CUBE(PS2) ];
   typedef real Flux_t   [9][NFLUX_TOTAL][ SQR(PS2) ];
   typedef real Ele_t    [9][NCOMP_ELE][ PS2P1*PS2 ];

   MicroPhy_t MicroPhy;
   MicroPhy.useless = false;

// production registers the dual-energy field with FLOOR_YES (src/Init/Init_Field.cpp:148, :264)
#  ifdef DUAL_ENERGY
   const long PassiveFloor_Default = BIDX( DUAL );
#  else
   const long PassiveFloor_Default = 0L;
#  endif
   const long PassiveFloor = ( g_floor_default ) ? PassiveFloor_Default : g_passive_floor;

   for (int p0=0; p0<NPG; p0+=Chunk)
   {
      const int n = ( NPG - p0 < Chunk ) ? NPG - p0 : Chunk;
      CPU_FluidSolver( (FluIn_t  *)flu_in  + p0, (FluOut_t *)flu_out + p0,
                       ( mag_in  == NULL ) ? NULL : (MagIn_t  *)mag_in  + p0,
                       ( mag_out == NULL ) ? NULL : (MagOut_t *)mag_out + p0,
                       ( de_out  == NULL ) ? NULL : (DE_t     *)de_out  + p0,
                       ( flux    == NULL ) ? NULL : (Flux_t   *)flux    + p0,
                       ( ele     == NULL ) ? NULL : (Ele_t    *)ele     + p0,
                       NULL, NULL, NULL, NULL, NULL,
                       n, (real)dt, (real)dh, store_flux != 0, store_ele != 0, false,
                       (LR_Limiter_t)lr_limiter, (real)minmod_coeff, minmod_maxiter,
                       NULL_REAL, NULL_REAL, false, 0.0, false, EXT_ACC_NONE, MicroPhy,
                       (real)min_dens, (real)min_pres, (real)min_eint, (real)de_switch,
                       PassiveFloor, g_nnorm > 0, g_nnorm, g_norm_idx, g_nfrac > 0, g_nfrac, g_frac_idx,
                       g_jeans != 0, (real)g_jeans_coeff, false );
   }
   return 0;
}

// dt of 8*NPG patches: flu [8*NPG][FLU_NIN_T][PS1^3], mag [8*NPG][3][(PS1+1)*PS1^2] (MHD), dt [8*NPG]
__attribute__((visibility("default")))
int gref_dt( const void *flu, const void *mag, void *dt, const int NPG, const double dh, const double safety,
             const double min_pres, const double gamma, const int nthreads )
{
   SetEoS( gamma );
   if ( nthreads > 0 )  omp_set_num_threads( nthreads );
   MicroPhy_t MicroPhy;
   MicroPhy.useless = false;
   typedef real Flu_t[FLU_NIN_T][ CUBE(PS1) ];
   typedef real Mag_t[NCOMP_MAG][ PS1P1*SQR(PS1) ];
   CPU_dtSolver_HydroCFL( (real*)dt, (const Flu_t*)flu, (const Mag_t*)mag, NPG, (real)dh, (real)safety,
                          (real)min_pres, 0L, EoS, MicroPhy );
   return 0;
}

} // extern "C"
