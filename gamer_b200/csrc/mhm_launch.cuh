// Launch wrapper and registry of the MHM kernel instantiations.
#pragma once
#include "mhm_kernel.cuh"

namespace gb {

template <typename R>
using MhmLaunchFn = cudaError_t (*)( const MhmArgs<R> &, int block, int ctas_per_sm, cudaStream_t, int *grid_used );

// Launch one instantiation: dynamic shared memory from mhm_layout, persistent grid sized by the
// occupancy calculator (CTAs stride over patch groups), at most ctas_per_sm CTAs per SM if > 0.
template <typename R, int P, int LR, int RS, int NC, int NIN, int LIMK, int SCH = SCH_MHM, int REG = 0>
cudaError_t mhm_launch( const MhmArgs<R> &a, int block, int ctas_per_sm, cudaStream_t st, int *grid_used )
{
   typedef typename std::conditional<P == P_MIXED, double, R>::type A;
   typedef typename std::conditional<P == P_MIXED && NC == 5 && LR == LR_PLM, double, R>::type FP;
   const MhmLayout lay = mhm_layout( sizeof(R), sizeof(A), sizeof(FP), NC, a.nin, LR, mhm_carry_smem( P, NC ),
                                     mhm_conv_in_a( P, LR, NC, SCH ) );
   const void *fn = (const void*)mhm_kernel<R,P,LR,RS,NC,NIN,LIMK,SCH,REG>;
   int dev = 0, nsm = 0, per_sm = 0, smem_optin = 0;
   cudaGetDevice( &dev );
   cudaDeviceGetAttribute( &nsm, cudaDevAttrMultiProcessorCount, dev );
   cudaDeviceGetAttribute( &smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev );
   // a configuration whose plane buffers do not fit one SM's shared memory is not supported
   if ( lay.total > smem_optin ) return cudaErrorNotSupported;
   cudaFuncAttributes fa;
   cudaError_t err = cudaFuncGetAttributes( &fa, fn );
   if ( err != cudaSuccess ) return err;
   if ( block > fa.maxThreadsPerBlock ) block = fa.maxThreadsPerBlock & ~31;
   if ( block < MHM_MIN_BLOCK ) return cudaErrorInvalidConfiguration;
   err = cudaFuncSetAttribute( fn, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.total );
   if ( err != cudaSuccess ) return err;
   err = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, fn, block, lay.total );
   if ( err != cudaSuccess ) return err;
   if ( per_sm < 1 ) return cudaErrorInvalidConfiguration;
   if ( ctas_per_sm > 0 && ctas_per_sm < per_sm ) per_sm = ctas_per_sm;
   int grid = nsm*per_sm;
   if ( grid > a.npg ) grid = a.npg;
   if ( grid_used != nullptr ) *grid_used = grid;
   if ( grid == 0 ) return cudaSuccess;
   mhm_kernel<R,P,LR,RS,NC,NIN,LIMK,SCH,REG><<< grid, block, lay.total, st >>>( a );
   return cudaGetLastError();
}

// registries (one per precision policy, defined in the instantiation units); reg != 0 asks for the
// register-capped variant, which exists for the float policies' MHM + PLM + HLLC, 5 variables,
// FLU_NXT = 20, generalized MinMod built in (the headline kernel), with caps 64, 72, 80 and 128
bool mhm_lookup_fp32 ( int sch, int lr, int rs, int nc, int nin, int limk, int reg, MhmLaunchFn<float>  *fn );
bool mhm_lookup_mixed( int sch, int lr, int rs, int nc, int nin, int limk, int reg, MhmLaunchFn<float>  *fn );
bool mhm_lookup_fp64 ( int sch, int lr, int rs, int nc, int nin, int limk, int reg, MhmLaunchFn<double> *fn );

} // namespace gb

// expands to a lookup function covering PLM/PPM x HLLC/HLLE/ROE/EXACT (EXACT with the run-time
// or the characteristic limiter) x variable set (NC 5/6 with the scheme's own FLU_NXT and FLU_NXT+2; NC 7/8, the two user
// passive scalars without / with the dual-energy field, with the scheme's own FLU_NXT) x limiter kind (generalized MinMod built in, any
// limiter chosen at run time, or, PLM only, any limiter applied to characteristic variables) for
// one policy
#define GB_MHM_PICK_L( R, P, LR, RS, L )                                                            \
   if ( nc == 5 && nin == GB_NMIN(LR)     ) { *fn = mhm_launch<R,P,LR,RS,5,GB_NMIN(LR),L>;     return true; } \
   if ( nc == 6 && nin == GB_NMIN(LR)     ) { *fn = mhm_launch<R,P,LR,RS,6,GB_NMIN(LR),L>;     return true; } \
   if ( nc == 5 && nin == GB_NMIN(LR) + 2 ) { *fn = mhm_launch<R,P,LR,RS,5,GB_NMIN(LR) + 2,L>; return true; } \
   if ( nc == 6 && nin == GB_NMIN(LR) + 2 ) { *fn = mhm_launch<R,P,LR,RS,6,GB_NMIN(LR) + 2,L>; return true; } \
   if ( nc == 7 && nin == GB_NMIN(LR)     ) { *fn = mhm_launch<R,P,LR,RS,7,GB_NMIN(LR),L>;     return true; } \
   if ( nc == 8 && nin == GB_NMIN(LR)     ) { *fn = mhm_launch<R,P,LR,RS,8,GB_NMIN(LR),L>;     return true; }
#define GB_MHM_PICK( R, P, LR, RS )                                                                 \
   if ( limk == LIMK_GMINMOD ) { GB_MHM_PICK_L( R, P, LR, RS, LIMK_GMINMOD ) }                      \
   if ( limk == LIMK_ANY     ) { GB_MHM_PICK_L( R, P, LR, RS, LIMK_ANY ) }
// PLM adds the characteristic-variable limiting (CHAR_RECONSTRUCTION)
#define GB_MHM_PICK_PLM( R, P, RS )                                                                 \
   GB_MHM_PICK( R, P, LR_PLM, RS )                                                                  \
   if ( limk == LIMK_CHAR    ) { GB_MHM_PICK_L( R, P, LR_PLM, RS, LIMK_CHAR ) }
#define GB_NMIN( LR ) ( ( LR ) == gb::LR_PPM ? 22 : 20 )
// PPM adds the characteristic-variable limiting of its slopes for 5 and 6 variables on its own
// FLU_NXT and on the window two cells wider, and for 7 and 8 on its own FLU_NXT
#define GB_MHM_PICK_PPM( R, P, RS )                                                                 \
   GB_MHM_PICK( R, P, LR_PPM, RS )                                                                  \
   if ( limk == LIMK_CHAR && nc == 5 && nin == 22 ) { *fn = mhm_launch<R,P,LR_PPM,RS,5,22,LIMK_CHAR>; return true; } \
   if ( limk == LIMK_CHAR && nc == 6 && nin == 22 ) { *fn = mhm_launch<R,P,LR_PPM,RS,6,22,LIMK_CHAR>; return true; } \
   if ( limk == LIMK_CHAR && nc == 5 && nin == 24 ) { *fn = mhm_launch<R,P,LR_PPM,RS,5,24,LIMK_CHAR>; return true; } \
   if ( limk == LIMK_CHAR && nc == 6 && nin == 24 ) { *fn = mhm_launch<R,P,LR_PPM,RS,6,24,LIMK_CHAR>; return true; } \
   if ( limk == LIMK_CHAR && nc == 7 && nin == 22 ) { *fn = mhm_launch<R,P,LR_PPM,RS,7,22,LIMK_CHAR>; return true; } \
   if ( limk == LIMK_CHAR && nc == 8 && nin == 22 ) { *fn = mhm_launch<R,P,LR_PPM,RS,8,22,LIMK_CHAR>; return true; }

// two user passive scalars (NC 7 / 8) in the MHM_RP full step: the run-time limiter only (the
// generalized MinMod then runs through it)
#define GB_MHM_RP_PICK_PASSIVE( R, P, LR, RS, NV )                                                  \
   if ( limk == LIMK_ANY     && nc == 7 ) { *fn = mhm_launch<R,P,LR,RS,7,NV,LIMK_ANY,SCH_MHM_RP>;     return true; } \
   if ( limk == LIMK_ANY     && nc == 8 ) { *fn = mhm_launch<R,P,LR,RS,8,NV,LIMK_ANY,SCH_MHM_RP>;     return true; }
// the MHM_RP full step: PLM x HLLC/HLLE/ROE x NC 5/6 (the half-step state is 20^3) x limiter kind
// (generalized MinMod built in, any run-time limiter, or any limiter on characteristic variables)
#define GB_MHM_RP_PICK( R, P, RS )                                                                  \
   if ( limk == LIMK_GMINMOD && nc == 5 ) { *fn = mhm_launch<R,P,LR_PLM,RS,5,RP_NV,LIMK_GMINMOD,SCH_MHM_RP>; return true; } \
   if ( limk == LIMK_GMINMOD && nc == 6 ) { *fn = mhm_launch<R,P,LR_PLM,RS,6,RP_NV,LIMK_GMINMOD,SCH_MHM_RP>; return true; } \
   if ( limk == LIMK_ANY     && nc == 5 ) { *fn = mhm_launch<R,P,LR_PLM,RS,5,RP_NV,LIMK_ANY,SCH_MHM_RP>;     return true; } \
   if ( limk == LIMK_ANY     && nc == 6 ) { *fn = mhm_launch<R,P,LR_PLM,RS,6,RP_NV,LIMK_ANY,SCH_MHM_RP>;     return true; } \
   if ( limk == LIMK_CHAR    && nc == 5 ) { *fn = mhm_launch<R,P,LR_PLM,RS,5,RP_NV,LIMK_CHAR,SCH_MHM_RP>;    return true; } \
   if ( limk == LIMK_CHAR    && nc == 6 ) { *fn = mhm_launch<R,P,LR_PLM,RS,6,RP_NV,LIMK_CHAR,SCH_MHM_RP>;    return true; } \
   GB_MHM_RP_PICK_PASSIVE( R, P, LR_PLM, RS, RP_NV )                                                \
   if ( limk == LIMK_CHAR    && nc == 7 ) { *fn = mhm_launch<R,P,LR_PLM,RS,7,RP_NV,LIMK_CHAR,SCH_MHM_RP>;    return true; } \
   if ( limk == LIMK_CHAR    && nc == 8 ) { *fn = mhm_launch<R,P,LR_PLM,RS,8,RP_NV,LIMK_CHAR,SCH_MHM_RP>;    return true; }

// the MHM_RP full step with PPM: x HLLC/HLLE/ROE x NC 5/6 (the half-step state is 22^3) x limiter kind
#define GB_MHM_RP_PICK_PPM( R, P, RS )                                                              \
   if ( limk == LIMK_GMINMOD && nc == 5 ) { *fn = mhm_launch<R,P,LR_PPM,RS,5,RP_NV + 2,LIMK_GMINMOD,SCH_MHM_RP>; return true; } \
   if ( limk == LIMK_GMINMOD && nc == 6 ) { *fn = mhm_launch<R,P,LR_PPM,RS,6,RP_NV + 2,LIMK_GMINMOD,SCH_MHM_RP>; return true; } \
   if ( limk == LIMK_ANY     && nc == 5 ) { *fn = mhm_launch<R,P,LR_PPM,RS,5,RP_NV + 2,LIMK_ANY,SCH_MHM_RP>;     return true; } \
   if ( limk == LIMK_ANY     && nc == 6 ) { *fn = mhm_launch<R,P,LR_PPM,RS,6,RP_NV + 2,LIMK_ANY,SCH_MHM_RP>;     return true; } \
   if ( limk == LIMK_CHAR    && nc == 5 ) { *fn = mhm_launch<R,P,LR_PPM,RS,5,RP_NV + 2,LIMK_CHAR,SCH_MHM_RP>;    return true; } \
   if ( limk == LIMK_CHAR    && nc == 6 ) { *fn = mhm_launch<R,P,LR_PPM,RS,6,RP_NV + 2,LIMK_CHAR,SCH_MHM_RP>;    return true; } \
   GB_MHM_RP_PICK_PASSIVE( R, P, LR_PPM, RS, RP_NV + 2 )                                            \
   if ( limk == LIMK_CHAR    && nc == 7 ) { *fn = mhm_launch<R,P,LR_PPM,RS,7,RP_NV + 2,LIMK_CHAR,SCH_MHM_RP>;    return true; } \
   if ( limk == LIMK_CHAR    && nc == 8 ) { *fn = mhm_launch<R,P,LR_PPM,RS,8,RP_NV + 2,LIMK_CHAR,SCH_MHM_RP>;    return true; }

// the register-capped variants of the headline configuration (float policies)
#define GB_MHM_REG_PICK( R, P )                                                                     \
   if ( reg != 0 )                                                                                 \
   {                                                                                               \
      if ( sch != SCH_MHM || lr != LR_PLM || rs != RS_HLLC || nc != 5 || nin != 20 ||              \
           limk != LIMK_GMINMOD ) return false;                                                    \
      if ( reg == 64  ) { *fn = mhm_launch<R,P,LR_PLM,RS_HLLC,5,20,LIMK_GMINMOD,SCH_MHM,64>;  return true; } \
      if ( reg == 72  ) { *fn = mhm_launch<R,P,LR_PLM,RS_HLLC,5,20,LIMK_GMINMOD,SCH_MHM,72>;  return true; } \
      if ( reg == 80  ) { *fn = mhm_launch<R,P,LR_PLM,RS_HLLC,5,20,LIMK_GMINMOD,SCH_MHM,80>;  return true; } \
      if ( reg == 128 ) { *fn = mhm_launch<R,P,LR_PLM,RS_HLLC,5,20,LIMK_GMINMOD,SCH_MHM,128>; return true; } \
      return false;                                                                                \
   }
#define GB_MHM_NO_REG_PICK( R, P )  if ( reg != 0 ) return false;

#define GB_MHM_REGISTRY( NAME, R, P, REGPICK )                                                     \
namespace gb {                                                                                     \
bool NAME( int sch, int lr, int rs, int nc, int nin, int limk, int reg, MhmLaunchFn<R> *fn )       \
{                                                                                                  \
   REGPICK( R, P )                                                                                 \
   if ( sch == SCH_MHM_RP )                                                                        \
   {                                                                                               \
      if ( lr == LR_PLM && nin == RP_NV )                                                          \
      {                                                                                            \
         if ( rs == RS_HLLC ) { GB_MHM_RP_PICK( R, P, RS_HLLC ) }                                  \
         if ( rs == RS_HLLE ) { GB_MHM_RP_PICK( R, P, RS_HLLE ) }                                  \
         if ( rs == RS_ROE  ) { GB_MHM_RP_PICK( R, P, RS_ROE  ) }                                  \
      }                                                                                            \
      if ( lr == LR_PPM && nin == RP_NV + 2 )                                                      \
      {                                                                                            \
         if ( rs == RS_HLLC ) { GB_MHM_RP_PICK_PPM( R, P, RS_HLLC ) }                              \
         if ( rs == RS_HLLE ) { GB_MHM_RP_PICK_PPM( R, P, RS_HLLE ) }                              \
         if ( rs == RS_ROE  ) { GB_MHM_RP_PICK_PPM( R, P, RS_ROE  ) }                              \
      }                                                                                            \
      return false;                                                                                \
   }                                                                                               \
   if ( lr == LR_PLM && rs == RS_HLLC ) { GB_MHM_PICK_PLM( R, P, RS_HLLC ) }                   \
   if ( lr == LR_PLM && rs == RS_HLLE ) { GB_MHM_PICK_PLM( R, P, RS_HLLE ) }                   \
   if ( lr == LR_PLM && rs == RS_ROE  ) { GB_MHM_PICK_PLM( R, P, RS_ROE  ) }                   \
   if ( lr == LR_PPM && rs == RS_HLLC ) { GB_MHM_PICK_PPM( R, P, RS_HLLC ) }                       \
   if ( lr == LR_PPM && rs == RS_HLLE ) { GB_MHM_PICK_PPM( R, P, RS_HLLE ) }                       \
   if ( lr == LR_PPM && rs == RS_ROE  ) { GB_MHM_PICK_PPM( R, P, RS_ROE  ) }                       \
   if ( lr == LR_PLM && rs == RS_EXACT && limk == LIMK_ANY ) { GB_MHM_PICK_L( R, P, LR_PLM, RS_EXACT, LIMK_ANY ) } \
   if ( lr == LR_PPM && rs == RS_EXACT && limk == LIMK_ANY ) { GB_MHM_PICK_L( R, P, LR_PPM, RS_EXACT, LIMK_ANY ) } \
   if ( lr == LR_PLM && rs == RS_EXACT && limk == LIMK_CHAR ) { GB_MHM_PICK_L( R, P, LR_PLM, RS_EXACT, LIMK_CHAR ) } \
   if ( lr == LR_PPM && rs == RS_EXACT && limk == LIMK_CHAR && nc == 5 && nin == 22 ) { *fn = mhm_launch<R,P,LR_PPM,RS_EXACT,5,22,LIMK_CHAR>; return true; } \
   if ( lr == LR_PPM && rs == RS_EXACT && limk == LIMK_CHAR && nc == 6 && nin == 22 ) { *fn = mhm_launch<R,P,LR_PPM,RS_EXACT,6,22,LIMK_CHAR>; return true; } \
   return false;                                                                                   \
}                                                                                                  \
}
