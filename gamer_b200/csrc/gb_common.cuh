// Shared definitions of the B200 patch-group fluid solver kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <float.h>
#include "../../include/gamer_b200_fluid.h"

#define GB_DEV __device__ __forceinline__

namespace gb {

constexpr int PS1 = 8;            // PATCH_SIZE
constexpr int PS2 = 16;           // patch-group width
constexpr int NFC = PS2 + 2;      // N_FC_VAR of MHM / hydro CTU (include/CUFLU.h:86)
constexpr int NFLX = PS2 + 1;     // faces along the normal direction

// precision policies
//   P_FP32 : float storage, float arithmetic everywhere
//   P_MIXED: float storage and bulk arithmetic; internal-energy recovery E - 1/2 m^2/rho, the
//            dual-energy selection and the flux-difference accumulation into the conserved
//            variables are done in double
//   P_FP64 : double storage and arithmetic (the reference's FLOAT8 build)
enum Prec { P_FP32 = 0, P_MIXED = 1, P_FP64 = 2 };

// limiter ids: include/Typedef.h:184-194 of the reference
enum { LIM_VANLEER = 1, LIM_GMINMOD = 2, LIM_ALBADA = 3, LIM_VL_GMINMOD = 4, LIM_CENTRAL = 6 };
// Riemann solver ids: include/Macro.h of the reference
enum { RS_EXACT = 1, RS_ROE = 2, RS_HLLE = 3, RS_HLLC = 4, RS_HLLD = 5 };
enum { LR_PLM = 1, LR_PPM = 2 };

// the configurations with a magnetic field: HLLD is the MHD solver (with CTU or MHM_RP)
inline bool cfg_mhd( const gb_fluid_config &c ) { return c.rsolver == GB_RSOLVER_HLLD; }

// DE status chars: include/Macro.h:97-99 of the reference
constexpr char DE_BY_ETOT = '0';
constexpr char DE_BY_DUAL = '1';

// kernel status bits (written to the status word by the kernels, read by the host)
enum {
   GB_ST_TMA_TIMEOUT = 1,    // a bulk-copy wait gave up
   GB_ST_UNPHYSICAL  = 2,    // some patch group still had an unphysical cell after all retries
};

template <typename R> struct Lim;
template <> struct Lim<float>  {
   static GB_DEV float tiny() { return FLT_MIN; }
   static GB_DEV float huge() { return FLT_MAX; }
   static GB_DEV float eps()  { return FLT_EPSILON; }
};
template <> struct Lim<double> {
   static GB_DEV double tiny() { return DBL_MIN; }
   static GB_DEV double huge() { return DBL_MAX; }
   static GB_DEV double eps()  { return DBL_EPSILON; }
};

// the scalar under a value type: itself, or the value part of a dual number (dual.cuh)
template <typename R> struct ScalarOf { typedef R type;  static constexpr bool dual = false;  static constexpr int ntan = 0; };

GB_DEV float  gsqrt( float x )  { return sqrtf( x ); }
GB_DEV double gsqrt( double x ) { return sqrt( x ); }
GB_DEV float  gabs( float x )   { return fabsf( x ); }
GB_DEV double gabs( double x )  { return fabs( x ); }
GB_DEV float  gmax( float a, float b )   { return fmaxf( a, b ); }
GB_DEV double gmax( double a, double b ) { return fmax( a, b ); }
GB_DEV float  gmin( float a, float b )   { return fminf( a, b ); }
GB_DEV double gmin( double a, double b ) { return fmin( a, b ); }
GB_DEV float  gpow( float a, float b )   { return powf( a, b ); }
GB_DEV double gpow( double a, double b ) { return pow( a, b ); }

template <typename R> GB_DEV R gsign( R a ) { return ( a < R(0) ) ? R(-1) : R(1); }

// a product rounded on its own (never contracted into a following add): sums that must cancel
// exactly, as in the reference's CPU build (compiled without FMA contraction), use it
GB_DEV float  mul_rn( float a, float b )   { return __fmul_rn( a, b ); }
GB_DEV double mul_rn( double a, double b ) { return __dmul_rn( a, b ); }

// max(x, floor) that keeps a NaN input (Hydro_CheckMinPres/Eint, CPU_Shared_FluUtility.cpp:1170-1206)
template <typename R> GB_DEV R check_floor( R x, R floor ) { return ( x == x ) ? gmax( x, floor ) : x; }

// 1/x in double from a float seed and two Newton steps (relative error ~1e-15); used by the
// mixed-precision recoveries so that they do not pay for a full IEEE double division
GB_DEV double rcp_dd( double x )
{
   double r = (double)__frcp_rn( (float)x );
   r = r*( 2.0 - x*r );
   r = r*( 2.0 - x*r );
   return r;
}

// index of the normal / transverse momentum components for a face normal along D
template <int D> struct Dir {
   static constexpr int n  = 1 + D;
   static constexpr int t1 = 1 + (D + 1) % 3;
   static constexpr int t2 = 1 + (D + 2) % 3;
};

} // namespace gb
