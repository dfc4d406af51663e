// CFL time-step solver: per-patch maximum signal speed -> dt = Safety*dh / max_speed.
//
// Reference: CPU_dtSolver_HydroCFL / CUFLU_dtSolver_HydroCFL
// (src/Model_Hydro/CPU_Hydro/CPU_dtSolver_HydroCFL.cpp:57-233): for every cell of a patch
// (PS1^3 = 512 cells) the speed |v_d| + c_d along x, y, z with c_d the sound speed (hydro) or the
// fast magnetosonic speed along d (MHD, B averaged from the faces); the patch's dt uses the maximum
// over its cells and directions.  The maximum is exact, so the reduction order does not matter.
//
// Two entry points: one on GAMER's dt-solver arrays ([NPATCH][5][8^3], filled by dt_Prepare_Flu),
// and one that reads the fluid solver's own output arrays ([NPG][NCOMP][16^3]) and writes the eight
// patches of each patch group in GAMER's LocalID order (TABLE_02, src/Tables/Table_02.cpp), so the
// next step's dt needs no host-side repacking.
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "hydro_physics.cuh"

namespace gb {

namespace {

constexpr int PS1 = 8;
constexpr int DT_BLOCK = 128;      // 4 cells per thread, one patch per CTA

// offset (in cells) of patch LocalID within its patch group (TABLE_02)
GB_DEV void local_offset( int lid, int &ox, int &oy, int &oz )
{
   ox = ( lid == 1 || lid == 4 || lid == 6 || lid == 7 ) ? PS1 : 0;
   oy = ( lid == 2 || lid == 4 || lid == 5 || lid == 7 ) ? PS1 : 0;
   oz = ( lid == 3 || lid == 5 || lid == 6 || lid == 7 ) ? PS1 : 0;
}

// max over x, y, z of |v_d| + c_d for one cell (CPU_dtSolver_HydroCFL.cpp:111-188)
template <typename R, int P, bool MHD>
GB_DEV R cell_speed( const Phys<R> &ph, R d, R mx, R my, R mz, R e, R bx, R by, R bz )
{
   R emag = R(0), bx2 = R(0), by2 = R(0), bz2 = R(0), b2 = R(0);
   if constexpr ( MHD )
   {
      bx2 = bx*bx;  by2 = by*by;  bz2 = bz*bz;
      b2 = bx2 + by2 + bz2;
      emag = R(0.5)*b2;
   }
   const R ird = R(1)/d;
   const R vx = gabs( mx )*ird, vy = gabs( my )*ird, vz = gabs( mz )*ird;
   R eint;
   if constexpr ( P == P_MIXED )
   {
      const double m2 = (double)mx*(double)mx + (double)my*(double)my + (double)mz*(double)mz;
      eint = (R)( (double)e - 0.5*m2/(double)d - (double)emag );
   }
   else
      eint = e - R(0.5)*( mx*mx + my*my + mz*mz )/d - emag;
   const R pres = check_floor( eint*ph.gm1, ph.min_pres );
   const R a2 = ph.gamma*pres/d;
   R cx, cy, cz;
   if constexpr ( MHD )
   {
      const R cp = b2*ird + a2, cm = b2*ird - a2, cm2 = cm*cm, f = R(4)*a2*ird;
      cx = gsqrt( R(0.5)*( cp + gsqrt( cm2 + f*( by2 + bz2 ) ) ) );
      cy = gsqrt( R(0.5)*( cp + gsqrt( cm2 + f*( bx2 + bz2 ) ) ) );
      cz = gsqrt( R(0.5)*( cp + gsqrt( cm2 + f*( bx2 + by2 ) ) ) );
   }
   else
   {
      cx = gsqrt( a2 );  cy = cx;  cz = cx;
   }
   return gmax( gmax( cx + vx, cy + vy ), cz + vz );
}

// one patch per CTA.  Patch arrays (from_output == 0): fluid [p][5][8^3], B [p][3][9*8*8].  Solver
// outputs (from_output != 0): patch p is LocalID p%8 of patch group p/8 in fluid [pg][ncomp][16^3]
// and B [pg][3][17*16*16].  Face component c at cell (i,j,k) of an n^3 grid: IDX321_BX/BY/BZ.
template <typename R, int P, bool MHD>
__global__ void __launch_bounds__( DT_BLOCK ) dt_cfl_kernel( const R *flu, const R *mag, R *dt, int npatch,
                                                             int from_output, int ncomp, Phys<R> ph, R dh_safety )
{
   const int p = blockIdx.x;
   if ( p >= npatch ) return;
   int n, ox = 0, oy = 0, oz = 0;
   size_t fbase, mbase, vstride;
   if ( from_output )
   {
      n = PS2;
      local_offset( p & 7, ox, oy, oz );
      vstride = (size_t)PS2*PS2*PS2;
      fbase = (size_t)( p >> 3 )*ncomp*vstride;
      mbase = (size_t)( p >> 3 )*3*( PS2 + 1 )*PS2*PS2;
   }
   else
   {
      n = PS1;
      vstride = (size_t)PS1*PS1*PS1;
      fbase = (size_t)p*5*vstride;
      mbase = (size_t)p*3*( PS1 + 1 )*PS1*PS1;
   }
   const size_t mcomp = (size_t)( n + 1 )*n*n;
   R vmax = R(0);
   for (int t = threadIdx.x; t < PS1*PS1*PS1; t += DT_BLOCK)
   {
      const int i = t % PS1 + ox, j = ( t / PS1 ) % PS1 + oy, k = t / ( PS1*PS1 ) + oz;
      const size_t c = fbase + ( (size_t)k*n + j )*n + i;
      R bx = R(0), by = R(0), bz = R(0);
      if constexpr ( MHD )
      {
         // MHD_GetCellCenteredBField (CPU_Shared_FluUtility.cpp:1653-1665)
         const R *m = mag + mbase;
         const size_t ix = ( (size_t)k*n + j )*( n + 1 ) + i;
         const size_t iy = ( (size_t)k*( n + 1 ) + j )*n + i;
         const size_t iz = ( (size_t)k*n + j )*n + i;
         bx = R(0.5)*( m[ix] + m[ix + 1] );
         by = R(0.5)*( m[mcomp + iy] + m[mcomp + iy + n] );
         bz = R(0.5)*( m[2*mcomp + iz] + m[2*mcomp + iz + (size_t)n*n] );
      }
      const R s = cell_speed<R,P,MHD>( ph, flu[c], flu[c + vstride], flu[c + 2*vstride], flu[c + 3*vstride],
                                       flu[c + 4*vstride], bx, by, bz );
      vmax = gmax( s, vmax );
   }
#  pragma unroll
   for (int o = 16; o > 0; o >>= 1) vmax = gmax( vmax, (R)__shfl_xor_sync( 0xffffffffu, vmax, o ) );
   __shared__ R s_max[DT_BLOCK/32];
   if ( ( threadIdx.x & 31 ) == 0 ) s_max[threadIdx.x >> 5] = vmax;
   __syncthreads();
   if ( threadIdx.x == 0 )
   {
      R m = s_max[0];
#     pragma unroll
      for (int w = 1; w < DT_BLOCK/32; w++) m = gmax( m, s_max[w] );
      dt[p] = dh_safety/m;
   }
}

template <typename R, int P>
int launch_dt( const gb_fluid_config &c, const void *flu, const void *mag, void *dt, int npatch, int from_output,
               int ncomp, double dh, double safety, double min_pres, cudaStream_t st )
{
   // EoS_SetAuxArray_Gamma: constants formed in double, then cast
   Phys<R> ph;
   ph.gamma = (R)c.gamma;  ph.gm1 = (R)( c.gamma - 1.0 );  ph.inv_gm1 = (R)( 1.0/( c.gamma - 1.0 ) );
   ph.min_dens = R(0);  ph.min_pres = (R)min_pres;  ph.min_eint = R(0);  ph.de_switch = R(0);
   const R dh_safety = (R)safety*(R)dh;
   if ( cfg_mhd( c ) )
      dt_cfl_kernel<R,P,true><<< npatch, DT_BLOCK, 0, st >>>( (const R*)flu, (const R*)mag, (R*)dt, npatch,
                                                              from_output, ncomp, ph, dh_safety );
   else
      dt_cfl_kernel<R,P,false><<< npatch, DT_BLOCK, 0, st >>>( (const R*)flu, nullptr, (R*)dt, npatch,
                                                               from_output, ncomp, ph, dh_safety );
   return ( cudaGetLastError() == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

int dt_common( const gb_fluid_config *cfg, const void *flu, const void *mag, void *dt, int npatch, int from_output,
               double dh, double safety, double min_pres, void *stream )
{
   if ( cfg == nullptr || npatch < 0 ) return GB_E_INVALID;
   if ( cfg->precision < GB_PREC_FP32 || cfg->precision > GB_PREC_FP64 || !( cfg->gamma > 1.0 ) ) return GB_E_INVALID;
   if ( cfg->scheme != GB_SCHEME_MHM && cfg->scheme != GB_SCHEME_MHM_RP && cfg->scheme != GB_SCHEME_CTU ) return GB_E_INVALID;
   if ( !( dh > 0.0 ) || !( safety > 0.0 ) ) return GB_E_INVALID;
   if ( npatch == 0 ) return GB_OK;
   if ( flu == nullptr || dt == nullptr || ( cfg_mhd( *cfg ) && mag == nullptr ) ) return GB_E_INVALID;
   // variables of the solver outputs: the fluid, the user passive scalars, the dual-energy field
   if ( cfg->npassive_user < 0 || cfg->npassive_user > GB_NPASSIVE_USER ) return GB_E_INVALID;
   const int ncomp = 5 + cfg->npassive_user + ( ( cfg->dual_energy == GB_DE_ENPY ) ? 1 : 0 );
   cudaStream_t st = (cudaStream_t)stream;
   if ( cfg->precision == GB_PREC_FP64 )
      return launch_dt<double,P_FP64>( *cfg, flu, mag, dt, npatch, from_output, ncomp, dh, safety, min_pres, st );
   if ( cfg->precision == GB_PREC_MIXED )
      return launch_dt<float,P_MIXED>( *cfg, flu, mag, dt, npatch, from_output, ncomp, dh, safety, min_pres, st );
   return launch_dt<float,P_FP32>( *cfg, flu, mag, dt, npatch, from_output, ncomp, dh, safety, min_pres, st );
}

} // namespace
} // namespace gb

extern "C" {

int gb_dt_cfl_device( const gb_fluid_config *cfg, const void *flu, const void *mag, void *dt, int npatch,
                      double dh, double safety, double min_pres, void *stream )
{
   return gb::dt_common( cfg, flu, mag, dt, npatch, 0, dh, safety, min_pres, stream );
}

int gb_dt_cfl_from_output_device( const gb_fluid_config *cfg, const void *flu_out, const void *mag_out, void *dt,
                                  int npg, double dh, double safety, double min_pres, void *stream )
{
   if ( npg < 0 || npg > 0x0fffffff ) return GB_E_INVALID;
   return gb::dt_common( cfg, flu_out, mag_out, dt, 8*npg, 1, dh, safety, min_pres, stream );
}

} // extern "C"
