// Coarse-fine flux fix-up on the device: Flu_FixUp_Flux of src/Fluid/Flu_FixUp_Flux.cpp:23-400
// (gamma-law EoS; hydro, or MHD with the patches' face-centred field), on a batch of patches of one
// level held in device memory.
//
// Flu_FixUp_Flux corrects the layer of cells along every face of a coarse patch that borders finer
// patches, with the difference between the coarse flux and the sum of the fine fluxes through that
// face (patch_t::flux[s], accumulated by StoreFlux / CorrectFlux of Flu_Close).  One thread per cell
// of a patch: a cell on no face that carries a flux difference returns at once.  A cell on several
// such faces (an edge or a corner of the patch) applies them in the reference's order s = 0..5,
// each on the state the previous one left, so every cell's result depends only on its own data and
// the threads need no synchronisation.  Per face, exactly as the reference:
//   CorrVal = U + F[s] * (-1/dh, +1/dh for s even / odd) on the variables of the mask tvar;
//   internal energy and pressure from E - K (or from the dual-energy field where the cell's
//   dual-energy status says the total energy was not used);
//   the correction applies only if density, internal energy and pressure stay above their floors
//   and finite (and the dual-energy field above 2*TINY_NUMBER where it was used); then the total
//   energy is rebuilt from that internal energy and the dual-energy field from its pressure.
// With MHD the internal energy also subtracts, and the rebuilt total energy adds, the cell's
// magnetic energy 0.5 B^2 of the cell-centred field (MHD_GetCellCenteredBEnergyInPatch,
// src/Model_Hydro/MHD_GetCellCenteredBInPatch.cpp), which the fix-up does not change.
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "mhd_physics.cuh"

namespace gb {
namespace {

constexpr int FX_CELLS  = PS1*PS1*PS1;
constexpr int FX_THREADS = 256;
constexpr char DE_BY_MIN_PRES_C = '2';     // DE_UPDATED_BY_MIN_PRES, include/Macro.h:99
constexpr char DE_BY_ETOT_GRA_C = '3';     // DE_UPDATED_BY_ETOT_GRA, include/Macro.h:100

template <typename R>
struct FixArgs {
   R *fluid;  const char *de;  const R *flux;  const unsigned char *has_flux;
   const R *magnetic;           // MHD: [npatch][3][(PS1+1)*PS1^2]
   long npatch;
   long tvar;
   R    cst[6];                 // Const[s] of the reference: real( -+1.0/dh )
   Phys<R> ph;
};

template <typename R> GB_DEV bool fin( R x ) { return isfinite( x ); }

template <typename R, int P, int NC, bool MHD>
__global__ void __launch_bounds__(FX_THREADS) flux_fixup_kernel( const FixArgs<R> a )
{
   const long t = (long)blockIdx.x*FX_THREADS + threadIdx.x;
   const long p = t/FX_CELLS;
   if ( p >= a.npatch ) return;
   const int cell = (int)( t % FX_CELLS );
   const int i = cell % PS1, j = ( cell/PS1 ) % PS1, k = cell/( PS1*PS1 );
   const unsigned char *hf = a.has_flux + 6*p;
   const bool on[6] = { i == 0 && hf[0], i == PS1-1 && hf[1], j == 0 && hf[2], j == PS1-1 && hf[3],
                        k == 0 && hf[4], k == PS1-1 && hf[5] };
   if ( !( on[0] || on[1] || on[2] || on[3] || on[4] || on[5] ) ) return;

   R *fl = a.fluid + p*NC*FX_CELLS + cell;
   R u[NC];
#  pragma unroll
   for (int v=0; v<NC; v++) u[v] = fl[ v*FX_CELLS ];
   const char st = ( NC > 5 && a.de != nullptr ) ? a.de[ p*FX_CELLS + cell ] : DE_BY_ETOT;
   const Phys<R> &ph = a.ph;
   R emag = R(0);
   if constexpr ( MHD )
   {
      // 0.5 B^2 of the cell-centred field (MHD_GetCellCenteredBField on the patch's PS1^3 cells)
      constexpr long NB = (long)( PS1 + 1 )*PS1*PS1;
      const R *bx = a.magnetic + p*3*NB, *by = bx + NB, *bz = by + NB;
      const int ix = ( k*PS1 + j )*( PS1 + 1 ) + i, iy = ( k*( PS1 + 1 ) + j )*PS1 + i, iz = cell;
      const R b0 = R(0.5)*( bx[ix] + bx[ ix + 1 ] );
      const R b1 = R(0.5)*( by[iy] + by[ iy + PS1 ] );
      const R b2 = R(0.5)*( bz[iz] + bz[ iz + PS1*PS1 ] );
      emag = R(0.5)*( b0*b0 + b1*b1 + b2*b2 );
   }

   for (int s=0; s<6; s++)
   {
      if ( !on[s] ) continue;
      const int m = ( s < 4 ) ? k : j;                  // didx[s/2]: x faces (k, j), y (k, i), z (j, i)
      const int n = ( s < 2 ) ? j : i;
      const R *F = a.flux + ( p*6 + s )*NC*PS1*PS1 + m*PS1 + n;
      R c[NC];
#     pragma unroll
      for (int v=0; v<NC; v++) c[v] = ( a.tvar & ( 1L << v ) ) ? u[v] + F[ v*PS1*PS1 ]*a.cst[s] : u[v];

      R eint, pres;
      bool by_dual = false;
      if constexpr ( NC > 5 ) by_dual = !( st == DE_BY_ETOT || st == DE_BY_ETOT_GRA_C );
      if ( by_dual )
      {
         pres = c[NC-1]*gpow( c[0], ph.gm1 );                          // Hydro_DensDual2Pres
         eint = pres*ph.inv_gm1;                                       // EoS_DensPres2Eint
      }
      else
      {
         eint = c[4] - R(0.5)*( c[1]*c[1] + c[2]*c[2] + c[3]*c[3] )/c[0];   // Hydro_Con2Eint
         if constexpr ( MHD ) eint -= emag;
         pres = eint*ph.gm1;                                                // EoS_DensEint2Pres
      }
      bool bad = c[0] <= ph.min_dens || eint <= ph.min_eint || !fin( eint ) || pres <= ph.min_pres || !fin( pres );
      if constexpr ( NC > 5 )
         bad |= ( st == DE_BY_DUAL || st == DE_BY_MIN_PRES_C ) && c[5] <= R(2)*Lim<R>::tiny();
      if ( bad ) continue;

      if constexpr ( NC > 5 )
         if ( a.tvar & ( 1L << 5 ) ) c[5] = gmax( c[5], Lim<R>::tiny() );            // passive floor
      c[4] = R(0.5)*( c[1]*c[1] + c[2]*c[2] + c[3]*c[3] )/c[0] + eint;               // Hydro_ConEint2Etot
      if constexpr ( MHD ) c[4] += emag;
      if constexpr ( NC > 5 )
         c[5] = gmax( ( eint*ph.gm1 )*gpow( c[0], -ph.gm1 ), Lim<R>::tiny() );        // Hydro_DensPres2Dual
#     pragma unroll
      for (int v=0; v<NC; v++) if ( a.tvar & ( 1L << v ) ) u[v] = c[v];
   }
#  pragma unroll
   for (int v=0; v<NC; v++) fl[ v*FX_CELLS ] = u[v];
}

template <typename R, int P>
int fixup_run( const gb_fluid_config &c, void *fluid, const char *de, const void *flux, const unsigned char *has_flux,
               int npatch, const gb_fluid_params *prm, long tvar, cudaStream_t st, const void *magnetic = nullptr )
{
   FixArgs<R> a;
   a.fluid = (R*)fluid;  a.de = de;  a.flux = (const R*)flux;  a.has_flux = has_flux;
   a.magnetic = (const R*)magnetic;
   a.npatch = npatch;  a.tvar = tvar;
   for (int s=0; s<6; s++) a.cst[s] = (R)( ( s & 1 ) ? +1.0/prm->dh : -1.0/prm->dh );
   a.ph.gamma     = (R)c.gamma;
   a.ph.gm1       = (R)( c.gamma - 1.0 );
   a.ph.inv_gm1   = (R)( 1.0/( c.gamma - 1.0 ) );
   a.ph.min_dens  = (R)prm->min_dens;
   a.ph.min_pres  = (R)prm->min_pres;
   a.ph.min_eint  = (R)prm->min_eint;
   a.ph.de_switch = (R)prm->dual_energy_switch;
   const long nthr = (long)npatch*FX_CELLS;
   const unsigned grid = (unsigned)( ( nthr + FX_THREADS - 1 )/FX_THREADS );
   if      ( magnetic != nullptr )         flux_fixup_kernel<R,P,5,true ><<< grid, FX_THREADS, 0, st >>>( a );
   else if ( c.dual_energy == GB_DE_ENPY ) flux_fixup_kernel<R,P,6,false><<< grid, FX_THREADS, 0, st >>>( a );
   else                                    flux_fixup_kernel<R,P,5,false><<< grid, FX_THREADS, 0, st >>>( a );
   return ( cudaGetLastError() == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

} // namespace
} // namespace gb

extern "C"
int gb_flux_fixup_device( const gb_fluid_config *cfg, void *fluid, const char *de_status, const void *flux,
                          const unsigned char *has_flux, int npatch, const gb_fluid_params *prm, long tvar,
                          void *stream )
{
   using namespace gb;
   if ( cfg == nullptr || prm == nullptr ) return GB_E_INVALID;
   const gb_fluid_config c = *cfg;
   if ( c.scheme == GB_SCHEME_CTU && c.rsolver == GB_RSOLVER_HLLD ) return GB_E_INVALID;   // MHD: gb_flux_fixup_mhd_device
   if ( c.npassive_user != 0 ) return GB_E_UNSUPPORTED;   // user passive scalars: not built
   if ( c.precision < GB_PREC_FP32 || c.precision > GB_PREC_FP64 || !( c.gamma > 1.0 ) ) return GB_E_INVALID;
   if ( c.dual_energy != GB_DE_NONE && c.dual_energy != GB_DE_ENPY ) return GB_E_INVALID;
   if ( !( prm->dh > 0.0 ) || npatch < 0 ) return GB_E_INVALID;
   if ( npatch == 0 ) return GB_OK;
   if ( fluid == nullptr || flux == nullptr || has_flux == nullptr ) return GB_E_INVALID;
   if ( c.dual_energy == GB_DE_ENPY && de_status == nullptr ) return GB_E_INVALID;
   const cudaStream_t st = (cudaStream_t)stream;
   if ( c.precision == GB_PREC_FP64 ) return fixup_run<double,P_FP64>( c, fluid, de_status, flux, has_flux, npatch, prm, tvar, st );
   if ( c.precision == GB_PREC_MIXED ) return fixup_run<float,P_MIXED>( c, fluid, de_status, flux, has_flux, npatch, prm, tvar, st );
   return fixup_run<float,P_FP32>( c, fluid, de_status, flux, has_flux, npatch, prm, tvar, st );
}

extern "C"
int gb_flux_fixup_mhd_device( const gb_fluid_config *cfg, void *fluid, const void *magnetic, const void *flux,
                              const unsigned char *has_flux, int npatch, const gb_fluid_params *prm, long tvar,
                              void *stream )
{
   using namespace gb;
   if ( cfg == nullptr || prm == nullptr ) return GB_E_INVALID;
   const gb_fluid_config c = *cfg;
   if ( !( c.scheme == GB_SCHEME_CTU && c.rsolver == GB_RSOLVER_HLLD ) ) return GB_E_INVALID;   // MHD solvers only
   if ( c.precision < GB_PREC_FP32 || c.precision > GB_PREC_FP64 || !( c.gamma > 1.0 ) ) return GB_E_INVALID;
   if ( c.dual_energy != GB_DE_NONE || c.npassive_user != 0 ) return GB_E_UNSUPPORTED;
   if ( !( prm->dh > 0.0 ) || npatch < 0 ) return GB_E_INVALID;
   if ( npatch == 0 ) return GB_OK;
   if ( fluid == nullptr || magnetic == nullptr || flux == nullptr || has_flux == nullptr ) return GB_E_INVALID;
   const cudaStream_t st = (cudaStream_t)stream;
   if ( c.precision == GB_PREC_FP64 )
      return fixup_run<double,P_FP64>( c, fluid, nullptr, flux, has_flux, npatch, prm, tvar, st, magnetic );
   if ( c.precision == GB_PREC_MIXED )
      return fixup_run<float,P_MIXED>( c, fluid, nullptr, flux, has_flux, npatch, prm, tvar, st, magnetic );
   return fixup_run<float,P_FP32>( c, fluid, nullptr, flux, has_flux, npatch, prm, tvar, st, magnetic );
}
