// Coarse-fine flux fix-up on the device: Flu_FixUp_Flux of src/Fluid/Flu_FixUp_Flux.cpp:23-400
// (gamma-law EoS; hydro, or MHD with the patches' face-centred field), on a batch of patches of one
// level held in device memory.
//
// Flu_FixUp_Flux corrects the layer of cells along every face of a coarse patch that borders finer
// patches, with the difference between the coarse flux and the sum of the fine fluxes through that
// face (patch_t::flux[s], accumulated by StoreFlux / CorrectFlux of Flu_Close).  Per face, exactly as
// the reference:
//   CorrVal = U + F[s] * (-1/dh, +1/dh for s even / odd) on the variables of the mask tvar;
//   internal energy and pressure from E - K (or from the dual-energy field where the cell's
//   dual-energy status says the total energy was not used);
//   the correction applies only if density, internal energy and pressure stay above their floors
//   and finite (and the dual-energy field above 2*TINY_NUMBER where it was used); then the total
//   energy is rebuilt from that internal energy and the dual-energy field from its pressure.
// With MHD the internal energy also subtracts, and the rebuilt total energy adds, the cell's
// magnetic energy 0.5 B^2 of the cell-centred field (MHD_GetCellCenteredBEnergyInPatch,
// src/Model_Hydro/MHD_GetCellCenteredBInPatch.cpp), which the fix-up does not change.
//
// One CTA of 128 threads per patch.  A patch with no flux face ends after reading its six flags.
// Otherwise one thread stages the patch's fluid, the flux arrays of its flux faces, its dual-energy
// status and, with MHD, its magnetic field in shared memory with 1-D bulk copies (TMA) on one
// mbarrier; the faces are then corrected in three rounds of two opposite faces (x, then y, then z),
// one thread per face cell, so that a cell on several faces meets them in the reference's order
// s = 0..5, each on the state the previous one left; the rows of the corrected variables that hold
// a corrected cell are written back with 16-byte stores.  Many small CTAs per SM keep enough patches in flight to cover the DRAM latency of the
// flags and of the staging copies.
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "mhd_physics.cuh"
#include "tma.cuh"

namespace gb {
namespace {

constexpr int FX_CELLS   = PS1*PS1*PS1;
constexpr int FX_THREADS = 128;
constexpr int FX_FACE    = PS1*PS1;
constexpr int FX_NB      = 3*( PS1 + 1 )*PS1*PS1;   // face-centred B of a patch
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

// shared-memory layout of one patch: mbarrier, fluid [NC][512], flux [6][NC][64] (faces without a
// flux array left unfilled), magnetic [3][576] (MHD), dual-energy status [512] (NC > 5)
template <typename R, int NC, bool MHD>
struct FixSmem {
   static constexpr int    FLU   = NC*FX_CELLS;
   static constexpr int    FLX   = 6*NC*FX_FACE;
   static constexpr int    MAG   = MHD ? FX_NB : 0;
   static constexpr size_t o_flu = 16;
   static constexpr size_t o_flx = o_flu + FLU*sizeof(R);
   static constexpr size_t o_mag = o_flx + FLX*sizeof(R);
   static constexpr size_t o_de  = o_mag + MAG*sizeof(R);
   static constexpr size_t bytes = o_de + ( NC > 5 ? FX_CELLS : 0 );
};

template <typename R, int P, int NC, bool MHD>
__global__ void __launch_bounds__(FX_THREADS) flux_fixup_kernel( const FixArgs<R> a )
{
   typedef FixSmem<R,NC,MHD> L;
   extern __shared__ __align__(16) unsigned char smem[];
   __shared__ unsigned s_faces;
   uint64_t *bar  = (uint64_t*)smem;
   R        *s_u  = (R*)( smem + L::o_flu );
   R        *s_f  = (R*)( smem + L::o_flx );
   R        *s_b  = (R*)( smem + L::o_mag );
   char     *s_de = (char*)( smem + L::o_de );
   const int  tid = threadIdx.x;
   const long p   = blockIdx.x;

   if ( tid == 0 )
   {
      const unsigned char *hf = a.has_flux + 6*p;
      unsigned m = 0;
      for (int s=0; s<6; s++) if ( hf[s] ) m |= 1u << s;
      s_faces = m;
      if ( m )
      {
         mbar_init( bar, 1 );
         mbar_init_fence();
         uint32_t bytes = L::FLU*sizeof(R) + L::MAG*sizeof(R) + ( NC > 5 ? FX_CELLS : 0 );
         for (int s=0; s<6; s++) if ( m & ( 1u << s ) ) bytes += NC*FX_FACE*sizeof(R);
         mbar_expect_tx( bar, bytes );
         bulk_g2s( s_u, a.fluid + p*L::FLU, L::FLU*sizeof(R), bar );
         for (int s=0; s<6; s++)
            if ( m & ( 1u << s ) ) bulk_g2s( s_f + s*NC*FX_FACE, a.flux + ( p*6 + s )*NC*FX_FACE, NC*FX_FACE*sizeof(R), bar );
         if constexpr ( MHD ) bulk_g2s( s_b, a.magnetic + p*FX_NB, FX_NB*sizeof(R), bar );
         if constexpr ( NC > 5 ) bulk_g2s( s_de, a.de + p*FX_CELLS, FX_CELLS, bar );
      }
   }
   __syncthreads();
   const unsigned m = s_faces;
   if ( m == 0u ) return;
   // the copies complete within microseconds; a wait that gives up leaves the patch unchanged
   if ( !__syncthreads_and( mbar_wait_bounded( bar, 0 ) ) ) return;
   const Phys<R> &ph = a.ph;

   // three rounds, one per direction: in round d the threads 0-63 correct the 64 cells of face 2d,
   // the threads 64-127 those of face 2d+1 (the two faces share no cell); a cell on an edge or a
   // corner of the patch meets its faces in the reference's order s = 0..5, each round reading what
   // the previous one left
   static_assert( FX_THREADS == 2*FX_FACE, "one thread per cell of two opposite faces" );
   for (int d=0; d<3; d++)
   {
      const int s = 2*d + ( tid >> 6 );
      if ( m & ( 1u << s ) )
      {
         const int q  = tid & ( FX_FACE - 1 );
         const int mm = q / PS1, nn = q % PS1;              // element mm*PS1 + nn of the face's flux
         const int side = ( s & 1 )*( PS1 - 1 );
         int i, j, k;                                       // didx[s/2]: x faces (k, j), y (k, i), z (j, i)
         if      ( d == 0 ) { i = side;  j = nn;    k = mm;   }
         else if ( d == 1 ) { i = nn;    j = side;  k = mm;   }
         else               { i = nn;    j = mm;    k = side; }
         const int cell = ( k*PS1 + j )*PS1 + i;

         R u[NC];
#        pragma unroll
         for (int v=0; v<NC; v++) u[v] = s_u[ v*FX_CELLS + cell ];
         const char st = ( NC > 5 ) ? s_de[cell] : DE_BY_ETOT;
         R emag = R(0);
         if constexpr ( MHD )
         {
            // 0.5 B^2 of the cell-centred field (MHD_GetCellCenteredBField on the patch's PS1^3 cells)
            constexpr int NB1 = ( PS1 + 1 )*PS1*PS1;
            const R *bx = s_b, *by = s_b + NB1, *bz = s_b + 2*NB1;
            const int ix = ( k*PS1 + j )*( PS1 + 1 ) + i, iy = ( k*( PS1 + 1 ) + j )*PS1 + i, iz = cell;
            const R b0 = R(0.5)*( bx[ix] + bx[ ix + 1 ] );
            const R b1 = R(0.5)*( by[iy] + by[ iy + PS1 ] );
            const R b2 = R(0.5)*( bz[iz] + bz[ iz + PS1*PS1 ] );
            emag = R(0.5)*( b0*b0 + b1*b1 + b2*b2 );
         }

         const R *F = s_f + s*NC*FX_FACE + q;
         const R cst = ( s & 1 ) ? a.cst[1] : a.cst[0];      // Const[s]: real( -1/dh ), real( +1/dh )
         R c[NC];
#        pragma unroll
         for (int v=0; v<NC; v++) c[v] = ( a.tvar & ( 1L << v ) ) ? u[v] + F[ v*FX_FACE ]*cst : u[v];

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
         if ( !bad )
         {
            if constexpr ( NC > 5 )
               if ( a.tvar & ( 1L << 5 ) ) c[5] = gmax( c[5], Lim<R>::tiny() );            // passive floor
            c[4] = R(0.5)*( c[1]*c[1] + c[2]*c[2] + c[3]*c[3] )/c[0] + eint;               // Hydro_ConEint2Etot
            if constexpr ( MHD ) c[4] += emag;
            if constexpr ( NC > 5 )
               c[5] = gmax( ( eint*ph.gm1 )*gpow( c[0], -ph.gm1 ), Lim<R>::tiny() );        // Hydro_DensPres2Dual
#           pragma unroll
            for (int v=0; v<NC; v++) if ( a.tvar & ( 1L << v ) ) s_u[ v*FX_CELLS + cell ] = c[v];
         }
      }
      __syncthreads();
   }

   // write back the rows (k, j) of the corrected variables that hold a surface cell of a flux face
   constexpr int CH = PS1*(int)sizeof(R)/16;          // 16-byte chunks per row of PS1 cells
   R *g = a.fluid + p*L::FLU;
   for (int q=tid; q<NC*PS1*PS1*CH; q+=FX_THREADS)
   {
      const int v = q/( PS1*PS1*CH ), row = ( q/CH ) % ( PS1*PS1 ), part = q % CH;
      const int k = row/PS1, j = row % PS1;
      if ( !( a.tvar & ( 1L << v ) ) ) continue;
      const bool mod = ( m & 3u ) || ( ( m & 4u ) && j == 0 ) || ( ( m & 8u ) && j == PS1-1 ) ||
                       ( ( m & 16u ) && k == 0 ) || ( ( m & 32u ) && k == PS1-1 );
      if ( !mod ) continue;
      const int off = v*FX_CELLS + row*PS1;
      reinterpret_cast<int4*>( g + off )[part] = reinterpret_cast<const int4*>( s_u + off )[part];
   }
}

template <typename R, int P, int NC, bool MHD>
cudaError_t fixup_launch( const FixArgs<R> &a, cudaStream_t st )
{
   const size_t smem = FixSmem<R,NC,MHD>::bytes;
   cudaError_t err = cudaFuncSetAttribute( flux_fixup_kernel<R,P,NC,MHD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem );
   if ( err != cudaSuccess ) return err;
   flux_fixup_kernel<R,P,NC,MHD><<< (unsigned)a.npatch, FX_THREADS, smem, st >>>( a );
   return cudaGetLastError();
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
   cudaError_t err;
   if      ( magnetic != nullptr )         err = fixup_launch<R,P,5,true >( a, st );
   else if ( c.dual_energy == GB_DE_ENPY ) err = fixup_launch<R,P,6,false>( a, st );
   else                                    err = fixup_launch<R,P,5,false>( a, st );
   return ( err == cudaSuccess ) ? GB_OK : GB_E_CUDA;
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
   if ( cfg_mhd( c ) ) return GB_E_INVALID;   // MHD: gb_flux_fixup_mhd_device
   if ( c.npassive_user != 0 ) return GB_E_UNSUPPORTED;   // user passive scalars: not built
   if ( c.precision < GB_PREC_FP32 || c.precision > GB_PREC_FP64 || !( c.gamma > 1.0 ) ) return GB_E_INVALID;
   if ( c.dual_energy != GB_DE_NONE && c.dual_energy != GB_DE_ENPY ) return GB_E_INVALID;
   if ( !( prm->dh > 0.0 ) || npatch < 0 ) return GB_E_INVALID;
   if ( npatch == 0 ) return GB_OK;
   if ( fluid == nullptr || flux == nullptr || has_flux == nullptr ) return GB_E_INVALID;
   if ( c.dual_energy == GB_DE_ENPY && de_status == nullptr ) return GB_E_INVALID;
   // the bulk copies move whole patches: 16-byte aligned bases
   if ( ( (uintptr_t)fluid | (uintptr_t)flux | (uintptr_t)de_status ) & 15u ) return GB_E_ALIGN;
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
   if ( !cfg_mhd( c ) ) return GB_E_INVALID;   // MHD solvers only
   if ( c.precision < GB_PREC_FP32 || c.precision > GB_PREC_FP64 || !( c.gamma > 1.0 ) ) return GB_E_INVALID;
   if ( c.dual_energy != GB_DE_NONE || c.npassive_user != 0 ) return GB_E_UNSUPPORTED;
   if ( !( prm->dh > 0.0 ) || npatch < 0 ) return GB_E_INVALID;
   if ( npatch == 0 ) return GB_OK;
   if ( fluid == nullptr || magnetic == nullptr || flux == nullptr || has_flux == nullptr ) return GB_E_INVALID;
   if ( ( (uintptr_t)fluid | (uintptr_t)magnetic | (uintptr_t)flux ) & 15u ) return GB_E_ALIGN;
   const cudaStream_t st = (cudaStream_t)stream;
   if ( c.precision == GB_PREC_FP64 )
      return fixup_run<double,P_FP64>( c, fluid, nullptr, flux, has_flux, npatch, prm, tvar, st, magnetic );
   if ( c.precision == GB_PREC_MIXED )
      return fixup_run<float,P_MIXED>( c, fluid, nullptr, flux, has_flux, npatch, prm, tvar, st, magnetic );
   return fixup_run<float,P_FP32>( c, fluid, nullptr, flux, has_flux, npatch, prm, tvar, st, magnetic );
}
