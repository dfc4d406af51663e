// Coarse-fine electric-field fix-up on the device: MHD_FixUp_Electric of
// src/Model_Hydro/MHD_FixUp_Electric.cpp:22-250, on a batch of patches of one level held in device
// memory, with BIT_REP_ELECTRIC (always on in MHD builds, include/Macro.h:935-942).
//
// On every side of a coarse patch that borders finer patches, the electric field there (the sum of
// patch_t::electric and patch_t::electric_bitrep, which StoreElectric and CorrectElectric of
// Flu_Close leave as the difference between the coarse and the fine line integrals) corrects the
// transverse components of the patch's face-centred B:
//   face s (0..5, normal xyz = s/2, side LR = s%2): B_(xyz+2)%3 += C*E[0] and B_(xyz+1)%3 -= C*E[1] on
//   the faces of the cell layer next to the patch face, C = (2 LR - 1)/dh, the faces on the patch
//   edges excluded;
//   edge s (6..17): the two components normal to the edge on the faces along it, only where the
//   sibling patch across that face is a leaf or the non-periodic domain boundary (the faces
//   bordering a finer sibling are set by Flu_FixUp_Restrict).
// One thread per B component of a patch (3 x 9 x 8 x 8): it gathers the corrections that reach it in
// the reference's order (the six faces, then the twelve edges), each product rounded before it is
// added, so the result is the reference's bit for bit.  Both electric arrays are zeroed afterwards,
// as the reference leaves them.
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "gb_common.cuh"

namespace gb {
namespace {

constexpr int EF_THREADS = 256;
constexpr int NB1        = ( PS1 + 1 )*PS1*PS1;     // one face-centred component of a patch
constexpr int NBP        = 3*NB1;                   // the three components
constexpr int EFACE      = ( PS1 - 1 )*PS1;         // one of the two E components on a patch face
constexpr int EDGE0      = 6*2*EFACE;               // offset of the first edge in the packed sides
static_assert( GB_ELE_PER_PATCH == EDGE0 + 12*PS1, "packed electric-field layout" );

template <typename R>
struct EleArgs {
   R *mag;  const R *ele;  const R *ele_b;
   const unsigned char *has;    // [npatch][18]
   const unsigned char *sib;    // [npatch][6]
   long npatch;
   R    idh;                    // (real)( 1/dh )
};

// E of side s at element t: electric + electric_bitrep (step 1 of the reference)
template <typename R>
GB_DEV R ele_at( const EleArgs<R> &a, long p, int off )
{
   const long q = p*GB_ELE_PER_PATCH + off;
   return a.ele[q] + a.ele_b[q];
}

template <typename R>
__global__ void __launch_bounds__(EF_THREADS) ele_fixup_kernel( const EleArgs<R> a )
{
   const long t = (long)blockIdx.x*EF_THREADS + threadIdx.x;
   const long p = t/NBP;
   if ( p >= a.npatch ) return;
   const int e = (int)( t % NBP );
   const int c = e/NB1, r = e % NB1;
   int i, j, k;
   if      ( c == 0 ) { i = r % ( PS1 + 1 );  j = ( r/( PS1 + 1 ) ) % PS1;  k = r/( ( PS1 + 1 )*PS1 ); }
   else if ( c == 1 ) { i = r % PS1;  j = ( r/PS1 ) % ( PS1 + 1 );  k = r/( PS1*( PS1 + 1 ) ); }
   else               { i = r % PS1;  j = ( r/PS1 ) % PS1;          k = r/( PS1*PS1 ); }
   const unsigned char *has = a.has + 18*p;
   const unsigned char *sib = a.sib + 6*p;
   const R idh = a.idh;
   constexpr int M1 = PS1 - 1;

   R   b = R(0);
   bool touched = false;
   // b += sgn/dh * E, the product rounded on its own
   auto add = [&]( R sgn, R E ) {
      if ( !touched ) { b = a.mag[ p*NBP + e ];  touched = true; }
      b = b + mul_rn( sgn*idh, E );
   };

   if ( c == 0 )          // Bx [k][j][i], i in [0, PS1]
   {
      // faces 2, 3 (normal y, B1 = Bx): j = M1*LR, i in [1, PS1), E[0][(i-1)*PS1 + k]
      for (int LR=0; LR<2; LR++)
         if ( has[ 2 + LR ] && j == M1*LR && i >= 1 && i < PS1 )
            add( R( 2*LR - 1 ), ele_at( a, p, ( 2 + LR )*2*EFACE + ( i - 1 )*PS1 + k ) );
      // faces 4, 5 (normal z, B2 = Bx): k = M1*LR, i in [1, PS1), -E[1][j*M1 + i-1]
      for (int LR=0; LR<2; LR++)
         if ( has[ 4 + LR ] && k == M1*LR && i >= 1 && i < PS1 )
            add( -R( 2*LR - 1 ), ele_at( a, p, ( 4 + LR )*2*EFACE + EFACE + j*M1 + ( i - 1 ) ) );
      // edges 0-3 (along z, B1 = Bx): i = PS1*LR1, j = M1*LR2, t = k, sibling 0+LR1, C1 = 2 LR2 - 1
      for (int q=0; q<4; q++)
      {
         const int LR1 = q % 2, LR2 = q/2;
         if ( has[ 6 + q ] && i == PS1*LR1 && j == M1*LR2 && sib[ LR1 ] )
            add( R( 2*LR2 - 1 ), ele_at( a, p, EDGE0 + q*PS1 + k ) );
      }
      // edges 8-11 (along y, B2 = Bx): i = PS1*LR2, k = M1*LR1, t = j, sibling 0+LR2, C2 = 1 - 2 LR1
      for (int q=8; q<12; q++)
      {
         const int LR1 = q % 2, LR2 = ( q % 4 )/2;
         if ( has[ 6 + q ] && i == PS1*LR2 && k == M1*LR1 && sib[ LR2 ] )
            add( R( 1 - 2*LR1 ), ele_at( a, p, EDGE0 + q*PS1 + j ) );
      }
   }
   else if ( c == 1 )     // By [k][j][i], j in [0, PS1]
   {
      // faces 0, 1 (normal x, B2 = By): i = M1*LR, j in [1, PS1), -E[1][k*M1 + j-1]
      for (int LR=0; LR<2; LR++)
         if ( has[ LR ] && i == M1*LR && j >= 1 && j < PS1 )
            add( -R( 2*LR - 1 ), ele_at( a, p, LR*2*EFACE + EFACE + k*M1 + ( j - 1 ) ) );
      // faces 4, 5 (normal z, B1 = By): k = M1*LR, j in [1, PS1), E[0][(j-1)*PS1 + i]
      for (int LR=0; LR<2; LR++)
         if ( has[ 4 + LR ] && k == M1*LR && j >= 1 && j < PS1 )
            add( R( 2*LR - 1 ), ele_at( a, p, ( 4 + LR )*2*EFACE + ( j - 1 )*PS1 + i ) );
      // edges 0-3 (along z, B2 = By): i = M1*LR1, j = PS1*LR2, t = k, sibling 2+LR2, C2 = 1 - 2 LR1
      for (int q=0; q<4; q++)
      {
         const int LR1 = q % 2, LR2 = q/2;
         if ( has[ 6 + q ] && i == M1*LR1 && j == PS1*LR2 && sib[ 2 + LR2 ] )
            add( R( 1 - 2*LR1 ), ele_at( a, p, EDGE0 + q*PS1 + k ) );
      }
      // edges 4-7 (along x, B1 = By): j = PS1*LR1, k = M1*LR2, t = i, sibling 2+LR1, C1 = 2 LR2 - 1
      for (int q=4; q<8; q++)
      {
         const int LR1 = q % 2, LR2 = ( q % 4 )/2;
         if ( has[ 6 + q ] && j == PS1*LR1 && k == M1*LR2 && sib[ 2 + LR1 ] )
            add( R( 2*LR2 - 1 ), ele_at( a, p, EDGE0 + q*PS1 + i ) );
      }
   }
   else                   // Bz [k][j][i], k in [0, PS1]
   {
      // faces 0, 1 (normal x, B1 = Bz): i = M1*LR, k in [1, PS1), E[0][(k-1)*PS1 + j]
      for (int LR=0; LR<2; LR++)
         if ( has[ LR ] && i == M1*LR && k >= 1 && k < PS1 )
            add( R( 2*LR - 1 ), ele_at( a, p, LR*2*EFACE + ( k - 1 )*PS1 + j ) );
      // faces 2, 3 (normal y, B2 = Bz): j = M1*LR, k in [1, PS1), -E[1][i*M1 + k-1]
      for (int LR=0; LR<2; LR++)
         if ( has[ 2 + LR ] && j == M1*LR && k >= 1 && k < PS1 )
            add( -R( 2*LR - 1 ), ele_at( a, p, ( 2 + LR )*2*EFACE + EFACE + i*M1 + ( k - 1 ) ) );
      // edges 4-7 (along x, B2 = Bz): j = M1*LR1, k = PS1*LR2, t = i, sibling 4+LR2, C2 = 1 - 2 LR1
      for (int q=4; q<8; q++)
      {
         const int LR1 = q % 2, LR2 = ( q % 4 )/2;
         if ( has[ 6 + q ] && j == M1*LR1 && k == PS1*LR2 && sib[ 4 + LR2 ] )
            add( R( 1 - 2*LR1 ), ele_at( a, p, EDGE0 + q*PS1 + i ) );
      }
      // edges 8-11 (along y, B1 = Bz): k = PS1*LR1, i = M1*LR2, t = j, sibling 4+LR1, C1 = 2 LR2 - 1
      for (int q=8; q<12; q++)
      {
         const int LR1 = q % 2, LR2 = ( q % 4 )/2;
         if ( has[ 6 + q ] && k == PS1*LR1 && i == M1*LR2 && sib[ 4 + LR1 ] )
            add( R( 2*LR2 - 1 ), ele_at( a, p, EDGE0 + q*PS1 + j ) );
      }
   }
   if ( touched ) a.mag[ p*NBP + e ] = b;
}

template <typename R>
int ele_fixup_run( void *mag, void *ele, void *ele_b, const unsigned char *has, const unsigned char *sib, int npatch,
                   double dh, cudaStream_t st )
{
   EleArgs<R> a;
   a.mag = (R*)mag;  a.ele = (const R*)ele;  a.ele_b = (const R*)ele_b;  a.has = has;  a.sib = sib;
   a.npatch = npatch;
   a.idh = (R)( 1.0/dh );
   const long nthr = (long)npatch*NBP;
   ele_fixup_kernel<R><<< (unsigned)( ( nthr + EF_THREADS - 1 )/EF_THREADS ), EF_THREADS, 0, st >>>( a );
   if ( cudaGetLastError() != cudaSuccess ) return GB_E_CUDA;
   // step 4 of the reference: both electric arrays back to zero once the field is corrected
   const size_t bytes = (size_t)npatch*GB_ELE_PER_PATCH*sizeof(R);
   if ( cudaMemsetAsync( ele, 0, bytes, st ) != cudaSuccess ) return GB_E_CUDA;
   if ( cudaMemsetAsync( ele_b, 0, bytes, st ) != cudaSuccess ) return GB_E_CUDA;
   return GB_OK;
}

} // namespace
} // namespace gb

extern "C"
int gb_mhd_fixup_electric_device( const gb_fluid_config *cfg, void *magnetic, void *electric, void *electric_bitrep,
                                  const unsigned char *has_ele, const unsigned char *sib_leaf, int npatch, double dh,
                                  void *stream )
{
   using namespace gb;
   if ( cfg == nullptr ) return GB_E_INVALID;
   if ( !( cfg->scheme == GB_SCHEME_CTU && cfg->rsolver == GB_RSOLVER_HLLD ) ) return GB_E_INVALID;   // MHD only
   if ( cfg->precision < GB_PREC_FP32 || cfg->precision > GB_PREC_FP64 ) return GB_E_INVALID;
   if ( !( dh > 0.0 ) || npatch < 0 ) return GB_E_INVALID;
   if ( npatch == 0 ) return GB_OK;
   if ( magnetic == nullptr || electric == nullptr || electric_bitrep == nullptr || has_ele == nullptr ||
        sib_leaf == nullptr ) return GB_E_INVALID;
   const cudaStream_t st = (cudaStream_t)stream;
   if ( cfg->precision == GB_PREC_FP64 )
      return ele_fixup_run<double>( magnetic, electric, electric_bitrep, has_ele, sib_leaf, npatch, dh, st );
   return ele_fixup_run<float>( magnetic, electric, electric_bitrep, has_ele, sib_leaf, npatch, dh, st );
}
