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
// One CTA of 128 threads per patch.  A patch with no side on a coarse-fine boundary ends after
// reading its flags.  Otherwise one thread stages the patch's B and both electric arrays in shared
// memory with 1-D bulk copies (TMA) on one mbarrier; the threads add the two electric arrays and
// then apply the sides in six rounds that keep the reference's order wherever two sides reach the
// same B component: the x faces, the y faces, the z faces, then the edges along z, along x, along y
// (within a round no two sides share a component).  Each product is rounded before it is added, so
// the result is the reference's bit for bit.  B is written back whole and both electric arrays of
// the patch are zeroed, as the reference leaves them.
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "gb_common.cuh"
#include "tma.cuh"

namespace gb {
namespace {

constexpr int EF_THREADS = 128;
constexpr int NB1        = ( PS1 + 1 )*PS1*PS1;     // one face-centred component of a patch
constexpr int NBP        = 3*NB1;                   // the three components
constexpr int EFACE      = ( PS1 - 1 )*PS1;         // one of the two E components on a patch face
constexpr int EDGE0      = 6*2*EFACE;               // offset of the first edge in the packed sides
constexpr int NE         = GB_ELE_PER_PATCH;
static_assert( NE == EDGE0 + 12*PS1, "packed electric-field layout" );

template <typename R>
struct EleArgs {
   R *mag;  R *ele;  R *ele_b;
   const unsigned char *has;    // [npatch][18]
   const unsigned char *sib;    // [npatch][6]
   R    idh;                    // (real)( 1/dh )
};

// where side rounds write: the B component and the (offset, strides) of the reference's loops
// (MHD_FixUp_Electric.cpp:78-125 for faces, :157-190 for edges), in the patch's [3][9*8*8] B
struct FaceMap { int c1, off1, s1n, s1m, c2, off2, s2n, s2m; };
// faces with normal x, y, z: B1 = B_(xyz+2)%3 over m in [1, PS1), n in [0, PS1); B2 = B_(xyz+1)%3
// over m in [0, PS1), n in [1, PS1); offsets for the right face (LR = 1), zero for the left
__constant__ FaceMap c_face[3] = {
   { 2, PS1 - 1,                  PS1,             PS1*PS1, 1, PS1 - 1,           PS1,     ( PS1 + 1 )*PS1 },
   { 0, ( PS1 - 1 )*( PS1 + 1 ),  ( PS1 + 1 )*PS1, 1,       2, ( PS1 - 1 )*PS1,   PS1*PS1, 1 },
   { 1, PS1*( PS1 - 1 )*( PS1 + 1 ), 1,            PS1,     0, PS1*( PS1 - 1 )*( PS1 + 1 ), 1, PS1 + 1 } };
// edges along x, y, z (B1 = B_(xyz+1)%3, B2 = B_(xyz+2)%3): offset = LR1*a + LR2*b, stride
struct EdgeMap { int c1, a1, b1, st1, c2, a2, b2, st2; };
__constant__ EdgeMap c_edge[3] = {
   { 1, PS1*PS1,               PS1*( PS1 - 1 )*( PS1 + 1 ), 1,               2, ( PS1 - 1 )*PS1,             PS1*PS1*PS1, 1 },
   { 2, PS1*PS1*PS1,           PS1 - 1,                     PS1,             0, PS1*( PS1 - 1 )*( PS1 + 1 ), PS1,         PS1 + 1 },
   { 0, PS1,                   ( PS1 - 1 )*( PS1 + 1 ),     ( PS1 + 1 )*PS1, 1, PS1 - 1,                     PS1*PS1,     ( PS1 + 1 )*PS1 } };

template <typename R>
__global__ void __launch_bounds__(EF_THREADS) ele_fixup_kernel( const EleArgs<R> a )
{
   extern __shared__ __align__(16) unsigned char smem[];
   __shared__ unsigned s_has, s_sib;
   uint64_t *bar = (uint64_t*)smem;
   R *s_b  = (R*)( smem + 16 );
   R *s_e  = s_b + NBP;
   R *s_eb = s_e + NE;
   const int  tid = threadIdx.x;
   const long p   = blockIdx.x;
   R *g_b = a.mag + p*NBP, *g_e = a.ele + p*NE, *g_eb = a.ele_b + p*NE;

   if ( tid == 0 )
   {
      unsigned h = 0, sb = 0;
      for (int q=0; q<18; q++) if ( a.has[ 18*p + q ] ) h |= 1u << q;
      for (int q=0; q<6;  q++) if ( a.sib[ 6*p + q ]  ) sb |= 1u << q;
      s_has = h;  s_sib = sb;
      if ( h )
      {
         mbar_init( bar, 1 );
         mbar_init_fence();
         mbar_expect_tx( bar, ( NBP + 2*NE )*sizeof(R) );
         bulk_g2s( s_b,  g_b,  NBP*sizeof(R), bar );
         bulk_g2s( s_e,  g_e,  NE*sizeof(R),  bar );
         bulk_g2s( s_eb, g_eb, NE*sizeof(R),  bar );
      }
   }
   __syncthreads();
   const unsigned has = s_has, sib = s_sib;
   if ( has == 0u ) return;
   // the copies complete within microseconds; a wait that gives up leaves the patch unchanged
   if ( !__syncthreads_and( mbar_wait_bounded( bar, 0 ) ) ) return;
   const R idh = a.idh;

   // step 1 of the reference: electric += electric_bitrep
   for (int t=tid; t<NE; t+=EF_THREADS) s_e[t] = s_e[t] + s_eb[t];
   __syncthreads();

   // faces, one round per normal direction: items w = (LR, component, m, n), 2*2*56 per round
   for (int d=0; d<3; d++)
   {
      const FaceMap f = c_face[d];
      for (int w=tid; w<4*EFACE; w+=EF_THREADS)
      {
         const int LR = w/( 2*EFACE ), r = w % ( 2*EFACE ), sd = 2*d + LR;
         if ( !( has & ( 1u << sd ) ) ) continue;
         const R C = R( 2*LR - 1 )*idh;
         const R *E = s_e + sd*2*EFACE;
         if ( r < EFACE )
         {
            const int m = 1 + r/PS1, n = r % PS1;                                  // B1 += C*E[0]
            R &b = s_b[ f.c1*NB1 + LR*f.off1 + m*f.s1m + n*f.s1n ];
            b = b + mul_rn( C, E[r] );
         }
         else
         {
            const int r2 = r - EFACE, m = r2/( PS1 - 1 ), n = 1 + r2 % ( PS1 - 1 );   // B2 -= C*E[1]
            R &b = s_b[ f.c2*NB1 + LR*f.off2 + m*f.s2m + n*f.s2n ];
            b = b - mul_rn( C, E[ EFACE + r2 ] );
         }
      }
      __syncthreads();
   }

   // edges, one round per direction in the reference's order: along z (edges 0-3), x (4-7), y (8-11)
   for (int g=0; g<3; g++)
   {
      const int xyz = ( g + 2 ) % 3;
      const EdgeMap em = c_edge[xyz];
      if ( tid < 4*2*PS1 )
      {
         const int e = 4*g + tid/( 2*PS1 ), r = tid % ( 2*PS1 );
         const int LR1 = e % 2, LR2 = ( e % 4 )/2;
         const R *E = s_e + EDGE0 + e*PS1;
         if ( has & ( 1u << ( 6 + e ) ) )
         {
            if ( r < PS1 )
            {
               if ( sib & ( 1u << ( 2*em.c1 + LR1 ) ) )
               {
                  R &b = s_b[ em.c1*NB1 + LR1*em.a1 + LR2*em.b1 + r*em.st1 ];
                  b = b + mul_rn( R( 2*LR2 - 1 )*idh, E[r] );
               }
            }
            else if ( sib & ( 1u << ( 2*em.c2 + LR2 ) ) )
            {
               R &b = s_b[ em.c2*NB1 + LR1*em.a2 + LR2*em.b2 + ( r - PS1 )*em.st2 ];
               b = b + mul_rn( R( 1 - 2*LR1 )*idh, E[ r - PS1 ] );
            }
         }
      }
      __syncthreads();
   }

   // B back whole; both electric arrays zeroed (step 4 of the reference)
   constexpr int CB = NBP*(int)sizeof(R)/16, CE = NE*(int)sizeof(R)/16;
   const int4 z = make_int4( 0, 0, 0, 0 );
   for (int q=tid; q<CB; q+=EF_THREADS) reinterpret_cast<int4*>( g_b )[q] = reinterpret_cast<const int4*>( s_b )[q];
   for (int q=tid; q<CE; q+=EF_THREADS) { reinterpret_cast<int4*>( g_e )[q] = z;  reinterpret_cast<int4*>( g_eb )[q] = z; }
}

template <typename R>
int ele_fixup_run( void *mag, void *ele, void *ele_b, const unsigned char *has, const unsigned char *sib, int npatch,
                   double dh, cudaStream_t st )
{
   EleArgs<R> a;
   a.mag = (R*)mag;  a.ele = (R*)ele;  a.ele_b = (R*)ele_b;  a.has = has;  a.sib = sib;
   a.idh = (R)( 1.0/dh );
   const size_t smem = 16 + ( NBP + 2*NE )*sizeof(R);
   if ( cudaFuncSetAttribute( ele_fixup_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem ) != cudaSuccess )
      return GB_E_CUDA;
   ele_fixup_kernel<R><<< (unsigned)npatch, EF_THREADS, smem, st >>>( a );
   return ( cudaGetLastError() == cudaSuccess ) ? GB_OK : GB_E_CUDA;
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
   if ( !cfg_mhd( *cfg ) ) return GB_E_INVALID;   // MHD only
   if ( cfg->precision < GB_PREC_FP32 || cfg->precision > GB_PREC_FP64 ) return GB_E_INVALID;
   if ( !( dh > 0.0 ) || npatch < 0 ) return GB_E_INVALID;
   if ( npatch == 0 ) return GB_OK;
   if ( magnetic == nullptr || electric == nullptr || electric_bitrep == nullptr || has_ele == nullptr ||
        sib_leaf == nullptr ) return GB_E_INVALID;
   // the bulk copies move whole patches: 16-byte aligned bases
   if ( ( (uintptr_t)magnetic | (uintptr_t)electric | (uintptr_t)electric_bitrep ) & 15u ) return GB_E_ALIGN;
   const cudaStream_t st = (cudaStream_t)stream;
   if ( cfg->precision == GB_PREC_FP64 )
      return ele_fixup_run<double>( magnetic, electric, electric_bitrep, has_ele, sib_leaf, npatch, dh, st );
   return ele_fixup_run<float>( magnetic, electric, electric_bitrep, has_ele, sib_leaf, npatch, dh, st );
}
