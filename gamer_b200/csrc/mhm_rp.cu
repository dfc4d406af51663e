// MHM_RP half step (hydro): Hydro_RiemannPredict_Flux + Hydro_RiemannPredict
// (src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_MHM.cpp:593-950).
//
// The reference evaluates first-order Riemann fluxes between neighbouring input cells over the
// whole 22^3 window, stores them in global scratch (g_Flux_Half), then advances the inner 20^3
// cells by dt/2 with them and stores the primitive half-step state (g_PriVar_Half) for the PLM
// reconstruction of the full step (22^3 -> 20^3 with PLM, 24^3 -> 22^3 with PPM).  Here one CTA
// sweeps a patch group plane by plane along z:
//   * the conserved input planes kc-1..kc+1 stay in a three-plane ring in shared memory;
//   * for half-step plane k (input plane kc = k+1) it solves the z problems between kc and kc+1
//     (20x20), the x problems of plane kc (21 faces x 20 rows) and the y problems (20 columns x 21
//     faces) -- 1240 per plane -- into shared-memory flux planes; the z fluxes below, between kc-1
//     and kc, are the previous plane's;
//   * each half-step cell is then U_in - dt/(2dh) * ((dFx + dFy) + dFz) (the reference's summation
//     order), floored (MinDens, MinEint, PassiveFloor), converted to primitive variables (with the
//     Jeans pressure floor and FracPassive) and written to the half-step state [npg][NC][20^3], which
//     the MHM kernel's SCH_MHM_RP instantiation reconstructs from.
// Every Riemann problem is solved once; the global traffic is the input read once and the half-step
// state written once.  The mixed policy accumulates the flux differences in double.
#include <type_traits>
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "hydro_physics.cuh"

namespace gb {

template <typename R>
struct RpArgs {
   const R *in;       // [npg][NC][N^3] conserved (N = 22 with PLM, 24 with PPM)
   R       *half;     // [npg][NC][(N-2)^3] primitive half-step state
   int      npg;
   R        dt_dh2;   // dt/(2 dh)
   Phys<R>  ph;
};

// input width NXI (FLU_NXT: 22 with PLM, 24 with PPM), flux faces NXI - 1, half-state width NXI - 2
constexpr int RPH_BLOCK = 256;

__host__ __device__ inline size_t rp_half_smem( int rsz, int nc, int nxi )
{
   const int nf = nxi - 1, nv = nxi - 2;
   return (size_t)rsz*nc*( 3*nxi*nxi + 2*nv*nv + 2*nv*nf );
}

template <typename R, int P, int RS, int NC, int NXI>
__global__ void __launch_bounds__( RPH_BLOCK ) mhm_rp_half_kernel( const __grid_constant__ RpArgs<R> a )
{
   typedef typename std::conditional<P == P_MIXED, double, R>::type A;   // accumulation type
   constexpr int N = NXI, NF = NXI - 1, NV = NXI - 2, N2 = N*N, NV2 = NV*NV, NV3 = NV*NV*NV;
   constexpr int NZ = NV2, NXF = NV*NF;          // z problems, x (and y) problems per plane
   extern __shared__ __align__(16) unsigned char smem[];
   R *s_in = (R*)smem;                   // [3][NC][N*N]  conserved planes, slot = plane % 3
   R *s_fz = s_in + 3*NC*N2;             // [2][NC][NV][NV] z fluxes, slot = (upper input plane) & 1
   R *s_fx = s_fz + 2*NC*NV2;            // [NC][NV rows j-1][NF faces i]
   R *s_fy = s_fx + NC*NXF;              // [NC][NF faces j][NV columns i-1]
   const int tid = threadIdx.x, nth = blockDim.x;
   const Phys<R> ph = a.ph;

   for (int pg = blockIdx.x; pg < a.npg; pg += gridDim.x)
   {
      const R *g = a.in + (size_t)pg*NC*N*N2;
      R *h = a.half + (size_t)pg*NC*NV3;

      auto load = [&]( int c ) {
         R *dst = s_in + ( c % 3 )*NC*N2;
         for (int e = tid; e < NC*N2; e += nth)
         {
            const int v = e / N2, r = e % N2;
            dst[e] = g[(size_t)v*N*N2 + (size_t)c*N2 + r];
         }
      };
      // z problems between input planes c and c+1 at columns (i, j) = 1..NV, into slot (c+1) & 1
      auto zflux = [&]( int c, int e ) {
         const R *lo = s_in + ( c % 3 )*NC*N2, *hi = s_in + ( ( c + 1 ) % 3 )*NC*N2;
         const int i = 1 + e % NV, j = 1 + e / NV, q = j*N + i;
         R L[NC], Rr[NC], F[NC];
#        pragma unroll
         for (int v=0; v<NC; v++) { L[v] = lo[v*N2 + q];  Rr[v] = hi[v*N2 + q]; }
         riemann<RS,2,P,NC>( ph, L, Rr, F );
         R *dst = s_fz + ( ( c + 1 ) & 1 )*NC*NV2 + e;
#        pragma unroll
         for (int v=0; v<NC; v++) dst[v*NV2] = F[v];
      };

      __syncthreads();                    // the previous patch group's last reads are done
      load( 0 );
      load( 1 );
      __syncthreads();
      for (int e = tid; e < NZ; e += nth) zflux( 0, e );

      for (int k = 0; k < NV; k++)
      {
         const int kc = k + 1;            // input plane of half-step plane k
         load( kc + 1 );                  // its slot held plane kc-2, no longer read
         __syncthreads();
         // the z problems above plane kc and the x / y problems of plane kc
         const R *pc = s_in + ( kc % 3 )*NC*N2;
         for (int e = tid; e < NZ + 2*NXF; e += nth)
         {
            if ( e < NZ ) { zflux( kc, e );  continue; }
            R L[NC], Rr[NC], F[NC];
            if ( e < NZ + NXF )
            {
               const int f = e - NZ, i = f % NF, j = 1 + f / NF, q = j*N + i;   // face between i and i+1
#              pragma unroll
               for (int v=0; v<NC; v++) { L[v] = pc[v*N2 + q];  Rr[v] = pc[v*N2 + q + 1]; }
               riemann<RS,0,P,NC>( ph, L, Rr, F );
#              pragma unroll
               for (int v=0; v<NC; v++) s_fx[v*NXF + f] = F[v];
            }
            else
            {
               const int f = e - NZ - NXF, i = 1 + f % NV, j = f / NV, q = j*N + i;   // face between j and j+1
#              pragma unroll
               for (int v=0; v<NC; v++) { L[v] = pc[v*N2 + q];  Rr[v] = pc[v*N2 + q + N]; }
               riemann<RS,1,P,NC>( ph, L, Rr, F );
#              pragma unroll
               for (int v=0; v<NC; v++) s_fy[v*NXF + f] = F[v];
            }
         }
         __syncthreads();
         // half-step cells of plane k
         const R *fzl = s_fz + ( kc & 1 )*NC*NV2, *fzu = s_fz + ( ( kc + 1 ) & 1 )*NC*NV2;
         for (int e = tid; e < NV2; e += nth)
         {
            const int i = e % NV, j = e / NV, q = ( j + 1 )*N + ( i + 1 );
            R u[NC], w[NC];
#           pragma unroll
            for (int v=0; v<NC; v++)
            {
               const A dfx = (A)s_fx[v*NXF + j*NF + i + 1] - (A)s_fx[v*NXF + j*NF + i];
               const A dfy = (A)s_fy[v*NXF + ( j + 1 )*NV + i] - (A)s_fy[v*NXF + j*NV + i];
               const A dfz = (A)fzu[v*NV2 + e] - (A)fzl[v*NV2 + e];
               u[v] = (R)( (A)pc[v*N2 + q] - (A)a.dt_dh2*( ( dfx + dfy ) + dfz ) );
            }
            u[0] = gmax( u[0], ph.min_dens );
            u[4] = floor_eint_in_engy<P>( ph, u[0], u[1], u[2], u[3], u[4] );
#           pragma unroll
            for (int v=5; v<NC; v++) if ( ph.pfloor & ( 1u << v ) ) u[v] = gmax( u[v], Lim<R>::tiny() );
            con2pri_cc<P,NC>( ph, u, w );
#           pragma unroll
            for (int v=0; v<NC; v++) h[(size_t)v*NV3 + (size_t)k*NV2 + e] = w[v];
         }
         // the next iteration's load writes the slot of plane kc-1 (not read here) and its
         // barrier orders these reads of s_fx / s_fy / s_fz before the next writes
      }
   }
}

// one launch over npg patch groups (persistent grid: SMs x resident CTAs)
template <typename R, int P, int RS, int NC, int NXI>
cudaError_t rp_half_launch( const RpArgs<R> &a, cudaStream_t st )
{
   const void *fn = (const void*)mhm_rp_half_kernel<R,P,RS,NC,NXI>;
   const size_t smem = rp_half_smem( sizeof(R), NC, NXI );
   int dev = 0, nsm = 0, per_sm = 0;
   cudaGetDevice( &dev );
   cudaDeviceGetAttribute( &nsm, cudaDevAttrMultiProcessorCount, dev );
   cudaError_t err = cudaFuncSetAttribute( fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem );
   if ( err != cudaSuccess ) return err;
   err = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, fn, RPH_BLOCK, smem );
   if ( err != cudaSuccess ) return err;
   if ( per_sm < 1 ) return cudaErrorInvalidConfiguration;
   int grid = nsm*per_sm;
   if ( grid > a.npg ) grid = a.npg;
   if ( grid == 0 ) return cudaSuccess;
   mhm_rp_half_kernel<R,P,RS,NC,NXI><<< grid, RPH_BLOCK, smem, st >>>( a );
   return cudaGetLastError();
}

template <typename R, int P, int NXI>
cudaError_t rp_half_pick_n( int rs, int nc, const RpArgs<R> &a, cudaStream_t st )
{
   if ( rs == RS_HLLC && nc == 5 ) return rp_half_launch<R,P,RS_HLLC,5,NXI>( a, st );
   if ( rs == RS_HLLC && nc == 6 ) return rp_half_launch<R,P,RS_HLLC,6,NXI>( a, st );
   if ( rs == RS_HLLE && nc == 5 ) return rp_half_launch<R,P,RS_HLLE,5,NXI>( a, st );
   if ( rs == RS_HLLE && nc == 6 ) return rp_half_launch<R,P,RS_HLLE,6,NXI>( a, st );
   if ( rs == RS_ROE  && nc == 5 ) return rp_half_launch<R,P,RS_ROE,5,NXI>( a, st );
   if ( rs == RS_ROE  && nc == 6 ) return rp_half_launch<R,P,RS_ROE,6,NXI>( a, st );
   // two user passive scalars, without / with the dual-energy field (FP64 with 8 variables on the
   // 24^3 PPM input needs 237 KB of shared memory, above a CTA's 227 KB)
   if ( sizeof(R) == 8 && nc == 8 && NXI == 24 ) return cudaErrorNotSupported;
   if constexpr ( !( sizeof(R) == 8 && NXI == 24 ) )
   {
      if ( rs == RS_HLLC && nc == 8 ) return rp_half_launch<R,P,RS_HLLC,8,NXI>( a, st );
      if ( rs == RS_HLLE && nc == 8 ) return rp_half_launch<R,P,RS_HLLE,8,NXI>( a, st );
      if ( rs == RS_ROE  && nc == 8 ) return rp_half_launch<R,P,RS_ROE,8,NXI>( a, st );
   }
   if ( rs == RS_HLLC && nc == 7 ) return rp_half_launch<R,P,RS_HLLC,7,NXI>( a, st );
   if ( rs == RS_HLLE && nc == 7 ) return rp_half_launch<R,P,RS_HLLE,7,NXI>( a, st );
   if ( rs == RS_ROE  && nc == 7 ) return rp_half_launch<R,P,RS_ROE,7,NXI>( a, st );
   return cudaErrorNotSupported;
}

template <typename R, int P>
cudaError_t rp_half_pick( int rs, int nc, int nxi, const RpArgs<R> &a, cudaStream_t st )
{
   if ( nxi == 22 ) return rp_half_pick_n<R,P,22>( rs, nc, a, st );
   if ( nxi == 24 ) return rp_half_pick_n<R,P,24>( rs, nc, a, st );
   return cudaErrorNotSupported;
}

// The half step of npg patch groups: in [npg][nc][nxi^3] -> half [npg][nc][(nxi-2)^3] (nxi = FLU_NXT:
// 22 with PLM, 24 with PPM); ph carries the floors, the passive-floor mask and the reconstruction
// options.  Asynchronous on st.
int mhm_rp_half( int precision, int rsolver, int nc, int nxi, const void *in, void *half, int npg, double dt,
                 double dh, const Phys<double> &phd, cudaStream_t st )
{
   cudaError_t err;
   if ( precision == GB_PREC_FP64 )
   {
      RpArgs<double> a;
      a.in = (const double*)in;  a.half = (double*)half;  a.npg = npg;
      a.dt_dh2 = 0.5*dt/dh;  a.ph = phd;
      err = rp_half_pick<double,P_FP64>( rsolver, nc, nxi, a, st );
   }
   else
   {
      RpArgs<float> a;
      a.in = (const float*)in;  a.half = (float*)half;  a.npg = npg;
      a.dt_dh2 = (float)0.5f*(float)dt/(float)dh;
      a.ph.gamma = (float)phd.gamma;  a.ph.gm1 = (float)phd.gm1;  a.ph.inv_gm1 = (float)phd.inv_gm1;
      a.ph.min_dens = (float)phd.min_dens;  a.ph.min_pres = (float)phd.min_pres;  a.ph.min_eint = (float)phd.min_eint;
      a.ph.de_switch = (float)phd.de_switch;  a.ph.jeans_coeff = (float)phd.jeans_coeff;  a.ph.jeans = phd.jeans;
      a.ph.frac_mask = phd.frac_mask;  a.ph.pfloor = phd.pfloor;
      err = ( precision == GB_PREC_MIXED ) ? rp_half_pick<float,P_MIXED>( rsolver, nc, nxi, a, st )
                                           : rp_half_pick<float,P_FP32>( rsolver, nc, nxi, a, st );
   }
   if ( err == cudaErrorNotSupported ) return GB_E_UNSUPPORTED;
   return ( err == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

} // namespace gb
