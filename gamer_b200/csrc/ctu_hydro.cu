// Hydro CTU patch-group solver: PLM with characteristic tracing (HLL solvers: all waves,
// HLL_NO_REF_STATE; Roe and exact solvers: the reference states of the fastest waves), half-step
// Riemann fluxes, transverse-gradient correction, full-step Riemann fluxes, update.
//
// Reference path replaced: CPU_FluidSolver_CTU without MHD
// (src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_CTU.cpp:157-342, Hydro_TGradientCorrection :368-599).
// Sizes (CTU, no MHD): PLM FLU_NXT 20, FLU_GHOST_SIZE 2, LR_GHOST_SIZE 1; PPM FLU_NXT 22, 3, 2;
// N_FC_VAR = N_HF_FLUX = N_FL_FLUX = 18 for both (include/CUFLU.h:107-118, include/Macro.h:643-665).
// Like the MHD pipeline, the stages are separate kernels over (patch group x cell/face) items with
// per-patch-group scratch (~1.2 MB in FP32), run over chunks of patch groups.
// Dual energy (DE_ENPY, NC = 6): the dual-energy field is the last variable, a passive scalar to the
// reconstruction (traced with the entropy wave, :555-562), the Riemann solvers (upwinded with the
// mass flux) and the transverse correction, floored by PassiveFloor, and the full step ends with the
// dual-energy fix of Hydro_FullStepUpdate (CPU_Shared_FullStepUpdate.cpp:144-201).
#include <cstring>
#include <type_traits>
#include "../../include/gamer_b200_fluid.h"
#include "hydro_physics.cuh"

namespace gb {

namespace hctu {
constexpr int NX  = 20;                // FLU_NXT
constexpr int NX3 = NX*NX*NX;
constexpr int NF  = 18;                // N_FC_VAR = N_HF_FLUX = N_FL_FLUX
constexpr int NF3 = NF*NF*NF;
// input sizes of the reconstruction LR: PLM FLU_NXT 20 (LR_GHOST_SIZE 1, FLU_GHOST_SIZE 2), PPM
// FLU_NXT 22 (2, 3) (include/Macro.h:643-665); the face-state, flux and output grids are the same
template <int LR> struct G {
   static constexpr int NX  = ( LR == LR_PPM ) ? 22 : 20;   // FLU_NXT
   static constexpr int NX3 = NX*NX*NX;
   static constexpr int LRG = ( LR == LR_PPM ) ? 2 : 1;     // LR_GHOST_SIZE
   static constexpr int FLG = LRG + 1;                       // FLU_GHOST_SIZE
};

GB_DEV int idx3( int i, int j, int k, int ni, int nj ) { return ( k*nj + j )*ni + i; }

template <typename R>
struct Args {
   const R *in;      // [npg][NC][20^3]
   R *out;           // [npg][NC][16^3]
   R *flux;          // [npg][9][NC][16^2]  (nullptr: not stored)
   char *de;         // [npg][16^3] dual-energy status (NC = 6 or 8; nullptr: not stored)
   R *pri;           // scratch [npg][NC][20^3]
   R *fcv;           // scratch [npg][6][NC][18^3]
   R *fcf;           // scratch [npg][3][NC][18^3]
   int npg, limiter;
   int nnorm;        // NormPassive: number of listed passive scalars (0 = off)
   int norm_idx[4];  // NormIdx (passive indices, no repeats)
   R coeff, dt, dh;
   Phys<R> ph;
};
}

// items of one patch group per grid.z index (blockIdx.z = patch group of the chunk), 32-bit indices
#define HCTU_PG_LOOP( r, per ) \
   const int pg = blockIdx.z; \
   for (int r = blockIdx.x*blockDim.x + threadIdx.x; r < ( per ); r += gridDim.x*blockDim.x)

// kernels over the three face directions run them along grid.y, so that each direction's extents
// are compile-time constants (index decoding by constant division, no divergence)
#define HCTU_DIR( call ) \
   if      ( blockIdx.y == 0 ) { call( 0 ); } \
   else if ( blockIdx.y == 1 ) { call( 1 ); } \
   else                        { call( 2 ); }

// ---- conserved -> primitive (CPU_Shared_DataReconstruction.cpp:300-336) ----------------------
template <typename R, int P, int NC, int LR>
__global__ void hctu_con2pri( const __grid_constant__ hctu::Args<R> a )
{
   using namespace hctu;
   constexpr int NX3 = G<LR>::NX3;
   HCTU_PG_LOOP( c, NX3 )
   {
      const R *u = a.in + (size_t)pg*NC*NX3;
      R cu[NC], w[NC];
#     pragma unroll
      for (int v=0; v<NC; v++) cu[v] = u[v*NX3 + c];
      con2pri_cc<P,NC>( a.ph, cu, w );
      R *pri = a.pri + (size_t)pg*NC*NX3;
#     pragma unroll
      for (int v=0; v<NC; v++) pri[v*NX3 + c] = w[v];
   }
}

// ---- PLM + characteristic tracing along D (CPU_Shared_DataReconstruction.cpp:376-560, hydro) ----
// Hydro_GetEigenSystem (:1611-1892, no MHD): eigenvalues v_d - a, v_d (x3), v_d + a; the left and
// right eigenvectors in the rotated frame (rho, v_n, v_t1, v_t2, P) do not depend on the direction.
// RS: the HLL solvers trace with all waves (:454-477, HLL_INCLUDE_ALL_WAVES); Roe and the exact
// solver trace each face from the reference state of the fastest wave toward it (:513-553)
// CH: CHAR_RECONSTRUCTION, the PLM slopes limited in the characteristic variables of the cell
// LR_PPM: PPM face values (:704-1135, the limited slopes of the cell and its two neighbours, the
// parabola and its monotonicity constraint) and the tracing of the parabola (:1136-1290): each
// wave's correction over its domain of dependence adds the curvature term dfc6 = 6 (cc - (fL+fR)/2)
template <int D, int RS, int NC, int CH, int LR, typename R>
GB_DEV void hctu_recon_dir( const hctu::Args<R> &a, const R *pri, const R *cc, int c, R (&fcon)[2][NC] )
{
   using namespace hctu;
   typedef Dir<D> M;
   constexpr int NX = G<LR>::NX, NX3 = G<LR>::NX3;
   const int dcc[3] = { 1, NX, NX*NX };
   const R rho = cc[0], irho = R(1)/rho;
   const R a2 = a.ph.gamma*cc[4]/rho, as = gsqrt( a2 ), ia = R(1)/as, ia2 = ia*ia;
   R LE[5][5], RE[5][5];
#  pragma unroll
   for (int r=0; r<5; r++)
#     pragma unroll
      for (int q=0; q<5; q++) { LE[r][q] = R(0);  RE[r][q] = R(0); }
   LE[0][1] = -R(0.5)*rho*ia;  LE[0][4] = R(0.5)*ia2;
   LE[1][0] = R(1);            LE[1][4] = -ia2;
   LE[2][2] = R(1);            LE[3][3] = R(1);
   LE[4][1] = -LE[0][1];       LE[4][4] = LE[0][4];
   RE[0][0] = R(1);  RE[0][1] = -as*irho;  RE[0][4] = a2;
   RE[1][0] = R(1);
   RE[2][2] = R(1);  RE[3][3] = R(1);
   RE[4][0] = R(1);  RE[4][1] = -RE[0][1];  RE[4][4] = a2;
   const R vn = cc[M::n];
   const R ev[5] = { vn - as, vn, vn, vn, vn + as };
   R fl[NC], fr[NC];
   if constexpr ( LR == LR_PPM )
   {
      // the slopes of the cells c-1, c, c+1 (limited in primitive or characteristic variables)
      R sl[NC], sc[NC], sr[NC];
      if constexpr ( CH )
      {
         R ll[NC], cl[NC], cr[NC], rr[NC];
#        pragma unroll
         for (int v=0; v<NC; v++)
         {
            const R *q = pri + v*NX3 + c;
            ll[v] = q[-2*dcc[D]];  cl[v] = q[-dcc[D]];  cr[v] = q[dcc[D]];  rr[v] = q[2*dcc[D]];
         }
         ppm_char_slopes<D,NC>( a.ph, ll, cl, cc, cr, rr, a.limiter, a.coeff, sl, sc, sr );
      }
      else
      {
#        pragma unroll
         for (int v=0; v<NC; v++)
         {
            const R *q = pri + v*NX3 + c;
            sl[v] = limit_slope( q[-2*dcc[D]], q[-dcc[D]], q[0],         a.limiter, a.coeff );
            sc[v] = limit_slope( q[-dcc[D]],   q[0],       q[dcc[D]],    a.limiter, a.coeff );
            sr[v] = limit_slope( q[0],         q[dcc[D]],  q[2*dcc[D]],  a.limiter, a.coeff );
         }
      }
#     pragma unroll
      for (int v=0; v<NC; v++)
         ppm_faces( pri[v*NX3 + c - dcc[D]], cc[v], pri[v*NX3 + c + dcc[D]], sl[v], sc[v], sr[v], a.limiter, fl[v], fr[v] );
   }
   else if constexpr ( CH )
   {
      R cl[NC], cr[NC];
#     pragma unroll
      for (int v=0; v<NC; v++) { cl[v] = pri[v*NX3 + c - dcc[D]];  cr[v] = pri[v*NX3 + c + dcc[D]]; }
      plm_faces_char<D,NC>( a.ph, cl, cc, cr, a.limiter, a.coeff, fl, fr );
   }
   else
   {
#     pragma unroll
      for (int v=0; v<NC; v++)
      {
         const R l = pri[v*NX3 + c - dcc[D]], r = pri[v*NX3 + c + dcc[D]];
         plm_faces( l, cc[v], r, a.limiter, a.coeff, true, fl[v], fr[v] );
      }
   }
   const R dt_dh2 = R(0.5)*a.dt/a.dh;
   const int wv[5] = { 0, M::n, M::t1, M::t2, 4 };
   R dfc[5];
#  pragma unroll
   for (int q=0; q<5; q++) dfc[q] = fr[wv[q]] - fl[wv[q]];
   if constexpr ( LR == LR_PPM )
   {
      // PPM (:1145-1257): dfc6 = 6 (cc - (fL + fR)/2) in the rotated frame
      R dfc6[5];
#     pragma unroll
      for (int q=0; q<5; q++) dfc6[q] = R(6)*( cc[wv[q]] - R(0.5)*( fl[wv[q]] + fr[wv[q]] ) );
      R corl[5], corr[5];
      if constexpr ( RS == RS_HLLC || RS == RS_HLLE )
      {
         // all waves toward both faces (HLL_INCLUDE_ALL_WAVES)
#        pragma unroll
         for (int q=0; q<5; q++) { corl[q] = R(0);  corr[q] = R(0); }
#        pragma unroll
         for (int m=0; m<5; m++)
         {
            const R cC = -dt_dh2*ev[m], cD = R(-4.0/3.0)*( cC*cC );
            R cfl = R(0), cfr = R(0);
#           pragma unroll
            for (int q=0; q<5; q++)
            {
               cfl += LE[m][q]*( cC*( dfc[q] + dfc6[q] ) + cD*dfc6[q] );
               cfr += LE[m][q]*( cC*( dfc[q] - dfc6[q] ) + cD*dfc6[q] );
            }
#           pragma unroll
            for (int q=0; q<5; q++) { corl[q] = corl[q] + mul_rn( cfl, RE[m][q] );  corr[q] = corr[q] + mul_rn( cfr, RE[m][q] ); }
         }
      }
      else
      {
         // Roe / exact: the reference states of the fastest waves, then the waves toward each face
         const R cl0 = -dt_dh2*gmin( ev[0], R(0) ), cr0 = -dt_dh2*gmax( ev[4], R(0) );
#        pragma unroll
         for (int q=0; q<5; q++)
         {
            corl[q] = cl0*( dfc[q] + ( R(1) - R(4.0/3.0)*cl0 )*dfc6[q] );
            corr[q] = cr0*( dfc[q] - ( R(1) + R(4.0/3.0)*cr0 )*dfc6[q] );
         }
#        pragma unroll
         for (int m=0; m<5; m++)
         {
            if ( ev[m] <= R(0) )
            {
               const R cC = dt_dh2*( ev[0] - ev[m] ), cD = R(4.0/3.0)*dt_dh2*cC*( ev[0] + ev[m] );
               R cf = R(0);
#              pragma unroll
               for (int q=0; q<5; q++) cf += LE[m][q]*( cC*( dfc[q] + dfc6[q] ) + cD*dfc6[q] );
#              pragma unroll
               for (int q=0; q<5; q++) corl[q] = corl[q] + mul_rn( cf, RE[m][q] );
            }
            if ( ev[m] >= R(0) )
            {
               const R cA = dt_dh2*( ev[4] - ev[m] ), cB = R(4.0/3.0)*dt_dh2*cA*( ev[4] + ev[m] );
               R cf = R(0);
#              pragma unroll
               for (int q=0; q<5; q++) cf += LE[m][q]*( cA*( dfc[q] - dfc6[q] ) + cB*dfc6[q] );
#              pragma unroll
               for (int q=0; q<5; q++) corr[q] = corr[q] + mul_rn( cf, RE[m][q] );
            }
         }
      }
      // passive scalars with the entropy wave, the parabola integrated over its domain (:1262-1273)
      if constexpr ( NC > 5 )
      {
         const R cl = -dt_dh2*gmin( ev[1], R(0) ), cr = -dt_dh2*gmax( ev[1], R(0) );
#        pragma unroll
         for (int v=5; v<NC; v++)
         {
            const R dv = fr[v] - fl[v], dv6 = R(6)*( cc[v] - R(0.5)*( fl[v] + fr[v] ) );
            fl[v] += cl*( dv + ( R(1) - R(4.0/3.0)*cl )*dv6 );
            fr[v] += cr*( dv - ( R(1) + R(4.0/3.0)*cr )*dv6 );
         }
      }
#     pragma unroll
      for (int q=0; q<5; q++) { fl[wv[q]] += corl[q];  fr[wv[q]] += corr[q]; }
   }
   else if constexpr ( RS == RS_HLLC || RS == RS_HLLE )
   {
      // HLL solvers: corrections from all waves, the same on both faces (HLL_INCLUDE_ALL_WAVES)
      R corr[5];
#     pragma unroll
      for (int q=0; q<5; q++) corr[q] = R(0);
#     pragma unroll
      for (int m=0; m<5; m++)
      {
         R cf = R(0);
#        pragma unroll
         for (int q=0; q<5; q++) cf += LE[m][q]*dfc[q];
         cf *= -dt_dh2*ev[m];
         // uncontracted, as the reference's CPU build: sums that cancel do so exactly
#        pragma unroll
         for (int q=0; q<5; q++) corr[q] = corr[q] + mul_rn( cf, RE[m][q] );
      }
#     pragma unroll
      for (int q=0; q<5; q++) { fl[wv[q]] += corr[q];  fr[wv[q]] += corr[q]; }
   }
   else
   {
      // Roe / exact: each face from the reference state of the fastest wave moving toward it, then
      // the waves moving toward the face relative to it
      const R cl0 = -dt_dh2*gmin( ev[0], R(0) ), cr0 = -dt_dh2*gmax( ev[4], R(0) );
      R corl[5], corr[5];
#     pragma unroll
      for (int q=0; q<5; q++) { corl[q] = mul_rn( cl0, dfc[q] );  corr[q] = mul_rn( cr0, dfc[q] ); }
#     pragma unroll
      for (int m=0; m<5; m++)
      {
         if ( ev[m] <= R(0) )
         {
            R cf = R(0);
#           pragma unroll
            for (int q=0; q<5; q++) cf += LE[m][q]*dfc[q];
            cf *= dt_dh2*( ev[0] - ev[m] );
#           pragma unroll
            for (int q=0; q<5; q++) corl[q] = corl[q] + mul_rn( cf, RE[m][q] );
         }
         if ( ev[m] >= R(0) )
         {
            R cf = R(0);
#           pragma unroll
            for (int q=0; q<5; q++) cf += LE[m][q]*dfc[q];
            cf *= dt_dh2*( ev[4] - ev[m] );
#           pragma unroll
            for (int q=0; q<5; q++) corr[q] = corr[q] + mul_rn( cf, RE[m][q] );
         }
      }
#     pragma unroll
      for (int q=0; q<5; q++) { fl[wv[q]] += corl[q];  fr[wv[q]] += corr[q]; }
   }
   // passive scalars travel with the flow: the entropy wave only (:555-562; PPM above)
   if constexpr ( NC > 5 && LR == LR_PLM )
   {
      const R cl = -dt_dh2*gmin( ev[1], R(0) ), cr = -dt_dh2*gmax( ev[1], R(0) );
#     pragma unroll
      for (int v=5; v<NC; v++)
      {
         const R dv = fr[v] - fl[v];
         fl[v] += cl*dv;
         fr[v] += cr*dv;
      }
   }
   fl[0] = gmax( fl[0], a.ph.min_dens );  fr[0] = gmax( fr[0], a.ph.min_dens );
   fl[4] = check_floor( fl[4], a.ph.min_pres );  fr[4] = check_floor( fr[4], a.ph.min_pres );
#  pragma unroll
   for (int v=5; v<NC; v++)
      if ( a.ph.pfloor & ( 1u << v ) ) { fl[v] = gmax( fl[v], Lim<R>::tiny() );  fr[v] = gmax( fr[v], Lim<R>::tiny() ); }
   pri2con<NC>( a.ph, fl, fcon[0] );
   pri2con<NC>( a.ph, fr, fcon[1] );
}

template <typename R, int P, int RS, int NC, int CH, int LR>
__global__ void __launch_bounds__( 256, ( sizeof(R) == 8 ) ? 1 : 4 ) hctu_recon( const __grid_constant__ hctu::Args<R> a )
{
   using namespace hctu;
   constexpr int NX = G<LR>::NX, NX3 = G<LR>::NX3, LRG = G<LR>::LRG;
   const int d = blockIdx.y;
   HCTU_PG_LOOP( f, NF3 )
   {
      const int ci = f % NF + LRG, cj = ( f / NF ) % NF + LRG, ck = f / ( NF*NF ) + LRG;
      const R *pri = a.pri + (size_t)pg*NC*NX3;
      const int c = idx3( ci, cj, ck, NX, NX );
      R cc[NC], fcon[2][NC];
#     pragma unroll
      for (int v=0; v<NC; v++) cc[v] = pri[v*NX3 + c];
      if      ( d == 0 ) hctu_recon_dir<0,RS,NC,CH,LR>( a, pri, cc, c, fcon );
      else if ( d == 1 ) hctu_recon_dir<1,RS,NC,CH,LR>( a, pri, cc, c, fcon );
      else               hctu_recon_dir<2,RS,NC,CH,LR>( a, pri, cc, c, fcon );
      R *fcv = a.fcv + (size_t)pg*6*NC*NF3;
#     pragma unroll
      for (int q=0; q<2; q++)
#        pragma unroll
         for (int v=0; v<NC; v++) fcv[( ( 2*d + q )*NC + v )*NF3 + f] = fcon[q][v];
   }
}

// ---- Riemann fluxes (Hydro_ComputeFlux, CPU_Shared_ComputeFlux.cpp:113-376) -------------------
// half step: NSkip_N = NSkip_T = 0 (17 x 18 x 18 faces per direction); full step: NSkip_N = 0,
// NSkip_T = 1 (17 x 16 x 16), with the coarse-fine planes (Hydro_StoreIntFlux :391-450, no MHD)
template <int D, typename R, int P, int RS, int FULL, int NC>
GB_DEV void hctu_face( const hctu::Args<R> &a, int pg, int fi, int fj, int fk )
{
   using namespace hctu;
   constexpr int st = FULL ? 1 : 0;                       // transverse skip
   const int sk[3] = { D == 0 ? 0 : st, D == 1 ? 0 : st, D == 2 ? 0 : st };
   const int dfc[3] = { 1, NF, NF*NF };
   const int ifc = idx3( fi + sk[0], fj + sk[1], fk + sk[2], NF, NF );
   const R *fcv = a.fcv + (size_t)pg*6*NC*NF3;
   R L[NC], Rr[NC], F[NC];
#  pragma unroll
   for (int v=0; v<NC; v++) { L[v] = fcv[( ( 2*D + 1 )*NC + v )*NF3 + ifc];  Rr[v] = fcv[( 2*D*NC + v )*NF3 + ifc + dfc[D]]; }
   riemann<RS,D,P,NC>( a.ph, L, Rr, F );
   R *fcf = a.fcf + (size_t)pg*3*NC*NF3;
   const int ix = idx3( fi, fj, fk, NF, NF );
#  pragma unroll
   for (int v=0; v<NC; v++) fcf[( D*NC + v )*NF3 + ix] = F[v];
   if ( FULL && a.flux != nullptr )
   {
      const int fl[3] = { fi, fj, fk };
      const int nrm = fl[D];
      if ( ( nrm & 7 ) == 0 )
      {
         // transverse index with the smaller axis number is the fastest
         const int a0 = ( D == 0 ) ? fj : fi, a1 = ( D == 2 ) ? fj : fk;
         R *dst = a.flux + (size_t)pg*9*NC*PS2*PS2 + (size_t)( 3*D + nrm/PS1 )*NC*PS2*PS2 + a1*PS2 + a0;
#        pragma unroll
         for (int v=0; v<NC; v++) dst[v*PS2*PS2] = F[v];
      }
   }
}

template <typename R, int P, int RS, int FULL, int NC>
__global__ void __launch_bounds__( 256, ( sizeof(R) == 8 ) ? 1 : 3 ) hctu_flux( const __grid_constant__ hctu::Args<R> a )
{
   using namespace hctu;
   constexpr int nn = NF - 1, nt = FULL ? NF - 2 : NF;         // faces along / across the normal
   constexpr int per = nn*nt*nt;
   HCTU_PG_LOOP( q, per )
   {
#     define HCTU_FACE( D ) { \
         constexpr int e0 = ( D == 0 ) ? nn : nt, e1 = ( D == 1 ) ? nn : nt; \
         hctu_face<D,R,P,RS,FULL,NC>( a, pg, q % e0, ( q / e0 ) % e1, q / ( e0*e1 ) ); }
      HCTU_DIR( HCTU_FACE )
#     undef HCTU_FACE
   }
}

// ---- transverse-gradient correction (Hydro_TGradientCorrection, CPU_FluidSolver_CTU.cpp:368-599,
// no MHD): along D the face cells of the whole 18-wide range, across it the inner 16 ----------------
template <int D, typename R, int P, int NC>
GB_DEV void hctu_tgrad_dir( const hctu::Args<R> &a, int pg, int i0, int j0, int k0 )
{
   using namespace hctu;
   constexpr int T1 = ( D + 1 ) % 3, T2 = ( D + 2 ) % 3;
   const int dfl[3] = { 1, NF, NF*NF };
   const int f = idx3( i0 + ( D != 0 ), j0 + ( D != 1 ), k0 + ( D != 2 ), NF, NF );
   R *fcv = a.fcv + (size_t)pg*6*NC*NF3;
   const R *F = a.fcf + (size_t)pg*3*NC*NF3;
   const R dt_dh2 = R(0.5)*a.dt/a.dh;
   R q0[NC], q1[NC];
#  pragma unroll
   for (int v=0; v<NC; v++) { q0[v] = fcv[( 2*D*NC + v )*NF3 + f];  q1[v] = fcv[( ( 2*D + 1 )*NC + v )*NF3 + f]; }
#  pragma unroll
   for (int v=0; v<NC; v++)
   {
      const R tg1 = F[( T1*NC + v )*NF3 + f] - F[( T1*NC + v )*NF3 + f - dfl[T1]];
      const R tg2 = F[( T2*NC + v )*NF3 + f] - F[( T2*NC + v )*NF3 + f - dfl[T2]];
      const R c = -dt_dh2*( tg1 + tg2 );
      q0[v] += c;  q1[v] += c;
   }
   q0[0] = gmax( q0[0], a.ph.min_dens );  q1[0] = gmax( q1[0], a.ph.min_dens );
   q0[4] = floor_eint_in_engy<P>( a.ph, q0[0], q0[1], q0[2], q0[3], q0[4] );
   q1[4] = floor_eint_in_engy<P>( a.ph, q1[0], q1[1], q1[2], q1[3], q1[4] );
#  pragma unroll
   for (int v=5; v<NC; v++)
      if ( a.ph.pfloor & ( 1u << v ) ) { q0[v] = gmax( q0[v], Lim<R>::tiny() );  q1[v] = gmax( q1[v], Lim<R>::tiny() ); }
#  pragma unroll
   for (int v=0; v<NC; v++) { fcv[( 2*D*NC + v )*NF3 + f] = q0[v];  fcv[( ( 2*D + 1 )*NC + v )*NF3 + f] = q1[v]; }
}

template <typename R, int P, int NC>
__global__ void hctu_tgrad( const __grid_constant__ hctu::Args<R> a )
{
   using namespace hctu;
   constexpr int N3 = NF*( NF - 2 )*( NF - 2 );
   HCTU_PG_LOOP( q, N3 )
   {
      // extent NF along d, NF-2 across
#     define HCTU_TG( D ) { \
         constexpr int e0 = ( D == 0 ) ? NF : NF - 2, e1 = ( D == 1 ) ? NF : NF - 2; \
         hctu_tgrad_dir<D,R,P,NC>( a, pg, q % e0, ( q / e0 ) % e1, q / ( e0*e1 ) ); }
      HCTU_DIR( HCTU_TG )
#     undef HCTU_TG
   }
}

// ---- full-step update (Hydro_FullStepUpdate, CPU_Shared_FullStepUpdate.cpp:64-271, no MHD) -------
template <typename R, int P, int NC, int LR>
__global__ void hctu_update( const __grid_constant__ hctu::Args<R> a )
{
   using namespace hctu;
   constexpr int NX = G<LR>::NX, NX3 = G<LR>::NX3, FLG = G<LR>::FLG;
   typedef typename std::conditional<P == P_MIXED, double, R>::type A;
   constexpr int N3 = PS2*PS2*PS2;
   const A dt_dh = (A)a.dt/(A)a.dh;
   HCTU_PG_LOOP( q, N3 )
   {
      const int io = q % PS2, jo = ( q / PS2 ) % PS2, ko = q / ( PS2*PS2 );
      const int ifl = idx3( io, jo, ko, NF, NF );
      const int dfl[3] = { 1, NF, NF*NF };
      const int iin = idx3( io + FLG, jo + FLG, ko + FLG, NX, NX );
      const R *F = a.fcf + (size_t)pg*3*NC*NF3;
      const R *u = a.in + (size_t)pg*NC*NX3;
      R *out = a.out + (size_t)pg*NC*N3;
      R w[NC];
#     pragma unroll
      for (int v=0; v<NC; v++)
      {
         A df[3];
#        pragma unroll
         for (int d=0; d<3; d++) df[d] = (A)F[( d*NC + v )*NF3 + ifl + dfl[d]] - (A)F[( d*NC + v )*NF3 + ifl];
         w[v] = (R)( (A)u[v*NX3 + iin] - dt_dh*( df[0] + df[1] + df[2] ) );
      }
      if constexpr ( NC > 5 )
      {
         // passive floor and normalisation, then the dual-energy fix (CPU_Shared_FullStepUpdate.cpp:144-201);
         // the dual-energy field is the last variable (NC = 6: alone, NC = 8: after two user scalars)
         constexpr bool DUAL = ( NC == 6 || NC == 8 );
         constexpr int  NPU  = NC - 5 - ( DUAL ? 1 : 0 );
#        pragma unroll
         for (int v=5; v<NC; v++) if ( a.ph.pfloor & ( 1u << v ) ) w[v] = gmax( w[v], Lim<R>::tiny() );
         if constexpr ( NPU > 0 ) if ( a.nnorm > 0 ) normalize_passive<NC>( w[0], w, a.nnorm, a.norm_idx );
         if constexpr ( DUAL )
         {
            const R ekin = R(0.5)*( w[1]*w[1] + w[2]*w[2] + w[3]*w[3] )/w[0];
            if ( w[0] > R(0) && w[4]*R(2) > ekin )
            {
               char st;
               dual_energy_fix<P>( a.ph, w[0], w[1], w[2], w[3], w[4], w[NC-1], st );
               if ( a.de != nullptr ) a.de[(size_t)pg*N3 + q] = st;
            }
         }
      }
#     pragma unroll
      for (int v=0; v<NC; v++) out[v*N3 + q] = w[v];
   }
}

namespace {

size_t hctu_scratch_per_pg( size_t rsz, int nc, int lr )
{
   using namespace hctu;
   const size_t nx3 = ( lr == LR_PPM ) ? G<LR_PPM>::NX3 : G<LR_PLM>::NX3;
   return rsz*( (size_t)nc*nx3 + 6*(size_t)nc*NF3 + 3*(size_t)nc*NF3 ) + 3*256;
}

// items of one patch group (and direction) along x, about 4 per thread; face directions along y;
// patch groups along z (the directions of one patch group are scheduled together, sharing L2)
dim3 hctu_grid( int per, int npg, int block, int ndir = 1 )
{
   return dim3( ( per + 4*block - 1 )/( 4*block ), ndir, npg );
}

template <typename R, int P, int RS, int NC, int LR>
int hctu_solve_t( const gb_fluid_config &cfg, const void *in, void *out, void *flux, char *de, int npg,
                  const gb_fluid_params *prm, void *scratch, size_t scratch_bytes, cudaStream_t st )
{
   using namespace hctu;
   constexpr int NX3 = G<LR>::NX3;
   size_t fit = scratch_bytes / hctu_scratch_per_pg( sizeof(R), NC, LR );
   if ( fit < 1 ) return GB_E_INVALID;
   const int chunk = ( fit > 65535 ) ? 65535 : (int)fit;
   for (int p0 = 0; p0 < npg; p0 += chunk)
   {
      const int n = ( npg - p0 < chunk ) ? npg - p0 : chunk;
      char *w = (char*)scratch;
      auto take = [&]( size_t elems ) { R *r = (R*)w;  w += ( elems*sizeof(R) + 255 ) & ~(size_t)255;  return r; };
      Args<R> a;
      memset( &a, 0, sizeof(a) );
      a.in   = (const R*)in  + (size_t)p0*NC*NX3;
      a.out  = (R*)out + (size_t)p0*NC*PS2*PS2*PS2;
      a.flux = ( prm->store_flux && flux ) ? (R*)flux + (size_t)p0*9*NC*PS2*PS2 : nullptr;
      a.de   = ( NC > 5 && de ) ? de + (size_t)p0*PS2*PS2*PS2 : nullptr;
      a.pri  = take( (size_t)n*NC*NX3 );
      a.fcv  = take( (size_t)n*6*NC*NF3 );
      a.fcf  = take( (size_t)n*3*NC*NF3 );
      a.npg  = n;
      a.limiter = prm->lr_limiter;
      a.coeff = (R)prm->minmod_coeff;
      a.dt = (R)prm->dt;  a.dh = (R)prm->dh;
      a.ph.gamma = (R)cfg.gamma;  a.ph.gm1 = (R)( cfg.gamma - 1.0 );  a.ph.inv_gm1 = (R)( 1.0/( cfg.gamma - 1.0 ) );
      a.ph.min_dens = (R)prm->min_dens;  a.ph.min_pres = (R)prm->min_pres;  a.ph.min_eint = (R)prm->min_eint;
      a.ph.de_switch = (R)prm->dual_energy_switch;
      a.ph.jeans = prm->jeans_min_pres;  a.ph.jeans_coeff = (R)prm->jeans_min_pres_coeff;
      a.ph.pfloor = 0u;
      for (int v=5; v<NC; v++) if ( prm->passive_floor & ( 1LL << v ) ) a.ph.pfloor |= 1u << v;
      // FracPassive (mass fractions in the reconstruction) and NormPassive of the user scalars
      a.ph.frac_mask = 0u;
      if ( prm->frac_passive ) for (int k=0; k<prm->nfrac; k++) a.ph.frac_mask |= 1u << prm->frac_idx[k];
      a.nnorm = 0;
      if ( prm->norm_passive )
      {
         a.nnorm = prm->nnorm;
         for (int k=0; k<prm->nnorm && k<4; k++) a.norm_idx[k] = prm->norm_idx[k];
      }
      const int B = 256;
      hctu_con2pri<R,P,NC,LR><<< hctu_grid( NX3, n, B ), B, 0, st >>>( a );
      if ( cfg.char_reconstruction ) hctu_recon<R,P,RS,NC,1,LR><<< hctu_grid( NF3, n, B, 3 ), B, 0, st >>>( a );
      else                           hctu_recon<R,P,RS,NC,0,LR><<< hctu_grid( NF3, n, B, 3 ), B, 0, st >>>( a );
      hctu_flux<R,P,RS,0,NC><<< hctu_grid( ( NF - 1 )*NF*NF, n, B, 3 ), B, 0, st >>>( a );
      hctu_tgrad<R,P,NC><<< hctu_grid( NF*( NF - 2 )*( NF - 2 ), n, B, 3 ), B, 0, st >>>( a );
      hctu_flux<R,P,RS,1,NC><<< hctu_grid( ( NF - 1 )*( NF - 2 )*( NF - 2 ), n, B, 3 ), B, 0, st >>>( a );
      hctu_update<R,P,NC,LR><<< hctu_grid( PS2*PS2*PS2, n, B ), B, 0, st >>>( a );
      if ( cudaGetLastError() != cudaSuccess ) return GB_E_CUDA;
   }
   return GB_OK;
}

template <typename R, int P, int NC, int LR>
int hctu_solve_rs( const gb_fluid_config &cfg, const void *in, void *out, void *flux, char *de, int npg,
                   const gb_fluid_params *prm, void *scratch, size_t scratch_bytes, cudaStream_t st )
{
   if ( cfg.rsolver == GB_RSOLVER_HLLE )
      return hctu_solve_t<R,P,RS_HLLE,NC,LR>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
   if ( cfg.rsolver == GB_RSOLVER_ROE )
      return hctu_solve_t<R,P,RS_ROE,NC,LR>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
   if ( cfg.rsolver == GB_RSOLVER_EXACT )
      return hctu_solve_t<R,P,RS_EXACT,NC,LR>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
   return hctu_solve_t<R,P,RS_HLLC,NC,LR>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
}

template <typename R, int P, int LR>
int hctu_solve_nc( const gb_fluid_config &cfg, const void *in, void *out, void *flux, char *de, int npg,
                   const gb_fluid_params *prm, void *scratch, size_t scratch_bytes, cudaStream_t st )
{
   const bool dual = ( cfg.dual_energy == GB_DE_ENPY );
   if ( cfg.npassive_user == GB_NPASSIVE_USER )
   {
      static_assert( GB_NPASSIVE_USER == 2, "the passive-scalar instantiations are built for two user scalars" );
      return dual ? hctu_solve_rs<R,P,8,LR>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st )
                  : hctu_solve_rs<R,P,7,LR>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
   }
   if ( dual )
      return hctu_solve_rs<R,P,6,LR>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
   return hctu_solve_rs<R,P,5,LR>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
}

template <typename R, int P>
int hctu_solve_lr( const gb_fluid_config &cfg, const void *in, void *out, void *flux, char *de, int npg,
                   const gb_fluid_params *prm, void *scratch, size_t scratch_bytes, cudaStream_t st )
{
   if ( cfg.lr_scheme == GB_LR_PPM )
      return hctu_solve_nc<R,P,LR_PPM>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
   return hctu_solve_nc<R,P,LR_PLM>( cfg, in, out, flux, de, npg, prm, scratch, scratch_bytes, st );
}

} // namespace

size_t ctu_hydro_scratch_bytes_per_pg( int precision, int ncomp, int lr_scheme )
{
   return hctu_scratch_per_pg( ( precision == GB_PREC_FP64 ) ? 8 : 4, ncomp, lr_scheme );
}

// one hydro CTU solve of npg patch groups in chunks of scratch_bytes / ctu_hydro_scratch_bytes_per_pg
int ctu_hydro_solve( const gb_fluid_config &cfg, const void *flu_in, void *flu_out, void *flux, char *de, int npg,
                     const gb_fluid_params *prm, void *scratch, size_t scratch_bytes, cudaStream_t st )
{
   if ( cfg.precision == GB_PREC_FP64 )
      return hctu_solve_lr<double,P_FP64>( cfg, flu_in, flu_out, flux, de, npg, prm, scratch, scratch_bytes, st );
   if ( cfg.precision == GB_PREC_MIXED )
      return hctu_solve_lr<float,P_MIXED>( cfg, flu_in, flu_out, flux, de, npg, prm, scratch, scratch_bytes, st );
   return hctu_solve_lr<float,P_FP32>( cfg, flu_in, flu_out, flux, de, npg, prm, scratch, scratch_bytes, st );
}

} // namespace gb
