// MHD CTU patch-group solver: PLM with characteristic tracing, HLLD (HLLE rescue), constrained
// transport (Gardiner & Stone 2008 upwinded EMFs), transverse-gradient correction.
//
// Reference path replaced: CUFLU_FluidSolver_CTU with MHD (src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_CTU.cpp:157-342).
// The CTU pipeline has ten dependent stages with different stencils and eight variables plus a
// staggered magnetic field; its working set per patch group (~2.8 MB in FP32: face states of six
// faces, two flux sets, edge EMFs, half-step B) does not fit one SM's shared memory, so each stage
// is a separate kernel over (patch group x cell/face/edge) items, run over chunks of patch groups
// whose scratch stays resident in the 126 MB L2 (gb_fluid_set_mhd_chunk).
//
// Sizes (CTU + MHD + PLM): FLU_NXT 22, N_FC_VAR 20, N_HF_FLUX 20, N_HF_VAR 18, N_HF_ELE 19,
// N_FL_FLUX 18, N_FL_ELE 17, LR_GHOST_SIZE 1, FLU_GHOST_SIZE 3 (include/CUFLU.h:96-134, include/Macro.h:645-665).
//
// MHM_RP with MHD (CUFLU_FluidSolver_MHM with MHD, CPU_FluidSolver_MHM.cpp:396-565) runs through the
// same pipeline: its own half step (first-order Riemann predictor, CT update of B over dt/2,
// half-step state, PLM on it), then the CTU full-step kernels, whose faces, edges and cells are
// the same (FLU_NXT 22: N_FL_FLUX 18, N_FL_ELE 17).
#include <cstring>
#include <type_traits>
#include "../../include/gamer_b200_fluid.h"
#include "mhd_physics.cuh"

namespace gb {

namespace ctu {
constexpr int NX   = 22;                // FLU_NXT
constexpr int NX3  = NX*NX*NX;
constexpr int NBIN = ( NX + 1 )*NX*NX;  // one face-centred B component of the input
constexpr int NF   = 20;                // N_FC_VAR = N_HF_FLUX
constexpr int NF3  = NF*NF*NF;
constexpr int NHV  = 18;                // N_HF_VAR
constexpr int NHE  = 19;                // N_HF_ELE
constexpr int NFF  = 18;                // N_FL_FLUX
constexpr int NFE  = 17;                // N_FL_ELE
constexpr int NBH  = ( NHV + 1 )*NHV*NHV;   // one half-step B component
constexpr int NEC  = NHE*NHE*NHE;       // one EMF component (largest stride)
constexpr int NBOUT = ( PS2 + 1 )*PS2*PS2;
constexpr int NELE  = ( PS2 + 1 )*PS2;
constexpr int LRG = 1, FLG = 3;
// MHM_RP + MHD + PLM (FLU_NXT 22): N_HF_FLUX 22, N_HF_VAR 20, N_HF_ELE 21, N_FC_VAR 18, N_FL_FLUX 18,
// N_FL_ELE 17 (include/CUFLU.h:96-106) -- the full step has the extents of the CTU full step; with PPM
// (FLU_NXT 24) N_HF_FLUX 24, N_HF_VAR 22, N_HF_ELE 23 and the same full step as CTU+PPM
constexpr int RHV  = 20;                // N_HF_VAR (PLM)
// MHM + MHD + PLM: FLU_NXT 20, FLU_GHOST_SIZE 2, N_FC_VAR 18, N_HF_ELE 19, N_FL_FLUX 18, N_FL_ELE 17
// (include/CUFLU.h:83-93) -- the full step again has the extents of the CTU full step
constexpr int MNX = 20, MNX3 = MNX*MNX*MNX, MNBIN = ( MNX + 1 )*MNX*MNX, MFLG = 2;
// input-width dependent sizes: FLU_NXT nxi = 20 (MHM), 22 (CTU+PLM, MHM_RP), 24 (CTU+PPM)
__host__ __device__ constexpr int flg_of( int nxi ) { return ( nxi - PS2 )/2; }                         // FLU_GHOST_SIZE
__host__ __device__ constexpr int plane_of( int nxi ) { return ( nxi > NX ) ? nxi*nxi*nxi : NX3; }       // `pri` plane
__host__ __device__ constexpr int nbin_of( int nxi ) { return ( nxi + 1 )*nxi*nxi; }                     // input B component
}

GB_DEV int idx3( int i, int j, int k, int ni, int nj ) { return ( k*nj + j )*ni + i; }

// index of face-centred component d at cell (i,j,k) of an n^3 cell grid (IDX321_BX/BY/BZ, include/Macro.h:1202-1204)
GB_DEV int idx_b( int d, int i, int j, int k, int n )
{
   return ( d == 0 ) ? idx3( i, j, k, n + 1, n ) : ( d == 1 ) ? idx3( i, j, k, n, n + 1 ) : idx3( i, j, k, n, n );
}
// offset to the next face along d of component d (n^3 cell grid)
GB_DEV int db_next( int d, int n ) { return ( d == 0 ) ? 1 : ( d == 1 ) ? n : n*n; }

template <typename R>
struct CtuArgs {
   const R *in;      // [npg][5][22^3]
   const R *bin;     // [npg][3][23*22*22]
   R *out;           // [npg][5][16^3]
   R *bout;          // [npg][3][17*16*16]
   R *flux;          // [npg][9][5][16^2]   (nullptr: not stored)
   R *ele;           // [npg][9][2][17*16]  (nullptr: not stored)
   R *pri;           // scratch [npg][8][22^3]  (later the half-step primitives, stride 18)
   R *fcv;           // scratch [npg][6][8][20^3]
   R *fcf;           // scratch [npg][3][8][20^3]
   R *bh;            // scratch [npg][3][19*18*18]
   R *ec;            // scratch [npg][3][19^3]
   const int *active;   // [npg] MinMod retry pass: nonzero for the patch groups it recomputes (nullptr: all)
   int *fail_next;      // [npg] set to 1 for a patch group with an unphysical output cell (nullptr: no check)
   int npg;
   int limiter;
   int ec_pg;        // EMF elements per patch group (3 components at the largest stride)
   R coeff, dt, dh;
   Phys<R> ph;
};

template <typename R> GB_DEV R minmod2( R a, R b )
{
   return ( a*b > R(0) ) ? gsign( a )*gmin( gabs( a ), gabs( b ) ) : R(0);
}

// items of one patch group per grid.z index (blockIdx.z = patch group of the chunk), 32-bit indices
#define PG_LOOP( r, per ) \
   const int pg = blockIdx.z; \
   if ( a.active != nullptr && a.active[pg] == 0 ) return; \
   for (int r = blockIdx.x*blockDim.x + threadIdx.x; r < ( per ); r += gridDim.x*blockDim.x)

// kernels over the three face / edge directions run them along grid.y, so that each direction's
// extents are compile-time constants (index decoding by constant division, no divergence)
#define GB_CTU_DIR( call ) \
   if      ( blockIdx.y == 0 ) { call( 0 ); } \
   else if ( blockIdx.y == 1 ) { call( 1 ); } \
   else                        { call( 2 ); }

// ---- K0: conserved -> primitive with cell-centred B (CPU_Shared_DataReconstruction.cpp:368-397) ----
// NXI: FLU_NXT of the input (22: CTU and MHM_RP; 20: MHM); `pri` planes of NXI^3
template <typename R, int P, int NXI = ctu::NX>
__global__ void ctu_con2pri( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int N = NXI, N3 = N*N*N, NB = ( N + 1 )*N*N;
   PG_LOOP( c, N3 )
   {
      const int i = c % N, j = ( c / N ) % N, k = c / ( N*N );
      const R *u = a.in + (size_t)pg*5*N3;
      const R *b = a.bin + (size_t)pg*3*NB;
      R cu[NM], w[NM];
#     pragma unroll
      for (int v=0; v<5; v++) cu[v] = u[v*N3 + c];
#     pragma unroll
      for (int d=0; d<3; d++)
      {
         const int ib = idx_b( d, i, j, k, N );
         cu[MO + d] = R(0.5)*( b[d*NB + ib] + b[d*NB + ib + db_next( d, N )] );
      }
      mhd_con2pri<P>( a.ph, cu, w );
      // Jeans pressure floor of the cell-centred primitive variables (CPU_Shared_FluUtility.cpp:272-281)
      if ( a.ph.jeans ) w[4] = check_floor( w[4], a.ph.jeans_coeff*( w[0]*w[0] ) );
      R *pri = a.pri + (size_t)pg*NM*plane_of( N );
#     pragma unroll
      for (int v=0; v<NM; v++) pri[v*N3 + c] = w[v];
   }
}

// ---- K1: PLM + characteristic tracing + MHD source terms (CPU_Shared_DataReconstruction.cpp:400-680) ----
// CH: CHAR_RECONSTRUCTION, the slopes limited in the 7-wave characteristic variables of the cell
// the face values of cell c along D from the primitive array (planes of PL cells, cell stride st
// along D): PLM, PLM with the slopes limited in the cell's MHD wave amplitudes (CH; LE / RE its
// eigenvectors along D), or PPM from the limited slopes of the cell and its two neighbours (each
// limited, with CH, in its own cell's wave amplitudes); CPU_Shared_DataReconstruction.cpp:386-430,
// :870-907, :1080-1130
template <int D, int CH, int LR, typename R>
GB_DEV void mhd_face_values( const CtuArgs<R> &a, const R *pri, int PL, int c, int st, const R *cc,
                             const R (&LE)[7][7], const R (&RE)[7][7], R (&fl)[NM], R (&fr)[NM] )
{
   const int NX3 = PL;
   const int dcc[3] = { st, st, st };
   if constexpr ( LR == LR_PPM )
   {
      R sl[NM], sc[NM], sr[NM];
      if constexpr ( CH )
      {
         R pm2[NM], pm1[NM], pp1[NM], pp2[NM];
#        pragma unroll
         for (int v=0; v<NM; v++)
         {
            const R *q = pri + v*NX3 + c;
            pm2[v] = q[-2*dcc[D]];  pm1[v] = q[-dcc[D]];  pp1[v] = q[dcc[D]];  pp2[v] = q[2*dcc[D]];
         }
         {
            R e_[7], L_[7][7], R_[7][7];
            mhd_eigen<D>( a.ph, pm1, e_, L_, R_ );
            mhd_char_limited_slopes<D>( a.ph, L_, R_, pm2, pm1, cc, a.limiter, a.coeff, sl );
         }
         mhd_char_limited_slopes<D>( a.ph, LE, RE, pm1, cc, pp1, a.limiter, a.coeff, sc );
         {
            R e_[7], L_[7][7], R_[7][7];
            mhd_eigen<D>( a.ph, pp1, e_, L_, R_ );
            mhd_char_limited_slopes<D>( a.ph, L_, R_, cc, pp1, pp2, a.limiter, a.coeff, sr );
         }
      }
      else
      {
#        pragma unroll
         for (int v=0; v<NM; v++)
         {
            const R *q = pri + v*NX3 + c;
            sl[v] = limit_slope( q[-2*dcc[D]], q[-dcc[D]], q[0],        a.limiter, a.coeff );
            sc[v] = limit_slope( q[-dcc[D]],   q[0],       q[dcc[D]],   a.limiter, a.coeff );
            sr[v] = limit_slope( q[0],         q[dcc[D]],  q[2*dcc[D]], a.limiter, a.coeff );
         }
      }
#     pragma unroll
      for (int v=0; v<NM; v++)
         ppm_faces( pri[v*NX3 + c - dcc[D]], cc[v], pri[v*NX3 + c + dcc[D]], sl[v], sc[v], sr[v], a.limiter, fl[v], fr[v] );
   }
   else if constexpr ( CH )
   {
      R cl[NM], cr[NM], s[NM];
#     pragma unroll
      for (int v=0; v<NM; v++) { cl[v] = pri[v*NX3 + c - dcc[D]];  cr[v] = pri[v*NX3 + c + dcc[D]]; }
      mhd_char_limited_slopes<D>( a.ph, LE, RE, cl, cc, cr, a.limiter, a.coeff, s );
#     pragma unroll
      for (int v=0; v<NM; v++) plm_clamped_faces( cl[v], cc[v], cr[v], s[v], fl[v], fr[v] );
   }
   else
   {
#     pragma unroll
      for (int v=0; v<NM; v++)
      {
         const R l = pri[v*NX3 + c - dcc[D]], r = pri[v*NX3 + c + dcc[D]];
         plm_faces( l, cc[v], r, a.limiter, a.coeff, true, fl[v], fr[v] );
      }
   }
}

// LR_PPM (FLU_NXT 24): PPM face values from the limited slopes of the cell and its two neighbours
// (each, with CH, limited in its own cell's MHD wave amplitudes), and the tracing of the parabola:
// each wave's correction carries the curvature term dfc6 = 6 (cc - (fL + fR)/2)
// (CPU_Shared_DataReconstruction.cpp:870-907, :1080-1290)
template <int D, int CH, int LR, typename R>
GB_DEV void ctu_recon_dir( const CtuArgs<R> &a, const R *pri, const R *bin, const R *cc,
                           int ci, int cj, int ck, R (&fcon)[2][NM] )
{
   using namespace ctu;
   typedef MDir<D> M;
   constexpr int N = ( LR == LR_PPM ) ? NX + 2 : NX, NX3 = plane_of( N ), NBIN = nbin_of( N );
   constexpr int t1 = ( D + 1 ) % 3, t2 = ( D + 2 ) % 3;
   const int dcc[3] = { 1, N, N*N };
   const int c = idx3( ci, cj, ck, N, N );
   R ev[7], LE[7][7], RE[7][7];
   mhd_eigen<D>( a.ph, cc, ev, LE, RE );
   R fl[NM], fr[NM];
   mhd_face_values<D,CH,LR>( a, pri, NX3, c, dcc[D], cc, LE, RE, fl, fr );
   // characteristic tracing with all waves (HLL solvers: HLL_NO_REF_STATE, HLL_INCLUDE_ALL_WAVES)
   const R dt_dh2 = R(0.5)*a.dt/a.dh;
   const int wv[7] = { 0, M::n, M::t1, M::t2, 4, M::b1, M::b2 };   // wave index -> storage index
   R dfc[7], corr[7], corl[7];
#  pragma unroll
   for (int q=0; q<7; q++) { dfc[q] = fr[wv[q]] - fl[wv[q]];  corr[q] = R(0);  corl[q] = R(0); }
   if constexpr ( LR == LR_PPM )
   {
      R dfc6[7];
#     pragma unroll
      for (int q=0; q<7; q++) dfc6[q] = R(6)*( cc[wv[q]] - R(0.5)*( fl[wv[q]] + fr[wv[q]] ) );
#     pragma unroll
      for (int m=0; m<7; m++)
      {
         const R cC = -dt_dh2*ev[m], cD = R(-4.0/3.0)*( cC*cC );
         R cfl = R(0), cfr = R(0);
#        pragma unroll
         for (int q=0; q<7; q++)
         {
            cfl += LE[m][q]*( cC*( dfc[q] + dfc6[q] ) + cD*dfc6[q] );
            cfr += LE[m][q]*( cC*( dfc[q] - dfc6[q] ) + cD*dfc6[q] );
         }
#        pragma unroll
         for (int q=0; q<7; q++) { corl[q] = corl[q] + mul_rn( cfl, RE[m][q] );  corr[q] = corr[q] + mul_rn( cfr, RE[m][q] ); }
      }
   }
   else
   {
#     pragma unroll
      for (int m=0; m<7; m++)
      {
         R cf = R(0);
#        pragma unroll
         for (int q=0; q<7; q++) cf += LE[m][q]*dfc[q];
         cf *= -dt_dh2*ev[m];
         // uncontracted: the Alfven pair (modes 1 and 5) cancels exactly in B_t when B = 0
#        pragma unroll
         for (int q=0; q<7; q++) corr[q] = corr[q] + mul_rn( cf, RE[m][q] );
      }
#     pragma unroll
      for (int q=0; q<7; q++) corl[q] = corr[q];
   }
   // MHD source terms of the transverse B (CPU_Shared_DataReconstruction.cpp:593-620)
   const int ib[3] = { idx_b( 0, ci, cj, ck, N ), idx_b( 1, ci, cj, ck, N ), idx_b( 2, ci, cj, ck, N ) };
   const R bnl  = bin[D*NBIN + ib[D]],   bnr  = bin[D*NBIN + ib[D] + dcc[D]];
   const R bt1l = bin[t1*NBIN + ib[t1]], bt1r = bin[t1*NBIN + ib[t1] + dcc[t1]];
   const R bt2l = bin[t2*NBIN + ib[t2]], bt2r = bin[t2*NBIN + ib[t2] + dcc[t2]];
   const R dbn = bnr - bnl, dbt1 = bt1r - bt1l, dbt2 = bt2r - bt2l;
   const R src1 = dt_dh2*cc[M::t1]*minmod2( dbn, -dbt1 ), src2 = dt_dh2*cc[M::t2]*minmod2( dbn, -dbt2 );
   corl[5] += src1;  corr[5] += src1;
   corl[6] += src2;  corr[6] += src2;
#  pragma unroll
   for (int q=0; q<7; q++) { fl[wv[q]] += corl[q];  fr[wv[q]] += corr[q]; }
   fl[0] = gmax( fl[0], a.ph.min_dens );  fr[0] = gmax( fr[0], a.ph.min_dens );
   fl[4] = check_floor( fl[4], a.ph.min_pres );  fr[4] = check_floor( fr[4], a.ph.min_pres );
   // longitudinal B from the input faces
   fl[M::bn] = bnl;  fr[M::bn] = bnr;
   mhd_pri2con( a.ph, fl, fcon[0] );
   mhd_pri2con( a.ph, fr, fcon[1] );
}

// one (cell, direction) per item: the two faces of that direction (the eigen-system of one
// direction is live at a time, which keeps the register count low)
// FP32: 4 CTAs of 256 threads per SM (64 registers, 104 bytes of spills); with characteristic
// limiting 2 CTAs (the wave projections spilled 464 bytes under 64, none under 128); FP64 uncapped
template <typename R, int P, int CH, int LR = LR_PLM>
__global__ void __launch_bounds__( 256, ( sizeof(R) == 8 ) ? 1 : ( ( CH || LR == LR_PPM ) ? 2 : 4 ) ) ctu_recon( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int N = ( LR == LR_PPM ) ? NX + 2 : NX, LRGc = flg_of( N ) - 2;
   const int d = blockIdx.y;
   PG_LOOP( f, NF3 )
   {
      const int ci = f % NF + LRGc, cj = ( f / NF ) % NF + LRGc, ck = f / ( NF*NF ) + LRGc;
      const R *pri = a.pri + (size_t)pg*NM*plane_of( N );
      const R *bin = a.bin + (size_t)pg*3*nbin_of( N );
      const int c = idx3( ci, cj, ck, N, N );
      R cc[NM], fcon[2][NM];
#     pragma unroll
      for (int v=0; v<NM; v++) cc[v] = pri[v*plane_of( N ) + c];
      if      ( d == 0 ) ctu_recon_dir<0,CH,LR>( a, pri, bin, cc, ci, cj, ck, fcon );
      else if ( d == 1 ) ctu_recon_dir<1,CH,LR>( a, pri, bin, cc, ci, cj, ck, fcon );
      else               ctu_recon_dir<2,CH,LR>( a, pri, bin, cc, ci, cj, ck, fcon );
      R *fcv = a.fcv + (size_t)pg*6*NM*NF3;
#     pragma unroll
      for (int q=0; q<2; q++)
#        pragma unroll
         for (int v=0; v<NM; v++) fcv[( ( 2*d + q )*NM + v )*NF3 + f] = fcon[q][v];
   }
}

// ---- K2/K7: Riemann fluxes (Hydro_ComputeFlux, CPU_Shared_ComputeFlux.cpp:113-376) ----------
// half step: NSkip_N = NSkip_T = 0, stride 20; full step: NSkip_N = NSkip_T = 1, stride 18
template <int D, typename R, int P>
GB_DEV void ctu_face( const CtuArgs<R> &a, int pg, int fi, int fj, int fk, int skip, int nflux, bool store_int )
{
   using namespace ctu;
   const int dfc[3] = { 1, NF, NF*NF };
   const int ifc = idx3( fi + skip, fj + skip, fk + skip, NF, NF );
   const R *fcv = a.fcv + (size_t)pg*6*NM*NF3;
   R L[NM], Rr[NM], F[NM];
#  pragma unroll
   for (int v=0; v<NM; v++) { L[v] = fcv[( ( 2*D + 1 )*NM + v )*NF3 + ifc];  Rr[v] = fcv[( 2*D*NM + v )*NF3 + ifc + dfc[D]]; }
   riemann_mhd<D,P>( a.ph, L, Rr, F );
   R *fcf = a.fcf + (size_t)pg*3*NM*NF3;
   const int ix = idx3( fi, fj, fk, nflux, nflux );
#  pragma unroll
   for (int v=0; v<NM; v++) fcf[( D*NM + v )*NF3 + ix] = F[v];
   // coarse-fine flux planes (Hydro_StoreIntFlux with MHD, CPU_Shared_ComputeFlux.cpp:391-450)
   if ( store_int && a.flux != nullptr )
   {
      const int fl[3] = { fi, fj, fk };
      const int nrm = fl[D];
      const int t1 = fl[( D + 1 ) % 3], t2 = fl[( D + 2 ) % 3];
      if ( ( nrm & 7 ) == 0 && t1 >= 1 && t1 <= PS2 && t2 >= 1 && t2 <= PS2 )
      {
         // idx_out: transverse index with the smaller axis number is the fastest
         const int a0 = ( D == 0 ) ? fj : fi, a1 = ( D == 2 ) ? fj : fk;
         const int io = ( a1 - 1 )*PS2 + ( a0 - 1 );
         R *dst = a.flux + (size_t)pg*9*5*PS2*PS2 + (size_t)( 3*D + nrm/PS1 )*5*PS2*PS2 + io;
#        pragma unroll
         for (int v=0; v<5; v++) dst[v*PS2*PS2] = F[v];
      }
   }
}

// FP32: 3 CTAs of 256 threads per SM (80 registers, no spills): MHD step 2.08 -> 1.94 ms per
// 512 PGs; FP64 keeps its registers (a cap would spill)
template <typename R, int P, int FULL>
__global__ void __launch_bounds__( 256, ( sizeof(R) == 8 ) ? 1 : 3 ) ctu_flux( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int full = FULL, skip = FULL ? 1 : 0, nflux = FULL ? NFF : NF;
   constexpr int nn = NF - 1 - 2*skip, nt = NF - 2*skip;      // faces along / across the normal
   constexpr int per = nn*nt*nt;
   PG_LOOP( q, per )
   {
#     define GB_FACE( D ) { \
         constexpr int e0 = ( D == 0 ) ? nn : nt, e1 = ( D == 1 ) ? nn : nt; \
         ctu_face<D,R,P>( a, pg, q % e0, ( q / e0 ) % e1, q / ( e0*e1 ), skip, nflux, full ); }
      GB_CTU_DIR( GB_FACE )
#     undef GB_FACE
   }
}

// ---- K3/K8: edge EMFs (MHD_ComputeElectric + dE_Upwind, CPU_Shared_ConstrainedTransport.cpp:90-432) ----
template <typename R>
GB_DEV R de_upwind( R fe_l, R fe_r, R fmom, R dl, R dr, R vl1, R vl2, R vr1, R vr2,
                    R bl1, R bl2, R br1, R br2, R dt_dh )
{
   const R maxerr = ( sizeof(R) == 8 ) ? R(1.0e-14) : R(1.0e-06);
   const R fv = R(2)*dt_dh*fmom/( dl + dr );
   if ( gabs( fv ) <= maxerr )
   {
      const R er = br1*vr2 - br2*vr1, el = bl1*vl2 - bl2*vl1;
      return R(0.5)*( fe_r - er + fe_l - el );
   }
   if ( fv > R(0) ) return fe_l - ( bl1*vl2 - bl2*vl1 );
   return fe_r - ( br1*vr2 - br2*vr1 );
}

// G (geometry) 0, CTU half step: NEle 19, NFlux 20, primitives of the input (stride 22, offset 1);
// G 1, full step of CTU and MHM_RP: NEle 17, NFlux 18, half-step primitives (stride 18, offset 0),
// Ele planes dumped; G 2, MHM_RP half step: NEle NXI - 1, NFlux NXI (the half-step fluxes, stored in
// the face-state region), primitives of the input (stride NXI, offset 0), EMF components of stride
// (NXI - 1)^3
// NXI: FLU_NXT of the input (22, or 24 with PPM; 20 for MHM's full step): the `pri` planes
template <int d, typename R, int G, int NXI = ctu::NX>
GB_DEV void ctu_emf_dir( const CtuArgs<R> &a, int pg, int q )
{
   using namespace ctu;
   constexpr int nele = ( G == 1 ) ? NFE : ( G == 0 ) ? NHE : NXI - 1;
   constexpr int nflux = ( G == 1 ) ? NFF : ( G == 0 ) ? NF : NXI, npri = ( G == 1 ) ? NHV : NXI;
   constexpr int off_pri = ( G == 0 ) ? flg_of( NXI ) - 2 : 0, pri_plane = plane_of( NXI ), dump = ( G == 1 );
   constexpr int fplane = ( G == 2 ) ? NXI*NXI*NXI : NF3, eplane = ( G == 2 ) ? ( NXI - 1 )*( NXI - 1 )*( NXI - 1 ) : NEC;
   constexpr int T1 = ( d + 1 ) % 3, T2 = ( d + 2 ) % 3;
   constexpr int TV1 = 1 + T1, TV2 = 1 + T2, TB1 = MO + T1, TB2 = MO + T2;
   constexpr int ex0 = ( d == 0 ) ? nele - 1 : nele, ex1 = ( d == 1 ) ? nele - 1 : nele;
   const R dt_dh = a.dt/a.dh;
   {
      const int ie = q % ex0, je = ( q / ex0 ) % ex1, ke = q / ( ex0*ex1 );
      constexpr int sf[3] = { d == 0, d == 1, d == 2 };
      const int ifl = idx3( ie + sf[0], je + sf[1], ke + sf[2], nflux, nflux );
      const int ip  = idx3( ie + sf[0] + off_pri, je + sf[1] + off_pri, ke + sf[2] + off_pri, npri, npri );
      const int dfl[3] = { 1, nflux, nflux*nflux }, dpr[3] = { 1, npri, npri*npri };
      const R *F = ( G == 2 ) ? a.fcv + (size_t)pg*6*NM*NF3 : a.fcf + (size_t)pg*3*NM*NF3;
      const R *W = a.pri + (size_t)pg*NM*pri_plane;
      auto f = [&]( int dir, int v, int idx ) { return F[( dir*NM + v )*fplane + idx]; };
      auto w = [&]( int v, int idx ) { return W[v*pri_plane + idx]; };
      R E = ( -f( T1, TB2, ifl + dfl[T2] ) - f( T1, TB2, ifl ) + f( T2, TB1, ifl + dfl[T1] ) + f( T2, TB1, ifl ) );
      int il, ir;
      il = ip;  ir = il + dpr[T2];
      E += de_upwind( -f( T1, TB2, ifl ), -f( T1, TB2, ifl + dfl[T2] ), f( T2, 0, ifl ),
                      w( 0, il ), w( 0, ir ), w( TV1, il ), w( TV2, il ), w( TV1, ir ), w( TV2, ir ),
                      w( TB1, il ), w( TB2, il ), w( TB1, ir ), w( TB2, ir ), dt_dh );
      il = ip + dpr[T1];  ir = il + dpr[T2];
      E += de_upwind( -f( T1, TB2, ifl ), -f( T1, TB2, ifl + dfl[T2] ), f( T2, 0, ifl + dfl[T1] ),
                      w( 0, il ), w( 0, ir ), w( TV1, il ), w( TV2, il ), w( TV1, ir ), w( TV2, ir ),
                      w( TB1, il ), w( TB2, il ), w( TB1, ir ), w( TB2, ir ), dt_dh );
      il = ip;  ir = il + dpr[T1];
      E += de_upwind( f( T2, TB1, ifl ), f( T2, TB1, ifl + dfl[T1] ), f( T1, 0, ifl ),
                      w( 0, il ), w( 0, ir ), w( TV1, il ), w( TV2, il ), w( TV1, ir ), w( TV2, ir ),
                      w( TB1, il ), w( TB2, il ), w( TB1, ir ), w( TB2, ir ), dt_dh );
      il = ip + dpr[T2];  ir = il + dpr[T1];
      E += de_upwind( f( T2, TB1, ifl ), f( T2, TB1, ifl + dfl[T1] ), f( T1, 0, ifl + dfl[T2] ),
                      w( 0, il ), w( 0, ir ), w( TV1, il ), w( TV2, il ), w( TV1, ir ), w( TV2, ir ),
                      w( TB1, il ), w( TB2, il ), w( TB1, ir ), w( TB2, ir ), dt_dh );
      E *= R(0.25);
      R *ec = a.ec + (size_t)pg*a.ec_pg;
      ec[d*eplane + idx3( ie, je, ke, nele, nele )] = E;
      // coarse-fine EMF planes (CPU_Shared_ConstrainedTransport.cpp:348-369)
      if ( dump && a.ele != nullptr )
      {
         R *g = a.ele + (size_t)pg*9*2*NELE;
         auto put = [&]( int plane, int comp, int idx ) { g[( plane*2 + comp )*NELE + idx] = E; };
         if ( d == 0 ) {
            if ( ( je & 7 ) == 0 ) put( 3 + je/PS1, 1, ie*( PS2 + 1 ) + ke );
            if ( ( ke & 7 ) == 0 ) put( 6 + ke/PS1, 0, je*PS2 + ie );
         } else if ( d == 1 ) {
            if ( ( ke & 7 ) == 0 ) put( 6 + ke/PS1, 1, je*( PS2 + 1 ) + ie );
            if ( ( ie & 7 ) == 0 ) put( 0 + ie/PS1, 0, ke*PS2 + je );
         } else {
            if ( ( ie & 7 ) == 0 ) put( 0 + ie/PS1, 1, ke*( PS2 + 1 ) + je );
            if ( ( je & 7 ) == 0 ) put( 3 + je/PS1, 0, ie*PS2 + ke );
         }
      }
   }
}

template <typename R, int G, int NXI = ctu::NX>
__global__ void ctu_emf( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int nele = ( G == 1 ) ? NFE : ( G == 0 ) ? NHE : NXI - 1;
   PG_LOOP( q, ( nele - 1 )*nele*nele )
   {
#     define GB_EMF( D ) ctu_emf_dir<D,R,G,NXI>( a, pg, q )
      GB_CTU_DIR( GB_EMF )
#     undef GB_EMF
   }
}

// ---- K4/K9: CT update of the face-centred B (MHD_UpdateMagnetic, CPU_Shared_ConstrainedTransport.cpp:529-590) ----
// G 0, CTU half step: B_half (18 cells + 1 face, EMFs of stride 19, input offset 2) over dt/2;
// G 1, full step: Mag_Out (16 cells + 1 face, EMFs of stride 17, input offset 3) over dt;
// G 2, MHM_RP half step: B_half (NXI - 2 cells + 1 face, EMFs of stride NXI - 1, input offset 1) over dt/2;
// G 3, MHM full step: Mag_Out (16 cells + 1 face, EMFs of stride 17) from the 20^3 input at offset 2
template <typename R, int G, int NXI = ctu::NX>
__global__ void ctu_bupdate( const __grid_constant__ CtuArgs<R> a, R *bout_base, size_t bout_pg_stride, int bout_comp_stride,
                             R dt )
{
   using namespace ctu;
   constexpr int nout = ( G == 1 || G == 3 ) ? PS2 : ( G == 0 ) ? NHV : NXI - 2;
   constexpr int nele = ( G == 1 || G == 3 ) ? NFE : ( G == 0 ) ? NHE : NXI - 1;
   constexpr int nin = ( G == 3 ) ? MNX : NXI, nbin = nbin_of( nin );
   constexpr int off_in = ( G == 1 || G == 3 ) ? flg_of( nin ) : ( G == 0 ) ? flg_of( nin ) - 1 : 1;
   constexpr int eplane = ( G == 2 ) ? ( NXI - 1 )*( NXI - 1 )*( NXI - 1 ) : NEC;
   constexpr int per = ( nout + 1 )*nout*nout;
   const R dt_dh = dt/a.dh;
   PG_LOOP( q, per )
   {
#     define GB_BUP( D ) { \
         constexpr int d = D, T1 = ( d + 1 ) % 3, T2 = ( d + 2 ) % 3; \
         constexpr int e0 = ( d == 0 ) ? nout + 1 : nout, e1 = ( d == 1 ) ? nout + 1 : nout; \
         const int io = q % e0, jo = ( q / e0 ) % e1, ko = q / ( e0*e1 ); \
         const int ie = idx3( io, jo, ko, nele, nele ); \
         constexpr int de[3] = { 1, nele, nele*nele }; \
         const R *ec = a.ec + (size_t)pg*a.ec_pg; \
         const R dE1 = ec[T1*eplane + ie + de[T2]] - ec[T1*eplane + ie]; \
         const R dE2 = ec[T2*eplane + ie + de[T1]] - ec[T2*eplane + ie]; \
         const R *bin = a.bin + (size_t)pg*3*nbin; \
         const int iin = idx_b( d, io + off_in, jo + off_in, ko + off_in, nin ); \
         bout_base[pg*bout_pg_stride + (size_t)d*bout_comp_stride + q] = bin[d*nbin + iin] + dt_dh*( dE1 - dE2 ); }
      GB_CTU_DIR( GB_BUP )
#     undef GB_BUP
   }
}

// ---- K5: transverse-gradient correction (Hydro_TGradientCorrection, CPU_FluidSolver_CTU.cpp:368-599) ----
template <int D, typename R, int P, int NXI = ctu::NX>
GB_DEV void ctu_tgrad_dir( const CtuArgs<R> &a, int pg, int i0, int j0, int k0 )
{
   using namespace ctu;
   typedef MDir<D> M;
   constexpr int T1 = ( D + 1 ) % 3, T2 = ( D + 2 ) % 3;
   const int dfl[3] = { 1, NF, NF*NF };
   const int f = idx3( i0 + 1, j0 + 1, k0 + 1, NF, NF );
   R *fcv = a.fcv + (size_t)pg*6*NM*NF3;
   const R *F = a.fcf + (size_t)pg*3*NM*NF3;
   const R dt_dh2 = R(0.5)*a.dt/a.dh;
   R q0[NM], q1[NM];
#  pragma unroll
   for (int v=0; v<NM; v++) { q0[v] = fcv[( 2*D*NM + v )*NF3 + f];  q1[v] = fcv[( ( 2*D + 1 )*NM + v )*NF3 + f]; }
#  pragma unroll
   for (int v=0; v<5; v++)
   {
      const R tg1 = F[( T1*NM + v )*NF3 + f] - F[( T1*NM + v )*NF3 + f - dfl[T1]];
      const R tg2 = F[( T2*NM + v )*NF3 + f] - F[( T2*NM + v )*NF3 + f - dfl[T2]];
      const R c = -dt_dh2*( tg1 + tg2 );
      q0[v] += c;  q1[v] += c;
   }
   // transverse B corrections from the half-step EMFs
   const R idh = R(1)/a.dh, dt_dh4 = R(0.25)*a.dt*idh, dt_2 = R(0.5)*a.dt;
   const R *ec = a.ec + (size_t)pg*a.ec_pg;
   const int ie = idx3( i0, j0, k0, NHE, NHE );
   const int de[3] = { 1, NHE, NHE*NHE };
#  pragma unroll
   for (int v=1; v<3; v++)
   {
      const int TD1 = ( D + v ) % 3, TD2 = ( D + 2*v ) % 3, TB = MO + TD1;
      const R tg1 = ec[D*NEC + ie + de[TD2]] - ec[D*NEC + ie];
      const R tg2 = ec[D*NEC + ie + de[TD2] + de[TD1]] - ec[D*NEC + ie + de[TD1]];
      const R c = R(2*v - 3)*dt_dh4*( tg2 + tg1 );
      q0[TB] += c;  q1[TB] += c;
   }
   // MHD source terms of the longitudinal-B divergence (CPU_FluidSolver_CTU.cpp:520-560)
   constexpr int LRGc = flg_of( NXI ) - 2, PL = plane_of( NXI ), NB = nbin_of( NXI );
   const int ci = i0 + 1 + LRGc, cj = j0 + 1 + LRGc, ck = k0 + 1 + LRGc;
   const R *W = a.pri + (size_t)pg*NM*PL;
   const int ip = idx3( ci, cj, ck, NXI, NXI );
   const R Vy = W[M::t1*PL + ip], Vz = W[M::t2*PL + ip];
   const R Bx = W[M::bn*PL + ip], By = W[M::b1*PL + ip], Bz = W[M::b2*PL + ip];
   const R *bin = a.bin + (size_t)pg*3*NB;
   const int dirs[3] = { D, T1, T2 };
   R dB[3];
#  pragma unroll
   for (int v=0; v<3; v++)
   {
      const int dd = dirs[v];
      const int ib = idx_b( dd, ci, cj, ck, NXI );
      dB[v] = ( bin[dd*NB + ib + db_next( dd, NXI )] - bin[dd*NB + ib] )*idh;
   }
   const R vy_mm = Vy*minmod2( -dB[2], dB[0] );
   const R vz_mm = Vz*minmod2( -dB[1], dB[0] );
   const R s1 = dt_2*Bx*dB[0], s2 = dt_2*By*dB[0], s3 = dt_2*Bz*dB[0];
   const R s4 = dt_2*( By*vy_mm + Bz*vz_mm );
   const R m1 = dt_2*vy_mm, m2 = dt_2*vz_mm;
   q0[M::n] += s1;  q0[M::t1] += s2;  q0[M::t2] += s3;  q0[4] += s4;  q0[M::b1] += m1;  q0[M::b2] += m2;
   q1[M::n] += s1;  q1[M::t1] += s2;  q1[M::t2] += s3;  q1[4] += s4;  q1[M::b1] += m1;  q1[M::b2] += m2;
   // longitudinal B from the half-step faces
   const R *bh = a.bh + (size_t)pg*3*NBH;
   const int ih = idx_b( D, i0, j0, k0, NHV );
   q0[M::bn] = bh[D*NBH + ih];
   q1[M::bn] = bh[D*NBH + ih + db_next( D, NHV )];
   // floors
   q0[0] = gmax( q0[0], a.ph.min_dens );  q1[0] = gmax( q1[0], a.ph.min_dens );
   {
      const R em0 = emag_of( q0 ), em1 = emag_of( q1 );
      R e;
      e = eint_con_mhd<P>( q0[0], R(1)/q0[0], q0[1], q0[2], q0[3], q0[4], em0 );
      if ( e == e && e < a.ph.min_eint ) q0[4] = q0[4] - e + a.ph.min_eint;
      e = eint_con_mhd<P>( q1[0], R(1)/q1[0], q1[1], q1[2], q1[3], q1[4], em1 );
      if ( e == e && e < a.ph.min_eint ) q1[4] = q1[4] - e + a.ph.min_eint;
   }
#  pragma unroll
   for (int v=0; v<NM; v++) { fcv[( 2*D*NM + v )*NF3 + f] = q0[v];  fcv[( ( 2*D + 1 )*NM + v )*NF3 + f] = q1[v]; }
}

// FP32: 4 CTAs of 256 threads per SM (64 registers, no spills); FP64 uncapped
template <typename R, int P, int NXI = ctu::NX>
__global__ void __launch_bounds__( 256, ( sizeof(R) == 8 ) ? 1 : 4 ) ctu_tgrad( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int N3 = NHV*NHV*NHV;
   PG_LOOP( q, N3 )
   {
      const int i0 = q % NHV, j0 = ( q / NHV ) % NHV, k0 = q / ( NHV*NHV );
#     define GB_TG( D ) ctu_tgrad_dir<D,R,P,NXI>( a, pg, i0, j0, k0 )
      GB_CTU_DIR( GB_TG )
#     undef GB_TG
   }
}

// ---- K6: half-step cell-centred primitives (MHD_HalfStepPrimitive, CPU_Shared_ConstrainedTransport.cpp:629-700) ----
template <typename R, int NXI = ctu::NX>
__global__ void ctu_halfprim( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int N3 = NHV*NHV*NHV;
   const R dt_dh2 = R(0.5)*a.dt/a.dh;
   PG_LOOP( q, N3 )
   {
      const int io = q % NHV, jo = ( q / NHV ) % NHV, ko = q / ( NHV*NHV );
      const int ifl = idx3( io + 1, jo + 1, ko + 1, NF, NF );
      const int dfl[3] = { 1, NF, NF*NF };
      constexpr int G1 = flg_of( NXI ) - 1, NI3 = NXI*NXI*NXI;
      const int iin = idx3( io + G1, jo + G1, ko + G1, NXI, NXI );
      const R *F = a.fcf + (size_t)pg*3*NM*NF3;
      const R *u = a.in + (size_t)pg*5*NI3;
      R o[4];
#     pragma unroll
      for (int v=0; v<4; v++)
      {
         R df[3];
#        pragma unroll
         for (int d=0; d<3; d++) df[d] = F[( d*NM + v )*NF3 + ifl] - F[( d*NM + v )*NF3 + ifl - dfl[d]];
         o[v] = u[v*NI3 + iin] - dt_dh2*( df[0] + df[1] + df[2] );
      }
      o[0] = gmax( o[0], a.ph.min_dens );
      const R ir = R(1)/o[0];
      o[1] *= ir;  o[2] *= ir;  o[3] *= ir;
      const R *bh = a.bh + (size_t)pg*3*NBH;
      R *W = a.pri + (size_t)pg*NM*plane_of( NXI );
#     pragma unroll
      for (int v=0; v<4; v++) W[v*plane_of( NXI ) + q] = o[v];
#     pragma unroll
      for (int d=0; d<3; d++)
      {
         const int ib = idx_b( d, io, jo, ko, NHV );
         W[( MO + d )*plane_of( NXI ) + q] = R(0.5)*( bh[d*NBH + ib] + bh[d*NBH + ib + db_next( d, NHV )] );
      }
   }
}

// ---- K10: full-step update (Hydro_FullStepUpdate with MHD, CPU_Shared_FullStepUpdate.cpp:64-271) ----
// NXI: FLU_NXT of the input (22, FLU_GHOST_SIZE 3: CTU and MHM_RP; 20, ghost 2: MHM)
// Hydro_IsUnphysical, UNPHY_MODE_CONS, EOS_GAMMA, with MHD (CPU_Shared_FluUtility.cpp:843-960): each
// test is written as the range a physical value lies in, so that a NaN fails it
template <int P, typename R>
GB_DEV bool is_unphysical_mhd( const R (&u)[5], R emag )
{
   bool ok = true;
#  pragma unroll
   for (int v=0; v<5; v++)
   {
      if ( v >= 1 && v <= 3 ) ok &= ( u[v] >= -Lim<R>::huge() && u[v] <= Lim<R>::huge() );
      else                    ok &= ( u[v] > R(0) && u[v] <= Lim<R>::huge() );
   }
   const R ei = eint_con_mhd<P>( u[0], R(1)/u[0], u[1], u[2], u[3], u[4], emag );
   ok &= ( ei >= R(-3)*u[4]*Lim<R>::eps() && ei <= Lim<R>::huge() );
   ok &= ( emag >= R(0) && emag <= Lim<R>::huge() );
   return !ok;
}

template <typename R, int P, int NXI = ctu::NX>
__global__ void ctu_update( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   typedef typename std::conditional<P == P_MIXED, double, R>::type A;
   constexpr int N3 = PS2*PS2*PS2, NXU = NXI, NXU3 = NXU*NXU*NXU, FLU = ( NXU - PS2 )/2;
   const A dt_dh = (A)a.dt/(A)a.dh;
   PG_LOOP( q, N3 )
   {
      const int io = q % PS2, jo = ( q / PS2 ) % PS2, ko = q / ( PS2*PS2 );
      const int ifl = idx3( io + 1, jo + 1, ko + 1, NFF, NFF );
      const int dfl[3] = { 1, NFF, NFF*NFF };
      const int iin = idx3( io + FLU, jo + FLU, ko + FLU, NXU, NXU );
      const R *F = a.fcf + (size_t)pg*3*NM*NF3;
      const R *u = a.in + (size_t)pg*5*NXU3;
      R *out = a.out + (size_t)pg*5*N3;
      R o[5];
#     pragma unroll
      for (int v=0; v<5; v++)
      {
         A df[3];
#        pragma unroll
         for (int d=0; d<3; d++) df[d] = (A)F[( d*NM + v )*NF3 + ifl] - (A)F[( d*NM + v )*NF3 + ifl - dfl[d]];
         o[v] = (R)( (A)u[v*NXU3 + iin] - dt_dh*( df[0] + df[1] + df[2] ) );
         out[v*N3 + q] = o[v];
      }
      // the MinMod retry test of the MHM schemes (Hydro_FullStepUpdate, CPU_Shared_FullStepUpdate.cpp:
      // 209-234): Hydro_IsUnphysical in UNPHY_MODE_CONS with the magnetic energy of the updated
      // face B, cell-centred (MHD_GetCellCenteredBEnergy)
      if ( a.fail_next != nullptr )
      {
         const R *bo = a.bout + (size_t)pg*3*NBOUT;
         R b[3];
#        pragma unroll
         for (int d=0; d<3; d++)
         {
            const int ib = idx_b( d, io, jo, ko, PS2 );
            b[d] = R(0.5)*( bo[d*NBOUT + ib] + bo[d*NBOUT + ib + db_next( d, PS2 )] );
         }
         const R emag = R(0.5)*( b[0]*b[0] + b[1]*b[1] + b[2]*b[2] );
         if ( is_unphysical_mhd<P>( o, emag ) ) a.fail_next[pg] = 1;
      }
   }
}

// ---------------------------------------------------------------------------------------------
// MHM_RP with MHD (CPU_FluidSolver_MHM.cpp:396-565): the half step is a first-order Riemann
// predictor with its own constrained-transport update; the full step reuses the CTU full-step
// kernels, which see the same faces, edges and half-step cells (N_FL_FLUX 18, N_FL_ELE 17, the
// central 18^3 half-step primitives).  Scratch use per patch group: `pri` the cell-centred input
// primitives (22^3), later the central half-step primitives (stride 18); the face-state region
// first holds the half-step fluxes [3][8][22^3]; the flux region first holds the half-step
// primitives [8][20^3]; `bh` the half-step B (21 x 20 x 20 per component); `ec` the EMFs.
// ---------------------------------------------------------------------------------------------

// Hydro_RiemannPredict_Flux with MHD (CPU_FluidSolver_MHM.cpp:615-790): first-order fluxes between
// the input cells c and c + e_D, the longitudinal B from the input face between them and the
// total energy corrected by the difference of its square and the cell-centred one's, the
// transverse B cell-centred; flux stored at the index of the left cell (stride 22)
template <int D, typename R, int P, int NXI>
GB_DEV void rp_half_face( const CtuArgs<R> &a, int pg, int i, int j, int k )
{
   using namespace ctu;
   constexpr int T1 = ( D + 1 ) % 3, T2 = ( D + 2 ) % 3;
   constexpr int NX = NXI, NX3 = NXI*NXI*NXI, NBIN = nbin_of( NXI );
   const int dc[3] = { 1, NX, NX*NX };
   const int c = idx3( i, j, k, NX, NX ), cr = c + dc[D];
   const R *u = a.in + (size_t)pg*5*NX3;
   const R *W = a.pri + (size_t)pg*NM*plane_of( NXI );
   const R *bin = a.bin + (size_t)pg*3*NBIN;
   R L[NM], Rr[NM], F[NM];
#  pragma unroll
   for (int v=0; v<5; v++) { L[v] = u[v*NX3 + c];  Rr[v] = u[v*NX3 + cr]; }
   const R bn = bin[D*NBIN + idx_b( D, i, j, k, NX ) + db_next( D, NX )];
   L[MO + D] = bn;  Rr[MO + D] = bn;
   L[MO + T1] = W[( MO + T1 )*NX3 + c];   L[MO + T2] = W[( MO + T2 )*NX3 + c];
   Rr[MO + T1] = W[( MO + T1 )*NX3 + cr]; Rr[MO + T2] = W[( MO + T2 )*NX3 + cr];
   const R bl = W[( MO + D )*NX3 + c], br = W[( MO + D )*NX3 + cr];
   L[4]  += R(0.5)*( bn*bn - bl*bl );
   Rr[4] += R(0.5)*( bn*bn - br*br );
   riemann_mhd<D,P>( a.ph, L, Rr, F );
   R *fh = a.fcv + (size_t)pg*6*NM*NF3;
#  pragma unroll
   for (int v=0; v<NM; v++) fh[( D*NM + v )*NX3 + c] = F[v];
}

template <typename R, int P, int NXI>
__global__ void __launch_bounds__( 256, ( sizeof(R) == 8 ) ? 1 : 3 ) rp_half_flux( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   PG_LOOP( q, ( NXI - 1 )*NXI*NXI )
   {
#     define GB_RPF( D ) { \
         constexpr int e0 = ( D == 0 ) ? NXI - 1 : NXI, e1 = ( D == 1 ) ? NXI - 1 : NXI; \
         rp_half_face<D,R,P,NXI>( a, pg, q % e0, ( q / e0 ) % e1, q / ( e0*e1 ) ); }
      GB_CTU_DIR( GB_RPF )
#     undef GB_RPF
   }
}

// Hydro_RiemannPredict with MHD (CPU_FluidSolver_MHM.cpp:828-948): the input cell (i+1, j+1, k+1)
// advanced by half a step with the half-step fluxes, its B the average of the half-step faces,
// density and internal-energy floors (Hydro_CheckMinEintInEngy, CPU_Shared_FluUtility.cpp:787-804),
// then conserved -> primitive; stored [8][(NXI - 2)^3] in the flux region
template <typename R, int P, int NXI>
__global__ void rp_predict( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int NX = NXI, NX3 = NXI*NXI*NXI, HV = NXI - 2, HV3 = HV*HV*HV, HNB = ( HV + 1 )*HV*HV;
   PG_LOOP( q, HV3 )
   {
      const int io = q % HV, jo = ( q / HV ) % HV, ko = q / ( HV*HV );
      const int c = idx3( io + 1, jo + 1, ko + 1, NX, NX );
      const int dc[3] = { 1, NX, NX*NX };
      const R *fh = a.fcv + (size_t)pg*6*NM*NF3;
      const R *u = a.in + (size_t)pg*5*NX3;
      const R dt_dh2 = R(0.5)*a.dt/a.dh;
      R cu[NM];
#     pragma unroll
      for (int v=0; v<5; v++)
      {
         R df[3];
#        pragma unroll
         for (int d=0; d<3; d++) df[d] = fh[( d*NM + v )*NX3 + c] - fh[( d*NM + v )*NX3 + c - dc[d]];
         cu[v] = u[v*NX3 + c] - dt_dh2*( df[0] + df[1] + df[2] );
      }
      const R *bh = a.bh + (size_t)pg*3*HNB;
#     pragma unroll
      for (int d=0; d<3; d++)
      {
         const int ib = idx_b( d, io, jo, ko, HV );
         cu[MO + d] = R(0.5)*( bh[d*HNB + ib] + bh[d*HNB + ib + db_next( d, HV )] );
      }
      cu[0] = gmax( cu[0], a.ph.min_dens );
      {
         const R e = eint_con_mhd<P>( cu[0], R(1)/cu[0], cu[1], cu[2], cu[3], cu[4], emag_of( cu ) );
         const R eo = gmax( e, a.ph.min_eint );
         if ( !( e == eo ) ) cu[4] = cu[4] - e + eo;
      }
      R w[NM];
      mhd_con2pri<P>( a.ph, cu, w );
      if ( a.ph.jeans ) w[4] = check_floor( w[4], a.ph.jeans_coeff*( w[0]*w[0] ) );
      R *hp = a.fcf + (size_t)pg*3*NM*NF3;
#     pragma unroll
      for (int v=0; v<NM; v++) hp[v*HV3 + q] = w[v];
   }
}

// Hydro_DataReconstruction (PLM) of MHM_RP with MHD (CPU_Shared_DataReconstruction.cpp:386-657): the
// face values of half-step cell (hi, hj, hk) along D, limited in primitive or (CH) characteristic
// variables, clamped between the neighbours, the longitudinal B from the half-step faces, then
// primitive -> conserved; no tracing
template <int D, int CH, int LR, typename R>
GB_DEV void rp_recon_dir( const CtuArgs<R> &a, const R *hp, const R *bh, int hi, int hj, int hk, const R *cc,
                          R (&fcon)[2][NM] )
{
   using namespace ctu;
   typedef MDir<D> M;
   constexpr int HV = ( LR == LR_PPM ) ? RHV + 2 : RHV, HV3 = HV*HV*HV, NBH_ = ( HV + 1 )*HV*HV;
   const int dh3[3] = { 1, HV, HV*HV };
   const int c = idx3( hi, hj, hk, HV, HV );
   R fl[NM], fr[NM];
   R ev[7], LE[7][7], RE[7][7];
   if constexpr ( CH ) mhd_eigen<D>( a.ph, cc, ev, LE, RE );
   mhd_face_values<D,CH,LR>( a, hp, HV3, c, dh3[D], cc, LE, RE, fl, fr );
   const int ib = idx_b( D, hi, hj, hk, HV );
   fl[M::bn] = bh[D*NBH_ + ib];
   fr[M::bn] = bh[D*NBH_ + ib + db_next( D, HV )];
   mhd_pri2con( a.ph, fl, fcon[0] );
   mhd_pri2con( a.ph, fr, fcon[1] );
}

// one (face-state cell, direction) per item: the face states go to the CTU layout (cells 1..18 of
// the 20^3 grid, where the full-step flux kernel reads them), and the direction-0 item of each cell
// copies its half-step primitives to `pri` (stride 18) for the full-step EMFs.  PLM: the half-step
// state is 20^3 and face-state cell i its cell i + 1; PPM: 22^3 and i + 2
template <typename R, int P, int CH, int LR = LR_PLM>
__global__ void __launch_bounds__( 256, ( sizeof(R) == 8 ) ? 1 : ( ( CH || LR == LR_PPM ) ? 2 : 4 ) ) rp_recon( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int HV = ( LR == LR_PPM ) ? RHV + 2 : RHV, HV3 = HV*HV*HV, NBH_ = ( HV + 1 )*HV*HV;
   constexpr int OFF = ( LR == LR_PPM ) ? 2 : 1, NXI = HV + 2;
   const int d = blockIdx.y;
   PG_LOOP( f, NFF*NFF*NFF )
   {
      const int i = f % NFF, j = ( f / NFF ) % NFF, k = f / ( NFF*NFF );
      const R *hp = a.fcf + (size_t)pg*3*NM*NF3;
      const R *bh = a.bh + (size_t)pg*3*NBH_;
      const int c = idx3( i + OFF, j + OFF, k + OFF, HV, HV );
      R cc[NM], fcon[2][NM];
#     pragma unroll
      for (int v=0; v<NM; v++) cc[v] = hp[v*HV3 + c];
      if      ( d == 0 ) rp_recon_dir<0,CH,LR>( a, hp, bh, i + OFF, j + OFF, k + OFF, cc, fcon );
      else if ( d == 1 ) rp_recon_dir<1,CH,LR>( a, hp, bh, i + OFF, j + OFF, k + OFF, cc, fcon );
      else               rp_recon_dir<2,CH,LR>( a, hp, bh, i + OFF, j + OFF, k + OFF, cc, fcon );
      R *fcv = a.fcv + (size_t)pg*6*NM*NF3;
      const int fo = idx3( i + 1, j + 1, k + 1, NF, NF );
#     pragma unroll
      for (int q=0; q<2; q++)
#        pragma unroll
         for (int v=0; v<NM; v++) fcv[( ( 2*d + q )*NM + v )*NF3 + fo] = fcon[q][v];
      if ( d == 0 )
      {
         R *W = a.pri + (size_t)pg*NM*plane_of( NXI );
#        pragma unroll
         for (int v=0; v<NM; v++) W[v*plane_of( NXI ) + f] = cc[v];
      }
   }
}

// ---------------------------------------------------------------------------------------------
// MHM with MHD (CPU_FluidSolver_MHM.cpp:489-565 with Hydro_DataReconstruction's MHD branch): a
// half-step EMF from the input cells, the PLM face states with the Hancock predictor (MHD fluxes)
// and the half-step update of their face B, the half-step cell primitives as the average of the
// six face states; then the CTU full-step kernels.  FLU_NXT 20: `pri` holds the input primitives
// (planes of 20^3), `bh` the half-step primitives of the 18^3 face-state cells (planes of 22^3, the
// stride the full-step EMF kernel reads), `ec` the half-step then the full-step EMFs.
// ---------------------------------------------------------------------------------------------

// stride of one cell along axis `dir` in the face-centred array of component c (n^3 cell grid)
GB_DEV int fb_stride( int c, int dir, int n )
{
   int st = 1;
   for (int q=0; q<dir; q++) st *= n + ( q == c );
   return st;
}

// MHD_ComputeElectric_Half (CPU_Shared_ConstrainedTransport.cpp:729-835): E_d at the lower edge of
// input cell (i+1, j+1, k+1) from the transverse velocities averaged over the four cells around the
// edge and the transverse B averaged over the two faces on it; 18 x 19 x 19 edges per direction
template <int d, typename R, int NXI>
GB_DEV void mm_emf_half_dir( const CtuArgs<R> &a, int pg, int q )
{
   using namespace ctu;
   constexpr int N = NXI, NE = NHE, N3 = N*N*N, NB = nbin_of( N ), OFF = flg_of( N ) - 1;   // OffsetCon = LR ghost
   constexpr int T1 = ( d + 1 ) % 3, T2 = ( d + 2 ) % 3;
   constexpr int ex0 = ( d == 0 ) ? NE - 1 : NE, ex1 = ( d == 1 ) ? NE - 1 : NE;
   const int ie = q % ex0, je = ( q / ex0 ) % ex1, ke = q / ( ex0*ex1 );
   const int ic = ie + OFF, jc = je + OFF, kc = ke + OFF;
   const int dc[3] = { 1, N, N*N };
   const int c = idx3( ic, jc, kc, N, N );
   const int cm[4] = { c, c - dc[T1], c - dc[T2], c - dc[T1] - dc[T2] };
   const R *u = a.in + (size_t)pg*5*N3;
   R V1 = R(0), V2 = R(0);
#  pragma unroll
   for (int m=0; m<4; m++) { V1 += u[( 1 + T1 )*N3 + cm[m]]/u[cm[m]];  V2 += u[( 1 + T2 )*N3 + cm[m]]/u[cm[m]]; }
   V1 *= R(0.25);  V2 *= R(0.25);
   const R *b = a.bin + (size_t)pg*3*NB;
   const int ib1 = idx_b( T1, ic, jc, kc, N ), ib2 = idx_b( T2, ic, jc, kc, N );
   const R B1 = R(0.5)*( b[T1*NB + ib1 - fb_stride( T1, T2, N )] + b[T1*NB + ib1] );
   const R B2 = R(0.5)*( b[T2*NB + ib2 - fb_stride( T2, T1, N )] + b[T2*NB + ib2] );
   R *ec = a.ec + (size_t)pg*a.ec_pg;
   ec[d*NEC + idx3( ie, je, ke, NE, NE )] = B1*V2 - B2*V1;
}

template <typename R, int NXI>
__global__ void mm_emf_half( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   PG_LOOP( q, ( NHE - 1 )*NHE*NHE )
   {
#     define GB_MME( D ) mm_emf_half_dir<D,R,NXI>( a, pg, q )
      GB_CTU_DIR( GB_MME )
#     undef GB_MME
   }
}

// PLM face states of face-state cell (i, j, k) along D (primitive or, CH, characteristic limiting),
// the normal B from the input faces (CPU_Shared_DataReconstruction.cpp:386-657)
template <int D, int CH, int LR, typename R>
GB_DEV void mm_faces_dir( const CtuArgs<R> &a, const R *pri, const R *bin, const R *cc, int ic, int jc, int kc,
                          R (&wl)[NM], R (&wr)[NM] )
{
   using namespace ctu;
   typedef MDir<D> M;
   constexpr int N = ( LR == LR_PPM ) ? MNX + 2 : MNX, PL = ( N == MNX ) ? MNX3 : plane_of( N ), NB = nbin_of( N );
   const int dcc[3] = { 1, N, N*N };
   const int c = idx3( ic, jc, kc, N, N );
   R ev[7], LE[7][7], RE[7][7];
   if constexpr ( CH ) mhd_eigen<D>( a.ph, cc, ev, LE, RE );
   mhd_face_values<D,CH,LR>( a, pri, PL, c, dcc[D], cc, LE, RE, wl, wr );
   const int ib = idx_b( D, ic, jc, kc, N );
   wl[M::bn] = bin[D*NB + ib];
   wr[M::bn] = bin[D*NB + ib + db_next( D, N )];
}

// MHD flux of a conserved face state along D (Hydro_Con2Flux with MHD, pressure from Hydro_Con2Pres
// with the magnetic energy and the pressure floor, CPU_Shared_FluUtility.cpp:458-548)
template <int D, int P, typename R>
GB_DEV void mm_con2flux( const Phys<R> &ph, const R *u, R *f )
{
   const R ird = R(1)/u[0];
   const R pres = check_floor( eint_con_mhd<P>( u[0], ird, u[1], u[2], u[3], u[4], emag_of( u ) )*ph.gm1, ph.min_pres );
   mhd_con2flux<D>( u, ird, pres, f );
}

// one face-state cell per item: the six face states, the Hancock predictor with MHD fluxes
// (Hydro_HancockPredict, CPU_Shared_DataReconstruction.cpp:2064-2160), MHD_UpdateMagnetic_Half
// (CPU_Shared_ConstrainedTransport.cpp:858-912) with the half-step EMFs at the cell's edges, the
// MHM_CHECK_PREDICT reset of the fluid variables (the face B keep their update) or the floors, and
// Hydro_ConFC2PriCC_MHM (CPU_Shared_DataReconstruction.cpp:2189-2229); the face states go to the CTU
// layout (cells 1..18 of the 20^3 grid), the half-step primitives to `bh`
template <typename R, int P, int CH, int LR = LR_PLM>
__global__ void __launch_bounds__( 256, 1 ) mm_recon( const __grid_constant__ CtuArgs<R> a )
{
   using namespace ctu;
   constexpr int N = ( LR == LR_PPM ) ? MNX + 2 : MNX, N3 = N*N*N, PL = ( N == MNX ) ? MNX3 : plane_of( N );
   constexpr int OFF = flg_of( N ) - 1;                        // the face-state cell's offset in the input
   PG_LOOP( f, NFF*NFF*NFF )
   {
      const int i = f % NFF, j = ( f / NFF ) % NFF, k = f / ( NFF*NFF );
      const int ic = i + OFF, jc = j + OFF, kc = k + OFF;      // the cell in the input window
      const R *pri = a.pri + (size_t)pg*NM*NX3;
      const R *bin = a.bin + (size_t)pg*3*nbin_of( N );
      const int c = idx3( ic, jc, kc, N, N );
      R cc[NM], w[6][NM], u[6][NM];
#     pragma unroll
      for (int v=0; v<NM; v++) cc[v] = pri[v*PL + c];
      mm_faces_dir<0,CH,LR>( a, pri, bin, cc, ic, jc, kc, w[0], w[1] );
      mm_faces_dir<1,CH,LR>( a, pri, bin, cc, ic, jc, kc, w[2], w[3] );
      mm_faces_dir<2,CH,LR>( a, pri, bin, cc, ic, jc, kc, w[4], w[5] );
#     pragma unroll
      for (int q=0; q<6; q++) mhd_pri2con( a.ph, w[q], u[q] );
      // Hancock: dFlux = dt/(2dh) (F1 - F0 + F3 - F2 + F5 - F4) of the fluid variables on every face
      {
         R fx[6][NM];
         mm_con2flux<0,P>( a.ph, u[0], fx[0] );  mm_con2flux<0,P>( a.ph, u[1], fx[1] );
         mm_con2flux<1,P>( a.ph, u[2], fx[2] );  mm_con2flux<1,P>( a.ph, u[3], fx[3] );
         mm_con2flux<2,P>( a.ph, u[4], fx[4] );  mm_con2flux<2,P>( a.ph, u[5], fx[5] );
         const R dt_dh2 = R(0.5)*a.dt/a.dh;
#        pragma unroll
         for (int v=0; v<5; v++)
         {
            const R df = dt_dh2*( fx[1][v] - fx[0][v] + fx[3][v] - fx[2][v] + fx[5][v] - fx[4][v] );
#           pragma unroll
            for (int q=0; q<6; q++) u[q][v] -= df;
         }
      }
      // the face B with the half-step EMFs at the cell's edges (EMF stride 19, the cell's lower edges
      // at its face-state index)
      {
         const R dt_dh2 = R(0.5)*a.dt/a.dh;
         const R *ec = a.ec + (size_t)pg*a.ec_pg;
         const int ie = idx3( i, j, k, NHE, NHE );
         const int de[3] = { 1, NHE, NHE*NHE };
         R src[2][3];
#        pragma unroll
         for (int d=0; d<3; d++)
         {
            const int T1 = ( d + 1 ) % 3, T2 = ( d + 2 ) % 3;
            src[0][d] = ( ec[T1*NEC + ie + de[T2]] - ec[T1*NEC + ie] )*dt_dh2 -
                        ( ec[T2*NEC + ie + de[T1]] - ec[T2*NEC + ie] )*dt_dh2;
            src[1][d] = ( ec[T1*NEC + ie + de[T2] + de[d]] - ec[T1*NEC + ie + de[d]] )*dt_dh2 -
                        ( ec[T2*NEC + ie + de[T1] + de[d]] - ec[T2*NEC + ie + de[d]] )*dt_dh2;
         }
#        pragma unroll
         for (int d=0; d<3; d++)
         {
            const int T1 = ( d + 1 ) % 3, T2 = ( d + 2 ) % 3;
            u[2*d][MO + d] += src[0][d];
            u[2*d + 1][MO + d] += src[1][d];
            const R s1 = R(0.5)*( src[0][T1] + src[1][T1] ), s2 = R(0.5)*( src[0][T2] + src[1][T2] );
            u[2*d][MO + T1] += s1;  u[2*d + 1][MO + T1] += s1;
            u[2*d][MO + T2] += s2;  u[2*d + 1][MO + T2] += s2;
         }
      }
      // MHM_CHECK_PREDICT: density and energy of the predicted states, pressure of the reconstructed ones
      bool bad = false;
#     pragma unroll
      for (int q=0; q<6; q++)
      {
         const R d0 = u[q][0], e4 = u[q][4], p4 = w[q][4];
         bad |= !( d0 >= Lim<R>::tiny() && d0 <= Lim<R>::huge() );
         bad |= !( e4 >= Lim<R>::tiny() && e4 <= Lim<R>::huge() );
         bad |= !( p4 >= R(0) && p4 <= Lim<R>::huge() );
      }
      if ( bad )
      {
         const R *uin = a.in + (size_t)pg*5*N3;
#        pragma unroll
         for (int v=0; v<5; v++)
         {
            const R cv = uin[v*N3 + c];
#           pragma unroll
            for (int q=0; q<6; q++) u[q][v] = cv;
         }
      }
      else
      {
#        pragma unroll
         for (int q=0; q<6; q++)
         {
            u[q][0] = gmax( u[q][0], a.ph.min_dens );
            const R e  = eint_con_mhd<P>( u[q][0], R(1)/u[q][0], u[q][1], u[q][2], u[q][3], u[q][4], emag_of( u[q] ) );
            const R eo = gmax( e, a.ph.min_eint );
            if ( !( e == eo ) ) u[q][4] = u[q][4] - e + eo;
         }
      }
      R *fcv = a.fcv + (size_t)pg*6*NM*NF3;
      const int fo = idx3( i + 1, j + 1, k + 1, NF, NF );
#     pragma unroll
      for (int q=0; q<6; q++)
#        pragma unroll
         for (int v=0; v<NM; v++) fcv[( q*NM + v )*NF3 + fo] = u[q][v];
      // Hydro_ConFC2PriCC_MHM: fluid variables averaged over the six faces, B over the two normal faces
      R ccon[NM], cw[NM];
#     pragma unroll
      for (int v=0; v<5; v++)
      {
         R sum = R(0);
#        pragma unroll
         for (int q=0; q<6; q++) sum += u[q][v];
         ccon[v] = sum*( R(1)/R(6) );
      }
#     pragma unroll
      for (int d=0; d<3; d++) ccon[MO + d] = R(0.5)*( u[2*d][MO + d] + u[2*d + 1][MO + d] );
      mhd_con2pri<P>( a.ph, ccon, cw );
      if ( a.ph.jeans ) cw[4] = check_floor( cw[4], a.ph.jeans_coeff*( cw[0]*cw[0] ) );
      R *hp = a.bh + (size_t)pg*NM*NX3;
#     pragma unroll
      for (int v=0; v<NM; v++) hp[v*NX3 + f] = cw[v];
   }
}

} // namespace gb

using namespace gb;

namespace {

// grid of a per-patch-group kernel: items of one patch group (and direction) along x (about 4 per
// thread, so that the light stages are not bound by CTA launch), the face / edge direction along y,
// patch groups along z (the directions of one patch group are scheduled together, sharing L2)
dim3 ctu_grid( int per, int npg, int block, int ndir = 1 )
{
   return dim3( ( per + 4*block - 1 )/( 4*block ), ndir, npg );
}

// scratch per patch group of an input of FLU_NXT nxi.  scheme: GB_SCHEME_CTU, GB_SCHEME_MHM_RP (its
// half-step B and EMF arrays span nxi - 2 cells and nxi - 1 edges; the face-state region holds the
// half-step fluxes, 3*8*nxi^3 <= 6*8*20^3, and the flux region the half-step primitives,
// 8*(nxi - 2)^3 <= 3*8*20^3) or GB_SCHEME_MHM (the `bh` region holds the half-step primitives,
// planes of 22^3)
size_t ctu_scratch_per_pg( size_t rsz, int scheme = GB_SCHEME_CTU, int nxi = ctu::NX )
{
   using namespace ctu;
   static_assert( 3*NM*( NX + 2 )*( NX + 2 )*( NX + 2 ) <= 6*NM*NF3 && NM*( RHV + 2 )*( RHV + 2 )*( RHV + 2 ) <= 3*NM*NF3,
                  "MHM_RP half-step arrays must fit the CTU regions" );
   const size_t hv = nxi - 2, he = nxi - 1;
   const size_t nb = ( scheme == GB_SCHEME_MHM_RP ) ? 3*( hv + 1 )*hv*hv : ( scheme == GB_SCHEME_MHM ) ? (size_t)NM*NX3 : 3*(size_t)NBH;
   const size_t ne = ( scheme == GB_SCHEME_MHM_RP ) ? he*he*he : NEC;
   const size_t flags = ( scheme == GB_SCHEME_CTU ) ? 0 : 2*sizeof(int) + 256;   // MinMod retry flags
   return rsz*( (size_t)NM*plane_of( nxi ) + 6*NM*NF3 + 3*NM*NF3 + nb + 3*ne ) + 5*256 + flags;
}

// the CTU half step (reconstruction with tracing, half-step fluxes, EMFs and B, transverse-gradient
// correction, half-step primitives) for PLM (FLU_NXT 22) or PPM (24)
template <typename R, int P, int LR>
void ctu_half_step( const CtuArgs<R> &a, int charr, int n, cudaStream_t st )
{
   using namespace ctu;
   constexpr int NXI = ( LR == LR_PPM ) ? NX + 2 : NX;
   const int B = 256;
   if ( charr ) ctu_recon<R,P,1,LR><<< ctu_grid( NF3, n, B, 3 ), B, 0, st >>>( a );
   else         ctu_recon<R,P,0,LR><<< ctu_grid( NF3, n, B, 3 ), B, 0, st >>>( a );
   ctu_flux<R,P,0><<< ctu_grid( ( NF - 1 )*NF*NF, n, B, 3 ), B, 0, st >>>( a );
   ctu_emf<R,0,NXI><<< ctu_grid( ( NHE - 1 )*NHE*NHE, n, B, 3 ), B, 0, st >>>( a );
   ctu_bupdate<R,0,NXI><<< ctu_grid( NBH, n, B, 3 ), B, 0, st >>>( a, a.bh, 3*(size_t)NBH, NBH, R(0.5)*a.dt );
   ctu_tgrad<R,P,NXI><<< ctu_grid( NHV*NHV*NHV, n, B, 3 ), B, 0, st >>>( a );
   ctu_halfprim<R,NXI><<< ctu_grid( NHV*NHV*NHV, n, B ), B, 0, st >>>( a );
}

// the MHM_RP half step: first-order half-step fluxes of the input cells, their EMFs and the CT
// update of B over dt/2, the half-step cells (FLU_NXT - 2 per side), then PLM (FLU_NXT 22) or PPM
// (24) face values of the half-step state without tracing
template <typename R, int P, int LR>
void rp_half_step( const CtuArgs<R> &a, int charr, int n, cudaStream_t st )
{
   using namespace ctu;
   constexpr int NXI = ( LR == LR_PPM ) ? NX + 2 : NX, HV = NXI - 2, HE = NXI - 1, HNB = ( HV + 1 )*HV*HV;
   const int B = 256;
   rp_half_flux<R,P,NXI><<< ctu_grid( ( NXI - 1 )*NXI*NXI, n, B, 3 ), B, 0, st >>>( a );
   ctu_emf<R,2,NXI><<< ctu_grid( ( HE - 1 )*HE*HE, n, B, 3 ), B, 0, st >>>( a );
   ctu_bupdate<R,2,NXI><<< ctu_grid( HNB, n, B, 3 ), B, 0, st >>>( a, a.bh, 3*(size_t)HNB, HNB, R(0.5)*a.dt );
   rp_predict<R,P,NXI><<< ctu_grid( HV*HV*HV, n, B ), B, 0, st >>>( a );
   if ( charr ) rp_recon<R,P,1,LR><<< ctu_grid( NFF*NFF*NFF, n, B, 3 ), B, 0, st >>>( a );
   else         rp_recon<R,P,0,LR><<< ctu_grid( NFF*NFF*NFF, n, B, 3 ), B, 0, st >>>( a );
}

// the full step shared by every scheme (the same faces, edges and half-step cells), on an input of
// FLU_NXT NXI (20: MHM; 22: CTU+PLM, MHM_RP; 24: CTU+PPM)
template <typename R, int P, int NXI>
void ctu_full_step( const CtuArgs<R> &af, int n, cudaStream_t st )
{
   using namespace ctu;
   const int B = 256;
   ctu_flux<R,P,1><<< ctu_grid( ( NF - 3 )*( NF - 2 )*( NF - 2 ), n, B, 3 ), B, 0, st >>>( af );
   ctu_emf<R,1,NXI><<< ctu_grid( ( NFE - 1 )*NFE*NFE, n, B, 3 ), B, 0, st >>>( af );
   if constexpr ( NXI == MNX )
      ctu_bupdate<R,3><<< ctu_grid( NBOUT, n, B, 3 ), B, 0, st >>>( af, af.bout, 3*(size_t)NBOUT, NBOUT, af.dt );
   else
      ctu_bupdate<R,1,NXI><<< ctu_grid( NBOUT, n, B, 3 ), B, 0, st >>>( af, af.bout, 3*(size_t)NBOUT, NBOUT, af.dt );
   ctu_update<R,P,NXI><<< ctu_grid( PS2*PS2*PS2, n, B ), B, 0, st >>>( af );
}

template <typename R, int P>
int ctu_solve_t( const gb_fluid_config &cfg, const void *in, const void *bin, void *out, void *bout,
                 void *flux, void *ele, int npg, const gb_fluid_params *prm, void *scratch, size_t scratch_bytes,
                 cudaStream_t st )
{
   using namespace ctu;
   const bool rp = ( cfg.scheme == GB_SCHEME_MHM_RP ), mm = ( cfg.scheme == GB_SCHEME_MHM );
   const bool ppm = ( ( cfg.scheme == GB_SCHEME_CTU || rp ) && cfg.lr_scheme == GB_LR_PPM );
   const bool mppm = ( mm && cfg.lr_scheme == GB_LR_PPM );
   const int nxi = mm ? ( mppm ? MNX + 2 : MNX ) : ppm ? NX + 2 : NX;     // FLU_NXT of the input
   const size_t nx3 = (size_t)nxi*nxi*nxi, nbin = nbin_of( nxi );
   int chunk = (int)( scratch_bytes / ctu_scratch_per_pg( sizeof(R), cfg.scheme, nxi ) );
   if ( chunk < 1 ) return GB_E_INVALID;
   if ( chunk > 65535 ) chunk = 65535;            // patch groups of a chunk run along grid.z
   for (int p0 = 0; p0 < npg; p0 += chunk)
   {
      const int n = ( npg - p0 < chunk ) ? npg - p0 : chunk;
      char *w = (char*)scratch;
      auto take = [&]( size_t elems ) { R *r = (R*)w;  w += ( elems*sizeof(R) + 255 ) & ~(size_t)255;  return r; };
      CtuArgs<R> a;
      memset( &a, 0, sizeof(a) );
      a.in   = (const R*)in   + (size_t)p0*5*nx3;
      a.bin  = (const R*)bin  + (size_t)p0*3*nbin;
      a.out  = (R*)out  + (size_t)p0*5*PS2*PS2*PS2;
      a.bout = (R*)bout + (size_t)p0*3*NBOUT;
      a.flux = ( prm->store_flux && flux ) ? (R*)flux + (size_t)p0*9*5*PS2*PS2 : nullptr;
      a.ele  = ( prm->store_electric && ele ) ? (R*)ele + (size_t)p0*9*2*NELE : nullptr;
      a.pri  = take( (size_t)n*NM*plane_of( nxi ) );
      a.fcv  = take( (size_t)n*6*NM*NF3 );
      a.fcf  = take( (size_t)n*3*NM*NF3 );
      const size_t hv = nxi - 2, rnec = (size_t)( nxi - 1 )*( nxi - 1 )*( nxi - 1 );   // MHM_RP half step
      a.bh   = take( (size_t)n*( rp ? 3*( hv + 1 )*hv*hv : mm ? (size_t)NM*NX3 : 3*(size_t)NBH ) );
      a.ec   = take( (size_t)n*3*( rp ? rnec : (size_t)NEC ) );
      a.npg  = n;
      a.ec_pg = 3*( rp ? rnec : (size_t)NEC );
      a.limiter = prm->lr_limiter;
      a.coeff = (R)prm->minmod_coeff;
      a.dt = (R)prm->dt;  a.dh = (R)prm->dh;
      a.ph.gamma = (R)cfg.gamma;  a.ph.gm1 = (R)( cfg.gamma - 1.0 );  a.ph.inv_gm1 = (R)( 1.0/( cfg.gamma - 1.0 ) );
      a.ph.min_dens = (R)prm->min_dens;  a.ph.min_pres = (R)prm->min_pres;  a.ph.min_eint = (R)prm->min_eint;
      a.ph.de_switch = (R)prm->dual_energy_switch;
      a.ph.jeans = prm->jeans_min_pres;  a.ph.jeans_coeff = (R)prm->jeans_min_pres_coeff;
      const int B = 256;
      // one pass of the whole pipeline; the MinMod retries of MHM and MHM_RP (CPU_FluidSolver_MHM.cpp:
      // 466-585) re-run it, with the reduced coefficient, for the patch groups whose previous pass
      // left an unphysical cell: every kernel returns at once for the others (`active`), and every
      // stage but the reconstruction gives the same values again
      auto pass = [&]( const CtuArgs<R> &a )
      {
         if ( mppm ) ctu_con2pri<R,P,MNX + 2><<< ctu_grid( NX3, n, B ), B, 0, st >>>( a );
         else if ( mm ) ctu_con2pri<R,P,MNX><<< ctu_grid( MNX3, n, B ), B, 0, st >>>( a );
         else if ( ppm ) ctu_con2pri<R,P,NX + 2><<< ctu_grid( ( NX + 2 )*( NX + 2 )*( NX + 2 ), n, B ), B, 0, st >>>( a );
         else      ctu_con2pri<R,P><<< ctu_grid( NX3, n, B ), B, 0, st >>>( a );
         CtuArgs<R> af = a;           // the full step's arguments
         if ( mm )
         {
            // MHM: half-step EMFs from the input, then the face states with the Hancock predictor
            const dim3 gr = ctu_grid( NFF*NFF*NFF, n, B ), ge = ctu_grid( ( NHE - 1 )*NHE*NHE, n, B, 3 );
            if ( mppm )
            {
               mm_emf_half<R,MNX + 2><<< ge, B, 0, st >>>( a );
               if ( cfg.char_reconstruction ) mm_recon<R,P,1,LR_PPM><<< gr, B, 0, st >>>( a );
               else                           mm_recon<R,P,0,LR_PPM><<< gr, B, 0, st >>>( a );
            }
            else
            {
               mm_emf_half<R,MNX><<< ge, B, 0, st >>>( a );
               if ( cfg.char_reconstruction ) mm_recon<R,P,1><<< gr, B, 0, st >>>( a );
               else                           mm_recon<R,P,0><<< gr, B, 0, st >>>( a );
            }
            af.pri = a.bh;            // the full-step EMFs read the half-step primitives
         }
         else if ( rp && ppm ) rp_half_step<R,P,LR_PPM>( a, cfg.char_reconstruction, n, st );
         else if ( rp )  rp_half_step<R,P,LR_PLM>( a, cfg.char_reconstruction, n, st );
         else if ( ppm ) ctu_half_step<R,P,LR_PPM>( a, cfg.char_reconstruction, n, st );
         else            ctu_half_step<R,P,LR_PLM>( a, cfg.char_reconstruction, n, st );
         if      ( mppm ) ctu_full_step<R,P,NX>( af, n, st );
         else if ( mm )  ctu_full_step<R,P,MNX>( af, n, st );
         else if ( ppm ) ctu_full_step<R,P,NX + 2>( af, n, st );
         else            ctu_full_step<R,P,NX>( af, n, st );
      };
      const int maxit = ( mm || rp ) ? prm->minmod_maxiter : 0;
      int *flags = nullptr;
      if ( maxit > 0 )
      {
         flags = (int*)w;
         if ( cudaMemsetAsync( flags, 0, 2*(size_t)n*sizeof(int), st ) != cudaSuccess ) return GB_E_CUDA;
         a.fail_next = flags;
      }
      pass( a );
      for (int it=1; it<=maxit; it++)
      {
         // AdaptiveMinModCoeff, in the precision of the reconstruction
         const R c0 = (R)prm->minmod_coeff;
         R cf = c0 - (R)it*c0/(R)maxit;
         cf = ( cf > R(0) ) ? cf : R(0);
         CtuArgs<R> r = a;
         r.coeff = cf;
         r.active = flags + (size_t)( ( it - 1 ) & 1 )*n;
         r.fail_next = ( it < maxit ) ? flags + (size_t)( it & 1 )*n : nullptr;
         if ( r.fail_next != nullptr && cudaMemsetAsync( r.fail_next, 0, (size_t)n*sizeof(int), st ) != cudaSuccess )
            return GB_E_CUDA;
         pass( r );
      }
      if ( cudaGetLastError() != cudaSuccess ) return GB_E_CUDA;
   }
   return GB_OK;
}

} // namespace

namespace gb {

size_t ctu_scratch_bytes_per_pg( int precision )
{
   return ctu_scratch_per_pg( ( precision == GB_PREC_FP64 ) ? 8 : 4 );
}

size_t mhmrp_mhd_scratch_bytes_per_pg( int precision )
{
   return ctu_scratch_per_pg( ( precision == GB_PREC_FP64 ) ? 8 : 4, GB_SCHEME_MHM_RP );
}

size_t mhmrp_ppm_mhd_scratch_bytes_per_pg( int precision )
{
   return ctu_scratch_per_pg( ( precision == GB_PREC_FP64 ) ? 8 : 4, GB_SCHEME_MHM_RP, ctu::NX + 2 );
}

size_t mhm_mhd_scratch_bytes_per_pg( int precision )
{
   return ctu_scratch_per_pg( ( precision == GB_PREC_FP64 ) ? 8 : 4, GB_SCHEME_MHM, ctu::MNX );
}

size_t mhm_ppm_mhd_scratch_bytes_per_pg( int precision )
{
   return ctu_scratch_per_pg( ( precision == GB_PREC_FP64 ) ? 8 : 4, GB_SCHEME_MHM, ctu::NX );
}

size_t ctu_ppm_mhd_scratch_bytes_per_pg( int precision )
{
   return ctu_scratch_per_pg( ( precision == GB_PREC_FP64 ) ? 8 : 4, GB_SCHEME_CTU, ctu::NX + 2 );
}

// one CTU+MHD or MHM_RP+MHD solve (cfg.scheme) of npg patch groups in chunks of scratch_bytes /
// (ctu / mhmrp_mhd)_scratch_bytes_per_pg PGs
int ctu_solve( const gb_fluid_config &cfg, const void *flu_in, const void *mag_in, void *flu_out, void *mag_out,
               void *flux, void *ele, int npg, const gb_fluid_params *prm, void *scratch, size_t scratch_bytes,
               cudaStream_t st )
{
   if ( cfg.precision == GB_PREC_FP64 )
      return ctu_solve_t<double,P_FP64>( cfg, flu_in, mag_in, flu_out, mag_out, flux, ele, npg, prm, scratch, scratch_bytes, st );
   if ( cfg.precision == GB_PREC_MIXED )
      return ctu_solve_t<float,P_MIXED>( cfg, flu_in, mag_in, flu_out, mag_out, flux, ele, npg, prm, scratch, scratch_bytes, st );
   return ctu_solve_t<float,P_FP32>( cfg, flu_in, mag_in, flu_out, mag_out, flux, ele, npg, prm, scratch, scratch_bytes, st );
}

} // namespace gb
