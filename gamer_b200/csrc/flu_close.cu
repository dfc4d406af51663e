// First-order-flux correction of the cells a solve left unphysical: CorrectUnphysical of
// src/Fluid/Flu_Close.cpp:542-1200 (gamma-law EoS; hydro, and the MHD branch for CTU+MHD), run in
// place on the device arrays of gb_fluid_solve_device, so that GAMER's closing step needs no
// device-to-host copy first.
//
// One CTA per patch group, one thread per 16 output cells.  Every cell is screened with a
// call-free form of the reference's Unphysical() (Flu_Close.cpp:412-490) and, if the screen cannot
// clear it, tested exactly; a patch group with no unphysical cell ends after one read of its
// output (the common case).  An unphysical cell is then, in the
// thread that owns it:
//   (A) re-advanced with first-order fluxes from the input array, all three directions at once
//       (OPT__1ST_FLUX_CORR = 3D), the Riemann solver chosen by OPT__1ST_FLUX_CORR_SCHEME;
//   (B) with 3D1D, if (A) failed, re-advanced direction by direction (x, y, z) on its 3^3
//       neighbourhood, each sweep reading the previous one's result;
//   floored (density, dual-energy field, internal energy or the dual-energy pressure floor) and
//   tested again.  A cell that passes replaces the output; with flux fix-up its first-order
//   fluxes replace the coarse-fine fluxes of the faces it touches.  A cell that fails stays as it
//   was and is counted.
// The reference walks the cells of a patch group in i-fastest order, so where two corrected cells
// touch the same flux face (the middle plane of a patch group), the later cell's flux is the one
// kept; here the cell below the middle plane stashes its flux in shared memory and it is written
// after every cell of the patch group has been decided, only if the cell above was not corrected.
//
// MHD (Flu_Close.cpp:610-780 under MHD): every test includes the magnetic energy of the cell, taken
// from the face-centred output field (MHD_GetCellCenteredBEnergy); the first-order fluxes use the
// cell-centred input field of the three cells of each direction, with the longitudinal component
// of both states reset to the face-centred value of the face between them and the total energy
// adjusted by the difference in magnetic energy (ResetLongB), the Riemann solver being Roe, HLLE
// or HLLD; the directionally split correction (3D1D) does not exist for MHD in the reference and
// is refused.
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "mhd_physics.cuh"

namespace gb {
namespace {

constexpr int CL_THREADS = 256;
constexpr int CL_CELLS   = PS2*PS2*PS2/CL_THREADS;   // cells per thread
constexpr char DE_BY_MIN_PRES = '2';                 // DE_UPDATED_BY_MIN_PRES, include/Macro.h:99

enum { CORR_NONE = 0, CORR_3D = 1, CORR_3D1D = 2 };      // include/Typedef.h:461-465
enum { RS1_ROE = 1, RS1_HLLC = 2, RS1_HLLE = 3, RS1_HLLD = 4 };   // include/Typedef.h:467-474

template <typename R>
struct CloseArgs {
   const R *in;  R *out;  char *de;  R *flux;
   const R *mag_in;  const R *mag_out;   // MHD: face-centred B of the solver's input and output
   int *counts;               // [0] cells corrected, [1] cells still unphysical (accumulated)
   int  npg, nin;
   int  corr, scheme, fixup, floor_on, cont, check_pres;
   R    dt_dh;
   Phys<R> ph;
};

template <typename R> GB_DEV bool is_fin( R x ) { return isfinite( x ); }

// Unphysical() (Flu_Close.cpp:412-490) without the OPT__UNIT speed-of-light test: CheckMinEtot
// (eint = false) or CheckMinEint (eint = true)
template <int P, int NC, typename R>
GB_DEV bool unphysical( const Phys<R> &ph, const R *u, bool eint, bool check_pres )
{
   if ( !is_fin( u[0] ) || !is_fin( u[1] ) || !is_fin( u[2] ) || !is_fin( u[3] ) || !is_fin( u[4] ) ||
        u[0] < ph.min_dens ) return true;
   if ( !eint && ( u[4] < ph.min_eint || u[4] != u[4] ) ) return true;
   if ( eint )
   {
      if constexpr ( NC > 5 )
      {
         // the dual-energy variable is validated against 2*TINY_NUMBER (Flu_Close.cpp:444-452)
         const R pres = u[5]*gpow( u[0], ph.gm1 );
         if ( pres < ph.min_pres || !is_fin( pres ) || u[5] < R(2)*Lim<R>::tiny() || !is_fin( u[5] ) ) return true;
      }
      else
      {
         const R ei = eint_con<P>( u[0], R(1)/u[0], u[1], u[2], u[3], u[4] );
         if ( ei < ph.min_eint || !is_fin( ei ) ) return true;
      }
   }
   if ( check_pres )
   {
      const R pres = ph.gm1*eint_con<P>( u[0], R(1)/u[0], u[1], u[2], u[3], u[4] );
      if ( pres < ph.min_pres || !is_fin( pres ) ) return true;
   }
   return false;
}

// The per-cell screen of the scan over every output cell: true unless the cell surely passes
// unphysical( eint = true ).  It makes no function call (the double recovery of P_MIXED and pow()
// are calls), so the compiler keeps all 16 cells' loads of a thread in flight; a cell it cannot
// clear is re-tested exactly before any correction.
template <int P, int NC, typename R>
GB_DEV bool unphysical_screen( const Phys<R> &ph, const R *u, bool check_pres )
{
   if ( check_pres ) return true;
   if ( !is_fin( u[0] ) || !is_fin( u[1] ) || !is_fin( u[2] ) || !is_fin( u[3] ) || !is_fin( u[4] ) ||
        u[0] < ph.min_dens ) return true;
   if constexpr ( NC > 5 )
   {
      // pres = dual*rho^(gamma-1) is finite and positive for a finite dual above 2*TINY_NUMBER and a
      // density in (0, 1e30]; a positive pressure floor needs the exact test
      return !( ph.min_pres <= R(0) && u[5] >= R(2)*Lim<R>::tiny() && u[5] <= R(1e30) &&
                u[0] > R(0) && u[0] <= R(1e30) );
   }
   else
   {
      // the float estimate E - K decides where it clears MIN_EINT by more than its rounding error
      // (16 eps (|E| + K) covers it); the exact recovery (double under P_MIXED) decides the rest
      const R ke  = R(0.5)*( u[1]*u[1] + u[2]*u[2] + u[3]*u[3] )/u[0];
      const R ef  = u[4] - ke;
      const R err = R(16)*Lim<R>::eps()*( gabs( u[4] ) + gabs( ke ) );
      return !( ef > ph.min_eint + err );
   }
}

// Hydro_DualEnergyFix with its pressure floor (src/Model_Hydro/CPU_Hydro/CPU_Shared_DualEnergy.cpp:64-119)
template <int P, typename R>
GB_DEV void dual_energy_fix_floor( const Phys<R> &ph, R *u, char &st, bool check_min_pres )
{
   typedef typename std::conditional<P == P_MIXED, double, R>::type T;
   const R d = u[0];
   u[5] = gmax( u[5], Lim<R>::tiny() );
   T eint;
   if constexpr ( P == P_MIXED )
      eint = (double)u[4] - 0.5*( (double)u[1]*u[1] + (double)u[2]*u[2] + (double)u[3]*u[3] )*rcp_dd( (double)d );
   else
      eint = eint_con<P>( d, R(1)/d, u[1], u[2], u[3], u[4] );
   const T enth = (T)u[4] - eint;
   const T gm1 = (T)ph.gm1;
   T pres;
   if ( eint/enth < (T)ph.de_switch )
   {
      pres = (T)u[5]*gpow( (T)d, gm1 );
      u[4] = (R)( enth + pres*(T)ph.inv_gm1 );
      st   = DE_BY_DUAL;
   }
   else
   {
      pres = eint*gm1;
      u[5] = gmax( (R)( pres*gpow( (T)d, -gm1 ) ), Lim<R>::tiny() );
      st   = DE_BY_ETOT;
   }
   if ( check_min_pres && pres < (T)ph.min_pres )
   {
      pres = (T)ph.min_pres;
      u[4] = (R)( enth + pres*(T)ph.inv_gm1 );
      u[5] = gmax( (R)( pres*gpow( (T)d, -gm1 ) ), Lim<R>::tiny() );
      st   = DE_BY_MIN_PRES;
   }
}

// first-order flux through the face between L and Rt along direction d (Flu_Close.cpp:666-780);
// the solvers are the ones of the patch-group solver, called without its HLLE rescue.  scheme
// RS1_ROE + 3 is Roe with the intermediate-state check, which the reference compiles in only when
// the solver itself is Roe (include/CUFLU.h:178-186).
template <int D, int P, int NC, typename R>
GB_DEV void flux_1st_dir( int scheme, const Phys<R> &ph, const R *L, const R *Rt, R *f )
{
   if      ( scheme == RS1_ROE     ) riemann_roe <D,P,NC,R,false>( ph, L, Rt, f );
   else if ( scheme == RS1_ROE + 3 ) riemann_roe <D,P,NC,R,true >( ph, L, Rt, f );
   else if ( scheme == RS1_HLLC    ) riemann_hllc<D,P,NC>( ph, L, Rt, f );
   else                              riemann_hlle<D,P,NC>( ph, L, Rt, f );
}

template <int P, int NC, typename R>
GB_DEV void flux_1st( int d, int scheme, const Phys<R> &ph, const R *L, const R *Rt, R *f )
{
   if      ( d == 0 ) flux_1st_dir<0,P,NC>( scheme, ph, L, Rt, f );
   else if ( d == 1 ) flux_1st_dir<1,P,NC>( scheme, ph, L, Rt, f );
   else               flux_1st_dir<2,P,NC>( scheme, ph, L, Rt, f );
}

// the correction of one unphysical cell (ijk: its index in the patch group); returns true if the
// corrected state passes, with it in upd and the first-order fluxes of its six faces in fl / fr
template <int P, int NC, typename R>
__device__ __noinline__ bool correct_cell( const CloseArgs<R> a, const R *in_pg, int i, int j, int k,
                                           const R *out, char *st, R *upd, R (*fl)[NC], R (*fr)[NC] )
{
   const int  g    = ( a.nin - PS2 )/2;
   const long nx   = a.nin, nxy = nx*nx, n3 = nxy*nx;
   const long didx[3] = { 1, nx, nxy };
   const long c0   = ( (long)( k + g )*nx + ( j + g ) )*nx + ( i + g );
   const Phys<R> &ph = a.ph;

   if ( a.corr != CORR_NONE )
   {
      // (A) all three directions from the input states
      R vc[NC];
#     pragma unroll
      for (int v=0; v<NC; v++) vc[v] = in_pg[ v*n3 + c0 ];
      for (int d=0; d<3; d++)
      {
         R vl[NC], vr[NC];
#        pragma unroll
         for (int v=0; v<NC; v++) { vl[v] = in_pg[ v*n3 + c0 - didx[d] ];  vr[v] = in_pg[ v*n3 + c0 + didx[d] ]; }
         flux_1st<P,NC>( d, a.scheme, ph, vl, vc, fl[d] );
         flux_1st<P,NC>( d, a.scheme, ph, vc, vr, fr[d] );
      }
#     pragma unroll
      for (int v=0; v<NC; v++)
      {
         const R df0 = fr[0][v] - fl[0][v], df1 = fr[1][v] - fl[1][v], df2 = fr[2][v] - fl[2][v];
         upd[v] = vc[v] - a.dt_dh*( ( df0 + df1 ) + df2 );
      }
   }

   if ( a.corr == CORR_3D1D )
   {
      // (B) directionally split: the dual-energy fix without its pressure floor first, and the
      // split update only if the unsplit one is still unphysical (Flu_Close.cpp:793-907)
      if constexpr ( NC > 5 ) dual_energy_fix_floor<P>( ph, upd, *st, false );
      if ( unphysical<P,NC>( ph, upd, true, a.check_pres ) )
      {
         R box[27][NC];
         for (int kk=0; kk<3; kk++)
         for (int jj=0; jj<3; jj++)
         for (int ii=0; ii<3; ii++)
         {
            const long c = c0 + (long)( kk - 1 )*nxy + (long)( jj - 1 )*nx + ( ii - 1 );
#           pragma unroll
            for (int v=0; v<NC; v++) box[ ( kk*3 + jj )*3 + ii ][v] = in_pg[ v*n3 + c ];
         }
         const int bstep[3] = { 1, 3, 9 };
         for (int d=0; d<3; d++)
         {
            // the sweep along d updates the cells whose coordinates along the directions not yet
            // swept are free and along d and the swept ones are centred
            const int i0 = 1,                  i1 = 1;
            const int j0 = ( d >= 1 ) ? 1 : 0, j1 = ( d >= 1 ) ? 1 : 2;
            const int k0 = ( d >= 2 ) ? 1 : 0, k1 = ( d >= 2 ) ? 1 : 2;
            for (int kk=k0; kk<=k1; kk++)
            for (int jj=j0; jj<=j1; jj++)
            for (int ii=i0; ii<=i1; ii++)
            {
               const int c = ( kk*3 + jj )*3 + ii;
               R f1[NC], f2[NC];
               flux_1st<P,NC>( d, a.scheme, ph, box[ c - bstep[d] ], box[c], f1 );
               flux_1st<P,NC>( d, a.scheme, ph, box[c], box[ c + bstep[d] ], f2 );
#              pragma unroll
               for (int v=0; v<NC; v++) box[c][v] -= a.dt_dh*( f2[v] - f1[v] );
               if ( c == 13 )
               {
#                 pragma unroll
                  for (int v=0; v<NC; v++) { fl[d][v] = f1[v];  fr[d][v] = f2[v]; }
               }
            }
         }
#        pragma unroll
         for (int v=0; v<NC; v++) upd[v] = box[13][v];
      }
   }

   if ( a.corr == CORR_NONE )
   {
#     pragma unroll
      for (int v=0; v<NC; v++) upd[v] = out[v];
   }

   // floors (Flu_Close.cpp:930-975)
   const bool floor_now = !a.cont && a.floor_on;
   if ( floor_now ) upd[0] = gmax( upd[0], ph.min_dens );
   if constexpr ( NC > 5 )
   {
      upd[5] = gmax( upd[5], Lim<R>::tiny() );
      dual_energy_fix_floor<P>( ph, upd, *st, floor_now );
   }
   else if ( floor_now )
      upd[4] = floor_eint_in_engy<P>( ph, upd[0], upd[1], upd[2], upd[3], upd[4] );

   return !unphysical<P,NC>( ph, upd, a.cont != 0, a.check_pres );
}

// ---- MHD ----------------------------------------------------------------------------------------

// 0.5 B^2 at the centre of cell (i, j, k) of a face-centred field on an n^3 grid of cells
// (MHD_GetCellCenteredBEnergy, CPU_Shared_FluUtility.cpp:1687): Bx [n][n][n+1], By [n][n+1][n],
// Bz [n+1][n][n], one after the other
template <typename R>
GB_DEV void cc_bfield( const R *mag, long n, long i, long j, long k, R *b )
{
   const long nb = ( n + 1 )*n*n;
   const R *bx = mag, *by = mag + nb, *bz = mag + 2*nb;
   const long ix = ( k*n + j )*( n + 1 ) + i, iy = ( k*( n + 1 ) + j )*n + i, iz = ( k*n + j )*n + i;
   b[0] = R(0.5)*( bx[ix] + bx[ ix + 1 ] );
   b[1] = R(0.5)*( by[iy] + by[ iy + n ] );
   b[2] = R(0.5)*( bz[iz] + bz[ iz + n*n ] );
}

template <typename R>
GB_DEV R cc_emag( const R *mag, long n, long i, long j, long k )
{
   R b[3];
   cc_bfield( mag, n, i, j, k, b );
   return R(0.5)*( b[0]*b[0] + b[1]*b[1] + b[2]*b[2] );
}

// Unphysical() with the magnetic energy (no dual energy in MHD builds here)
template <int P, typename R>
GB_DEV bool unphysical_mhd( const Phys<R> &ph, const R *u, R emag, bool eint, bool check_pres )
{
   if ( !is_fin( u[0] ) || !is_fin( u[1] ) || !is_fin( u[2] ) || !is_fin( u[3] ) || !is_fin( u[4] ) ||
        u[0] < ph.min_dens ) return true;
   if ( !is_fin( emag ) ) return true;
   if ( !eint && ( u[4] < ph.min_eint || u[4] != u[4] ) ) return true;
   if ( eint )
   {
      const R ei = eint_con_mhd<P>( u[0], R(1)/u[0], u[1], u[2], u[3], u[4], emag );
      if ( ei < ph.min_eint || !is_fin( ei ) ) return true;
   }
   if ( check_pres )
   {
      const R pres = ph.gm1*eint_con_mhd<P>( u[0], R(1)/u[0], u[1], u[2], u[3], u[4], emag );
      if ( pres < ph.min_pres || !is_fin( pres ) ) return true;
   }
   return false;
}

// the call-free screen of unphysical_mhd( eint = true ), as unphysical_screen
template <int P, typename R>
GB_DEV bool unphysical_screen_mhd( const Phys<R> &ph, const R *u, R emag, bool check_pres )
{
   if ( check_pres ) return true;
   if ( !is_fin( u[0] ) || !is_fin( u[1] ) || !is_fin( u[2] ) || !is_fin( u[3] ) || !is_fin( u[4] ) ||
        u[0] < ph.min_dens || !is_fin( emag ) ) return true;
   const R ke  = R(0.5)*( u[1]*u[1] + u[2]*u[2] + u[3]*u[3] )/u[0];
   const R ef  = u[4] - ke - emag;
   const R err = R(16)*Lim<R>::eps()*( gabs( u[4] ) + gabs( ke ) + gabs( emag ) );
   return !( ef > ph.min_eint + err );
}

// Hydro_CheckMinEintInEngy with the magnetic energy (CPU_Shared_FluUtility.cpp:787-803)
template <int P, typename R>
GB_DEV R floor_eint_in_engy_mhd( const Phys<R> &ph, const R *u, R emag )
{
   const R ein  = eint_con_mhd<P>( u[0], R(1)/u[0], u[1], u[2], u[3], u[4], emag );
   const R eout = check_floor( ein, ph.min_eint );
   return ( ein == eout ) ? u[4] : u[4] - ein + eout;
}

template <int D, int P, typename R>
GB_DEV void flux_1st_mhd_dir( int scheme, const Phys<R> &ph, const R *L, const R *Rt, R *f )
{
   if      ( scheme == RS1_ROE  ) roe_mhd <D,P>( ph, L, Rt, f );
   else if ( scheme == RS1_HLLD ) hlld    <D,P>( ph, L, Rt, f );
   else                           hlle_mhd<D,P>( ph, L, Rt, f );
}

// ResetLongB (Flu_Close.cpp:1673-1686): the longitudinal field of both states set to the face value,
// the total energies adjusted by the change in magnetic energy
template <typename R>
GB_DEV void reset_long_b( R *L, R *Rt, R fcb, int d )
{
   const int ib = MO + d;
   L[4]  += R(0.5)*( fcb*fcb - L[ib]*L[ib] );
   Rt[4] += R(0.5)*( fcb*fcb - Rt[ib]*Rt[ib] );
   L[ib] = fcb;
   Rt[ib] = fcb;
}

// one state of 8 variables: the input fluid of cell (i, j, k) of the FLU_NXT^3 window and its
// cell-centred input field
template <typename R>
GB_DEV void load_state_mhd( const R *in_pg, const R *mag_pg, long nx, long i, long j, long k, R *s )
{
   const long n3 = nx*nx*nx, c = ( k*nx + j )*nx + i;
#  pragma unroll
   for (int v=0; v<5; v++) s[v] = in_pg[ v*n3 + c ];
   cc_bfield( mag_pg, nx, i, j, k, s + MO );
}

// the MHD correction of one unphysical cell (the 3D correction or none), as correct_cell
template <int P, typename R>
__device__ __noinline__ bool correct_cell_mhd( const CloseArgs<R> a, const R *in_pg, const R *mag_pg, int i, int j,
                                               int k, const R *out, R emag_out, R *upd, R (*fl)[5], R (*fr)[5] )
{
   const int  g  = ( a.nin - PS2 )/2;
   const long nx = a.nin;
   const long ii = i + g, jj = j + g, kk = k + g;
   const Phys<R> &ph = a.ph;

   if ( a.corr != CORR_NONE )
   {
      R vc[NM];
      load_state_mhd( in_pg, mag_pg, nx, ii, jj, kk, vc );
      const R cc_b[3] = { vc[MO], vc[MO+1], vc[MO+2] };
      const R cc_e = vc[4];
      const long nb = ( nx + 1 )*nx*nx;
      for (int d=0; d<3; d++)
      {
         R vl[NM], vr[NM], f[NM];
         load_state_mhd( in_pg, mag_pg, nx, ii - ( d == 0 ), jj - ( d == 1 ), kk - ( d == 2 ), vl );
         load_state_mhd( in_pg, mag_pg, nx, ii + ( d == 0 ), jj + ( d == 1 ), kk + ( d == 2 ), vr );
         // the face-centred longitudinal field on the two faces of the cell along d (IDX321_B)
         const R *bd = mag_pg + d*nb;
         long ib, step;
         if      ( d == 0 ) { ib = ( kk*nx + jj )*( nx + 1 ) + ii;  step = 1;       }
         else if ( d == 1 ) { ib = ( kk*( nx + 1 ) + jj )*nx + ii;  step = nx;      }
         else               { ib = ( kk*nx + jj )*nx + ii;          step = nx*nx;   }
         const R fcb0 = bd[ib], fcb1 = bd[ ib + step ];

         reset_long_b( vl, vc, fcb0, d );
         if      ( d == 0 ) flux_1st_mhd_dir<0,P>( a.scheme, ph, vl, vc, f );
         else if ( d == 1 ) flux_1st_mhd_dir<1,P>( a.scheme, ph, vl, vc, f );
         else               flux_1st_mhd_dir<2,P>( a.scheme, ph, vl, vc, f );
#        pragma unroll
         for (int v=0; v<5; v++) fl[d][v] = f[v];
         reset_long_b( vc, vr, fcb1, d );
         if      ( d == 0 ) flux_1st_mhd_dir<0,P>( a.scheme, ph, vc, vr, f );
         else if ( d == 1 ) flux_1st_mhd_dir<1,P>( a.scheme, ph, vc, vr, f );
         else               flux_1st_mhd_dir<2,P>( a.scheme, ph, vc, vr, f );
#        pragma unroll
         for (int v=0; v<5; v++) fr[d][v] = f[v];
         vc[ MO + d ] = cc_b[d];
         vc[4]        = cc_e;
      }
      const long n3 = nx*nx*nx, c0 = ( kk*nx + jj )*nx + ii;
#     pragma unroll
      for (int v=0; v<5; v++)
      {
         const R df0 = fr[0][v] - fl[0][v], df1 = fr[1][v] - fl[1][v], df2 = fr[2][v] - fl[2][v];
         upd[v] = in_pg[ v*n3 + c0 ] - a.dt_dh*( ( df0 + df1 ) + df2 );
      }
   }
   else
   {
#     pragma unroll
      for (int v=0; v<5; v++) upd[v] = out[v];
   }

   // floors (Flu_Close.cpp:930-975)
   const bool floor_now = !a.cont && a.floor_on;
   if ( floor_now )
   {
      upd[0] = gmax( upd[0], ph.min_dens );
      upd[4] = floor_eint_in_engy_mhd<P>( ph, upd, emag_out );
   }
   return !unphysical_mhd<P>( ph, upd, emag_out, a.cont != 0, a.check_pres );
}

template <typename R, int P, int NC, bool MHD>
__global__ void __launch_bounds__(CL_THREADS) close_kernel( const CloseArgs<R> a )
{
   constexpr long NBO = (long)( PS2 + 1 )*PS2*PS2;   // face-centred B per component, output
   __shared__ R        s_mid[3][PS2*PS2][NC];      // fluxes of corrected cells just below a middle plane
   __shared__ uint32_t s_mid_set[3][PS2*PS2/32];
   __shared__ uint32_t s_fixed[PS2*PS2*PS2/32];    // corrected cells
   __shared__ int      s_count[2];

   const int tid = threadIdx.x;
   const long ncell = (long)PS2*PS2*PS2;
   const long n3in  = (long)a.nin*a.nin*a.nin;

   for (int pg=blockIdx.x; pg<a.npg; pg+=gridDim.x)
   {
      R *out = a.out + (long)pg*NC*ncell;
      const R *mag_out = MHD ? a.mag_out + (long)pg*3*NBO : nullptr;
      // the test of every cell: one coalesced read of the output
      uint32_t bad = 0;
#     pragma unroll
      for (int c=0; c<CL_CELLS; c++)
      {
         const int cell = c*CL_THREADS + tid;
         R u[NC];
#        pragma unroll
         for (int v=0; v<NC; v++) u[v] = out[ v*ncell + cell ];
         if constexpr ( MHD )
         {
            const R em = cc_emag( mag_out, PS2, cell % PS2, ( cell/PS2 ) % PS2, cell/( PS2*PS2 ) );
            if ( unphysical_screen_mhd<P>( a.ph, u, em, a.check_pres ) ) bad |= 1u << c;
         }
         else if ( unphysical_screen<P,NC>( a.ph, u, a.check_pres ) ) bad |= 1u << c;
      }
      if ( !__syncthreads_or( bad != 0 ) ) continue;

      for (int w=tid; w<PS2*PS2*PS2/32; w+=CL_THREADS) s_fixed[w] = 0u;
      for (int w=tid; w<3*PS2*PS2/32; w+=CL_THREADS) (&s_mid_set[0][0])[w] = 0u;
      if ( tid < 2 ) s_count[tid] = 0;
      __syncthreads();

      const R *in_pg = a.in + (long)pg*NC*n3in;
      R *flux = a.flux + (long)pg*9*NC*PS2*PS2;
      for (int c=0; c<CL_CELLS; c++)
      {
         if ( !( bad & ( 1u << c ) ) ) continue;
         const int cell = c*CL_THREADS + tid;
         const int i = cell % PS2, j = ( cell/PS2 ) % PS2, k = cell/( PS2*PS2 );
         R u[NC], upd[NC], fl[3][NC], fr[3][NC];
#        pragma unroll
         for (int v=0; v<NC; v++) u[v] = out[ v*ncell + cell ];
         bool ok;
         if constexpr ( MHD )
         {
            const R em = cc_emag( mag_out, PS2, i, j, k );
            if ( !unphysical_mhd<P>( a.ph, u, em, true, a.check_pres ) ) continue;   // cleared by the exact test
            const R *mag_in_pg = a.mag_in + (long)pg*3*( a.nin + 1 )*a.nin*a.nin;
            ok = correct_cell_mhd<P>( a, in_pg, mag_in_pg, i, j, k, u, em, upd, fl, fr );
         }
         else
         {
            if ( !unphysical<P,NC>( a.ph, u, true, a.check_pres ) ) continue;    // cleared by the exact test
            char st = ( a.de != nullptr ) ? a.de[ (long)pg*ncell + cell ] : DE_BY_ETOT;
            ok = correct_cell<P,NC>( a, in_pg, i, j, k, u, &st, upd, fl, fr );
            // the dual-energy fix writes the status of the cell whether or not the correction passes
            if ( NC > 5 ) a.de[ (long)pg*ncell + cell ] = st;
         }
         if ( !ok ) { atomicAdd( &s_count[1], 1 );  continue; }
         atomicAdd( &s_count[0], 1 );
#        pragma unroll
         for (int v=0; v<NC; v++) out[ v*ncell + cell ] = upd[v];
         atomicOr( &s_fixed[ cell >> 5 ], 1u << ( cell & 31 ) );
         if ( a.fixup && a.corr != CORR_NONE )
         {
            const int ijk[3] = { i, j, k };
            for (int d=0; d<3; d++)
            {
               const int m = ( d == 2 ) ? j : k, n = ( d == 0 ) ? j : i;   // dim_map (Flu_Close.cpp:1185)
               const int store = m*PS2 + n;
               if ( ijk[d] == 0 || ijk[d] == PS1 )
               {
                  R *f = flux + ( 3*d + ijk[d]/PS1 )*NC*PS2*PS2;
#                 pragma unroll
                  for (int v=0; v<NC; v++) f[ v*PS2*PS2 + store ] = fl[d][v];
               }
               else if ( ijk[d] == PS2 - 1 )
               {
                  R *f = flux + ( 3*d + 2 )*NC*PS2*PS2;
#                 pragma unroll
                  for (int v=0; v<NC; v++) f[ v*PS2*PS2 + store ] = fr[d][v];
               }
               else if ( ijk[d] == PS1 - 1 )
               {
#                 pragma unroll
                  for (int v=0; v<NC; v++) s_mid[d][store][v] = fr[d][v];
                  atomicOr( &s_mid_set[d][ store >> 5 ], 1u << ( store & 31 ) );
               }
            }
         }
      }
      __syncthreads();

      // the middle-plane fluxes of cells below it, where the cell above was not corrected
      for (int e=tid; e<3*PS2*PS2; e+=CL_THREADS)
      {
         const int d = e/( PS2*PS2 ), store = e % ( PS2*PS2 );
         if ( !( s_mid_set[d][ store >> 5 ] & ( 1u << ( store & 31 ) ) ) ) continue;
         const int m = store/PS2, n = store % PS2;
         int i, j, k;
         if      ( d == 0 ) { i = PS1;  j = n;    k = m; }
         else if ( d == 1 ) { i = n;    j = PS1;  k = m; }
         else               { i = n;    j = m;    k = PS1; }
         const int above = ( k*PS2 + j )*PS2 + i;
         if ( s_fixed[ above >> 5 ] & ( 1u << ( above & 31 ) ) ) continue;
         R *f = flux + ( 3*d + 1 )*NC*PS2*PS2;
#        pragma unroll
         for (int v=0; v<NC; v++) f[ v*PS2*PS2 + store ] = s_mid[d][store][v];
      }
      if ( tid == 0 )
      {
         if ( s_count[0] ) atomicAdd( &a.counts[0], s_count[0] );
         if ( s_count[1] ) atomicAdd( &a.counts[1], s_count[1] );
      }
      __syncthreads();
   }
}

template <typename R, int P, int NC, bool MHD = false>
cudaError_t close_launch( const CloseArgs<R> &a, cudaStream_t st )
{
   int dev = 0, nsm = 0, per_sm = 0;
   cudaGetDevice( &dev );
   cudaDeviceGetAttribute( &nsm, cudaDevAttrMultiProcessorCount, dev );
   cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, close_kernel<R,P,NC,MHD>, CL_THREADS, 0 );
   if ( err != cudaSuccess ) return err;
   if ( per_sm < 1 ) return cudaErrorInvalidConfiguration;
   const int grid = ( a.npg < nsm*per_sm ) ? a.npg : nsm*per_sm;
   close_kernel<R,P,NC,MHD><<< grid, CL_THREADS, 0, st >>>( a );
   return cudaGetLastError();
}

template <typename R, int P>
int close_run( const gb_fluid_config &c, const void *flu_in, void *flu_out, char *de_out, void *flux, int npg,
               const gb_fluid_params *prm, const gb_close_params *cp, int *counts, cudaStream_t st,
               const void *mag_in = nullptr, const void *mag_out = nullptr )
{
   CloseArgs<R> a;
   a.in = (const R*)flu_in;  a.out = (R*)flu_out;  a.de = de_out;  a.flux = (R*)flux;  a.counts = counts;
   a.mag_in = (const R*)mag_in;  a.mag_out = (const R*)mag_out;
   a.npg = npg;  a.nin = c.flu_nxt;
   a.corr = cp->first_flux_corr;  a.scheme = cp->first_flux_scheme;
   if ( a.scheme == RS1_ROE && c.rsolver == GB_RSOLVER_ROE ) a.scheme = RS1_ROE + 3;
   a.fixup = prm->store_flux && flux != nullptr;
   a.floor_on = cp->last_resort_floor;  a.cont = cp->auto_reduce_dt_continue;  a.check_pres = cp->check_pres_after_flu;
   a.dt_dh = (R)( prm->dt/prm->dh );
   a.ph.gamma     = (R)c.gamma;
   a.ph.gm1       = (R)( c.gamma - 1.0 );
   a.ph.inv_gm1   = (R)( 1.0/( c.gamma - 1.0 ) );
   a.ph.min_dens  = (R)prm->min_dens;
   a.ph.min_pres  = (R)prm->min_pres;
   a.ph.min_eint  = (R)prm->min_eint;
   a.ph.de_switch = (R)prm->dual_energy_switch;
   const cudaError_t err = ( mag_in != nullptr )            ? close_launch<R,P,5,true>( a, st )
                         : ( c.dual_energy == GB_DE_ENPY ) ? close_launch<R,P,6>( a, st ) : close_launch<R,P,5>( a, st );
   return ( err == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

} // namespace
} // namespace gb

struct gb_fluid_solver;
extern "C" int gb_fluid_get_config( const gb_fluid_solver *s, gb_fluid_config *cfg );

extern "C"
int gb_fluid_correct_unphysical_device( gb_fluid_solver *s, const void *flu_in, void *flu_out, char *de_out,
                                        void *flux, int npg, const gb_fluid_params *prm,
                                        const gb_close_params *cp, int *counts, void *stream )
{
   using namespace gb;
   if ( s == nullptr || prm == nullptr || cp == nullptr || counts == nullptr ) return GB_E_INVALID;
   gb_fluid_config c;
   if ( gb_fluid_get_config( s, &c ) != GB_OK ) return GB_E_INVALID;
   // CTU+MHD corrects with the magnetic field as well: gb_fluid_correct_unphysical_mhd_device
   if ( cfg_mhd( c ) ) return GB_E_INVALID;
   if ( c.npassive_user != 0 ) return GB_E_UNSUPPORTED;   // user passive scalars: not built
   if ( cp->first_flux_corr < CORR_NONE || cp->first_flux_corr > CORR_3D1D ) return GB_E_INVALID;
   if ( cp->first_flux_corr != CORR_NONE &&
        ( cp->first_flux_scheme < RS1_ROE || cp->first_flux_scheme > RS1_HLLE ) ) return GB_E_INVALID;
   if ( !( prm->dh > 0.0 ) || !( prm->dt >= 0.0 ) || npg < 0 ) return GB_E_INVALID;
   if ( npg == 0 ) return GB_OK;
   if ( flu_in == nullptr || flu_out == nullptr ) return GB_E_INVALID;
   if ( c.dual_energy == GB_DE_ENPY && de_out == nullptr ) return GB_E_INVALID;
   const cudaStream_t st = (cudaStream_t)stream;
   if ( c.precision == GB_PREC_FP64 )
      return close_run<double,P_FP64>( c, flu_in, flu_out, de_out, flux, npg, prm, cp, counts, st );
   if ( c.precision == GB_PREC_MIXED )
      return close_run<float,P_MIXED>( c, flu_in, flu_out, de_out, flux, npg, prm, cp, counts, st );
   return close_run<float,P_FP32>( c, flu_in, flu_out, de_out, flux, npg, prm, cp, counts, st );
}

extern "C"
int gb_fluid_correct_unphysical_mhd_device( gb_fluid_solver *s, const void *flu_in, const void *mag_in,
                                            void *flu_out, const void *mag_out, void *flux, int npg,
                                            const gb_fluid_params *prm, const gb_close_params *cp, int *counts,
                                            void *stream )
{
   using namespace gb;
   if ( s == nullptr || prm == nullptr || cp == nullptr || counts == nullptr ) return GB_E_INVALID;
   gb_fluid_config c;
   if ( gb_fluid_get_config( s, &c ) != GB_OK ) return GB_E_INVALID;
   if ( !cfg_mhd( c ) ) return GB_E_INVALID;   // MHD solvers only
   if ( cp->first_flux_corr < CORR_NONE || cp->first_flux_corr > CORR_3D1D ) return GB_E_INVALID;
   // the directionally split correction is not supported with MHD (Flu_Close.cpp:800-802)
   if ( cp->first_flux_corr == CORR_3D1D ) return GB_E_UNSUPPORTED;
   // HLLC is not an MHD solver (Aux_Check_Parameter.cpp:920-922)
   if ( cp->first_flux_corr != CORR_NONE && cp->first_flux_scheme != RS1_ROE && cp->first_flux_scheme != RS1_HLLE &&
        cp->first_flux_scheme != RS1_HLLD ) return GB_E_INVALID;
   if ( !( prm->dh > 0.0 ) || !( prm->dt >= 0.0 ) || npg < 0 ) return GB_E_INVALID;
   if ( npg == 0 ) return GB_OK;
   if ( flu_in == nullptr || flu_out == nullptr || mag_in == nullptr || mag_out == nullptr ) return GB_E_INVALID;
   const cudaStream_t st = (cudaStream_t)stream;
   if ( c.precision == GB_PREC_FP64 )
      return close_run<double,P_FP64>( c, flu_in, flu_out, nullptr, flux, npg, prm, cp, counts, st, mag_in, mag_out );
   if ( c.precision == GB_PREC_MIXED )
      return close_run<float,P_MIXED>( c, flu_in, flu_out, nullptr, flux, npg, prm, cp, counts, st, mag_in, mag_out );
   return close_run<float,P_FP32>( c, flu_in, flu_out, nullptr, flux, npg, prm, cp, counts, st, mag_in, mag_out );
}
