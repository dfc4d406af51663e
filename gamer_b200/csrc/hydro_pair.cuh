// Float hydrodynamics with sm_100's packed two-lane FP32 arithmetic.
//
// Much of the per-cell work comes in identical pairs: the left and right face of a cell along
// one direction (Hydro_DataReconstruction, CPU_Shared_DataReconstruction.cpp:386-430 and
// :523-560; Hydro_HancockPredict, :2064-2160), the left and right state of a Riemann problem
// (wave speeds and pressures of Hydro_RiemannSolver_HLLC, CPU_Shared_RiemannSolver_HLLC.cpp:392-
// 583), and two cells converted to primitive variables.  The float policies hold such a pair as
// one float2 and evaluate it with add/mul/fma.rn.f32x2 (__fadd2_rn, __fmul2_rn, __ffma2_rn): one
// instruction issues both lanes, and each lane is rounded exactly like the scalar operation it
// replaces.  Comparisons, min/max, reciprocals and square roots stay per lane.
#pragma once
#include "hydro_physics.cuh"

namespace gb {

GB_DEV float2 p_bc( float a )                         { return make_float2( a, a ); }
GB_DEV float2 p_add( float2 a, float2 b )             { return __fadd2_rn( a, b ); }
GB_DEV float2 p_mul( float2 a, float2 b )             { return __fmul2_rn( a, b ); }
GB_DEV float2 p_fma( float2 a, float2 b, float2 c )   { return __ffma2_rn( a, b, c ); }
// a - b, rounded once (b*(-1) is exact)
GB_DEV float2 p_sub( float2 a, float2 b )             { return __ffma2_rn( b, make_float2( -1.f, -1.f ), a ); }

// pressure of two conserved states (pres_con on both lanes; P_MIXED recovers a lane in double
// only where its subtraction cancels, as eint_con does)
template <int P>
GB_DEV float2 pres_con_pair( const Phys<float> &ph, float2 d, float2 ird, float2 a, float2 b, float2 c, float2 e )
{
   float2 m2 = p_mul( a, a );
   m2 = p_fma( b, b, m2 );
   m2 = p_fma( c, c, m2 );
   const float2 ke = p_mul( p_mul( p_bc( 0.5f ), m2 ), ird );
   float2 ei = p_sub( e, ke );
   if constexpr ( P == P_MIXED )
   {
      if ( !( ke.x <= 0.25f*e.x ) ) ei.x = eint_con_double( d.x, a.x, b.x, c.x, e.x );
      if ( !( ke.y <= 0.25f*e.y ) ) ei.y = eint_con_double( d.y, a.y, b.y, c.y, e.y );
   }
   const float2 p = p_mul( ei, p_bc( ph.gm1 ) );
   return make_float2( check_floor( p.x, ph.min_pres ), check_floor( p.y, ph.min_pres ) );
}

// conserved -> primitive of two cells (con2pri on both lanes)
template <int P, int NC>
GB_DEV void con2pri_pair( const Phys<float> &ph, const float2 *u, float2 *w )
{
   const float2 ir = make_float2( 1.f/u[0].x, 1.f/u[0].y );
   w[0] = u[0];
   w[1] = p_mul( u[1], ir );
   w[2] = p_mul( u[2], ir );
   w[3] = p_mul( u[3], ir );
   w[4] = pres_con_pair<P>( ph, u[0], ir, u[1], u[2], u[3], u[4] );
#  pragma unroll
   for (int v=5; v<NC; v++) w[v] = u[v];
}

// the cell-centred conversion of the data reconstruction on two cells (con2pri_cc on both lanes):
// Jeans pressure floor and FracPassive mass fractions
template <int P, int NC>
GB_DEV void con2pri_cc_pair( const Phys<float> &ph, const float2 *u, float2 *w )
{
   con2pri_pair<P,NC>( ph, u, w );
   if ( ph.jeans )
      w[4] = make_float2( check_floor( w[4].x, ph.jeans_coeff*( w[0].x*w[0].x ) ),
                          check_floor( w[4].y, ph.jeans_coeff*( w[0].y*w[0].y ) ) );
   if constexpr ( NC > 5 )
   {
      if ( ph.frac_mask )
      {
         const float2 ir = make_float2( 1.f/u[0].x, 1.f/u[0].y );
#        pragma unroll
         for (int v=5; v<NC; v++) if ( ph.frac_mask & ( 1u << ( v - 5 ) ) ) w[v] = p_mul( w[v], ir );
      }
   }
}

// HLLC with the left and right states' speeds formed as float2 lanes (x = left, y = right);
// the star state and the upwind flux are the scalar riemann_hllc's
// (CPU_Shared_RiemannSolver_HLLC.cpp:392-655, HD version)
template <int D, int P, int NC>
GB_DEV void riemann_hllc_pair( const Phys<float> &ph, const float *L, const float *Rt, float *fo )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   const float2 dd = make_float2( L[0], Rt[0] );
   const float2 ir = make_float2( 1.f/L[0], 1.f/Rt[0] );
   const float2 mn = make_float2( L[n], Rt[n] );
   const float2 uu = p_mul( ir, mn );
   const float2 pp = pres_con_pair<P>( ph, dd, ir, mn, make_float2( L[t1], Rt[t1] ), make_float2( L[t2], Rt[t2] ),
                                       make_float2( L[4], Rt[4] ) );
   const float2 c2 = p_mul( p_mul( p_bc( ph.gamma ), pp ), ir );
   const float2 cs = make_float2( sqrtf( c2.x ), sqrtf( c2.y ) );
   const float2 wm = p_sub( uu, cs );            // (ul - csl, ur - csr)
   const float2 wp = p_add( uu, cs );            // (ul + csl, ur + csr)
   const float ul = uu.x, ur = uu.y, csl = cs.x, csr = cs.y, pl = pp.x, pr = pp.y;
   const float wl = fminf( wm.x, wm.y ), wr = fmaxf( wp.x, wp.y );
   // star-region speed and pressure without u-W differences (HLLC.cpp:562-583)
   const float2 sel = make_float2( ( wm.x < wm.y ) ? csl : ( ul - ur ) + csr,
                                   ( wp.y > wp.x ) ? csr : ( ul - ur ) + csl );
   const float2 tt = p_mul( make_float2( L[0], -Rt[0] ), sel );      // (t1l, t1r)
   const float t1l = tt.x, t1r = tt.y;
   const float t2s = 1.f/( t1l - t1r );
   const float vs  = t2s*( pl - pr + t1l*ul - t1r*ur );
   const float2 xx = p_fma( tt, uu, pp );                           // (pl + t1l*ul, pr + t1r*ur)
   const float ps  = check_floor( t2s*( t1l*xx.y - t1r*xx.x ), ph.min_pres );
   // upwind side: left if V_S >= 0 (HLLC.cpp:589-631)
   const bool left = ( vs >= 0.f );
   const float *U  = left ? L : Rt;
   const float  iu = left ? ir.x : ir.y;
   const float  p  = left ? pl : pr;
   const float  mv = left ? fminf( wl, 0.f ) : fmaxf( wr, 0.f );
   float f[NC], clr, cst;
   con2flux<D,NC>( U, iu, p, f );
#  pragma unroll
   for (int v=0; v<5; v++) f[v] -= mv*U[v];
   if ( left && vs == 0.f && mv == 0.f ) { clr = 1.f; cst = 0.f; }
   else { const float t4 = 1.f/( vs - mv );  clr = t4*vs;  cst = -t4*mv*ps; }
#  pragma unroll
   for (int v=0; v<5; v++) fo[v] = clr*f[v];
   fo[n] += cst;
   fo[4] += cst*vs;
   passive_upwind<NC>( fo, L, Rt, ir.x, ir.y );
}

// Two HLLC problems as the lanes of float2 (e.g. an x face and a y face of the same plane), both
// given in the rotated frame: 0 = density, 1 = normal momentum, 2 and 3 = the transverse momenta
// in the order Hydro_Rotate3D gives them, 4 = energy.  Every lane follows riemann_hllc step by step
// (CPU_Shared_RiemannSolver_HLLC.cpp:392-655, HD version); the upwind choice becomes a per-lane
// select.  A lane whose flux comes out NaN is flagged in nan_x / nan_y for the HLLE rescue.
template <int P>
GB_DEV void riemann_hllc_x2( const Phys<float> &ph, const float2 (&L)[5], const float2 (&Rt)[5], float2 (&fo)[5],
                             bool &nan_x, bool &nan_y )
{
   const float2 irl = make_float2( 1.f/L[0].x, 1.f/L[0].y ), irr = make_float2( 1.f/Rt[0].x, 1.f/Rt[0].y );
   const float2 ul = p_mul( irl, L[1] ), ur = p_mul( irr, Rt[1] );
   const float2 pl = pres_con_pair<P>( ph, L[0],  irl, L[1],  L[2],  L[3],  L[4]  );
   const float2 pr = pres_con_pair<P>( ph, Rt[0], irr, Rt[1], Rt[2], Rt[3], Rt[4] );
   const float2 cl2 = p_mul( p_mul( p_bc( ph.gamma ), pl ), irl ), cr2 = p_mul( p_mul( p_bc( ph.gamma ), pr ), irr );
   const float2 csl = make_float2( sqrtf( cl2.x ), sqrtf( cl2.y ) ), csr = make_float2( sqrtf( cr2.x ), sqrtf( cr2.y ) );
   const float2 wl1 = p_sub( ul, csl ), wl2 = p_sub( ur, csr ), wr1 = p_add( ul, csl ), wr2 = p_add( ur, csr );
   const float2 wl = make_float2( fminf( wl1.x, wl2.x ), fminf( wl1.y, wl2.y ) );
   const float2 wr = make_float2( fmaxf( wr1.x, wr2.x ), fmaxf( wr1.y, wr2.y ) );
   // star-region speed and pressure without u-W differences (HLLC.cpp:562-583)
   const float2 du = p_sub( ul, ur );
   const float2 al = p_add( du, csr ), ar = p_add( du, csl );
   const float2 sl = make_float2( ( wl1.x < wl2.x ) ? csl.x : al.x, ( wl1.y < wl2.y ) ? csl.y : al.y );
   const float2 sr = make_float2( ( wr2.x > wr1.x ) ? csr.x : ar.x, ( wr2.y > wr1.y ) ? csr.y : ar.y );
   const float2 t1l  = p_mul( L[0], sl );
   const float2 nt1r = p_mul( Rt[0], sr );                     // -t1r
   const float2 t1r  = p_mul( nt1r, p_bc( -1.f ) );
   const float2 den  = p_add( t1l, nt1r );                     // t1l - t1r
   const float2 t2s  = make_float2( 1.f/den.x, 1.f/den.y );
   float2 a = p_sub( pl, pr );
   a = p_fma( t1l, ul, a );
   a = p_fma( nt1r, ur, a );
   const float2 vs = p_mul( t2s, a );
   const float2 xl = p_fma( t1l, ul, pl ), xr = p_fma( t1r, ur, pr );
   const float2 pq = p_mul( t2s, p_fma( nt1r, xl, p_mul( t1l, xr ) ) );
   const float2 ps = make_float2( check_floor( pq.x, ph.min_pres ), check_floor( pq.y, ph.min_pres ) );
   // upwind side: left if V_S >= 0 (HLLC.cpp:589-631)
   const bool lx = ( vs.x >= 0.f ), ly = ( vs.y >= 0.f );
   float2 U[5];
#  pragma unroll
   for (int v=0; v<5; v++) U[v] = make_float2( lx ? L[v].x : Rt[v].x, ly ? L[v].y : Rt[v].y );
   const float2 iu = make_float2( lx ? irl.x : irr.x, ly ? irl.y : irr.y );
   const float2 p  = make_float2( lx ? pl.x : pr.x, ly ? pl.y : pr.y );
   const float2 mv = make_float2( lx ? fminf( wl.x, 0.f ) : fmaxf( wr.x, 0.f ),
                                  ly ? fminf( wl.y, 0.f ) : fmaxf( wr.y, 0.f ) );
   // Hydro_Con2Flux of the upwind state, minus mv*U
   const float2 vx = p_mul( iu, U[1] );
   const float2 nmv = p_mul( mv, p_bc( -1.f ) );
   float2 f[5];
   f[0] = p_fma( nmv, U[0], U[1] );
   f[1] = p_fma( nmv, U[1], p_fma( vx, U[1], p ) );
   f[2] = p_fma( nmv, U[2], p_mul( vx, U[2] ) );
   f[3] = p_fma( nmv, U[3], p_mul( vx, U[3] ) );
   f[4] = p_fma( nmv, U[4], p_mul( vx, p_add( U[4], p ) ) );
   const float2 dv = p_sub( vs, mv );
   const float2 t4 = make_float2( 1.f/dv.x, 1.f/dv.y );
   float2 clr = p_mul( t4, vs );
   float2 cst = p_mul( p_mul( p_mul( t4, p_bc( -1.f ) ), mv ), ps );
   if ( lx && vs.x == 0.f && mv.x == 0.f ) { clr.x = 1.f;  cst.x = 0.f; }
   if ( ly && vs.y == 0.f && mv.y == 0.f ) { clr.y = 1.f;  cst.y = 0.f; }
#  pragma unroll
   for (int v=0; v<5; v++) fo[v] = p_mul( clr, f[v] );
   fo[1] = p_add( fo[1], cst );
   fo[4] = p_fma( cst, vs, fo[4] );
   nan_x = nan_y = false;
#  pragma unroll
   for (int v=0; v<5; v++) { nan_x |= ( fo[v].x != fo[v].x );  nan_y |= ( fo[v].y != fo[v].y ); }
}

// PLM face states of both faces along D, primitive -> conserved, and the Hancock flux difference
// (the float2 counterpart of recon_dir; fc[D][v] = (left face, right face) of variable v); CHARR:
// PLM with CHAR_RECONSTRUCTION
template <int D, int P, int NC, bool CHARR, bool HANC = true>
GB_DEV void recon_dir_pair( const Phys<float> &ph, const float *cc, const float *pl, const float *pr,
                            int lim, float coeff, bool clamp, float2 (&fc)[3][NC], float (&fpres)[6],
                            float (&acc)[NC] )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   float2 w[NC];
   if constexpr ( CHARR )
   {
      float fl[NC], fr[NC];
      plm_faces_char<D,NC>( ph, pl, cc, pr, lim, coeff, fl, fr );
#     pragma unroll
      for (int v=0; v<NC; v++) w[v] = make_float2( fl[v], fr[v] );
   }
   else
   {
#     pragma unroll
      for (int v=0; v<NC; v++)
      {
         float fl, fr;
         plm_faces( pl[v], cc[v], pr[v], lim, coeff, clamp, fl, fr );
         w[v] = make_float2( fl, fr );
      }
   }
   fpres[2*D] = w[4].x;  fpres[2*D+1] = w[4].y;
   // Hydro_Pri2Con + Hydro_ConEint2Etot
   float2 *u = fc[D];
   u[0] = w[0];
   u[1] = p_mul( w[0], w[1] );
   u[2] = p_mul( w[0], w[2] );
   u[3] = p_mul( w[0], w[3] );
   float2 v2 = p_mul( w[1], w[1] );
   v2 = p_fma( w[2], w[2], v2 );
   v2 = p_fma( w[3], w[3], v2 );
   u[4] = p_fma( w[4], p_bc( ph.inv_gm1 ), p_mul( p_mul( p_bc( 0.5f ), w[0] ), v2 ) );
#  pragma unroll
   for (int v=5; v<NC; v++) u[v] = w[v];
   if constexpr ( NC > 5 )
   {
      if ( ph.frac_mask )
      {
#        pragma unroll
         for (int v=5; v<NC; v++) if ( ph.frac_mask & ( 1u << ( v - 5 ) ) ) u[v] = p_mul( u[v], w[0] );
      }
   }
   if constexpr ( !HANC ) return;    // MHM_RP: no Hancock half step
   // fluxes of both faces from their primitive states (Hydro_Con2Flux)
   const float2 vx = w[n], pres = w[4];
   float2 f[NC];
   f[0]  = u[n];
   f[n]  = p_fma( vx, u[n], pres );
   f[t1] = p_mul( vx, u[t1] );
   f[t2] = p_mul( vx, u[t2] );
   f[4]  = p_mul( vx, p_add( u[4], pres ) );
#  pragma unroll
   for (int v=5; v<NC; v++) f[v] = p_mul( u[v], vx );
   // accumulated in the reference's order F1-F0+F3-F2+F5-F4
#  pragma unroll
   for (int v=0; v<NC; v++)
   {
      if constexpr ( D == 0 ) acc[v] = f[v].y - f[v].x;
      else                    acc[v] = ( acc[v] + f[v].y ) - f[v].x;
   }
}

// Hydro_CheckMinEintInEngy of two face states at once: the float test of P_MIXED (see
// floor_eint_in_engy) on both lanes, the per-lane evaluation only near the floor
template <int P>
GB_DEV float2 floor_eint_pair( const Phys<float> &ph, float2 d, float2 mx, float2 my, float2 mz, float2 e )
{
   const float2 ird = make_float2( 1.f/d.x, 1.f/d.y );
   float2 m2 = p_mul( mx, mx );
   m2 = p_fma( my, my, m2 );
   m2 = p_fma( mz, mz, m2 );
   const float2 ke = p_mul( p_mul( p_bc( 0.5f ), m2 ), ird );
   if constexpr ( P == P_MIXED )
   {
      const float2 ein = p_sub( e, ke );
      const float2 ae  = p_add( make_float2( fabsf( e.x ), fabsf( e.y ) ), make_float2( fabsf( ke.x ), fabsf( ke.y ) ) );
      const float2 thr = p_fma( p_bc( 16.f*FLT_EPSILON ), ae, p_bc( ph.min_eint ) );
      if ( ein.x > thr.x && ein.y > thr.y ) return e;
      return make_float2( floor_eint_in_engy<P>( ph, d.x, mx.x, my.x, mz.x, e.x ),
                          floor_eint_in_engy<P>( ph, d.y, mx.y, my.y, mz.y, e.y ) );
   }
   else
   {
      const float2 ein = p_sub( e, ke );
      const float eo0 = check_floor( ein.x, ph.min_eint ), eo1 = check_floor( ein.y, ph.min_eint );
      return make_float2( ( ein.x == eo0 ) ? e.x : e.x - ein.x + eo0,
                          ( ein.y == eo1 ) ? e.y : e.y - ein.y + eo1 );
   }
}

// Hancock half step on the six face states, MHM_CHECK_PREDICT reset and floors
// (the float2 counterpart of hancock_finish)
template <int P, int NC>
GB_DEV void hancock_finish_pair( const Phys<float> &ph, float dt_dh2, float2 (&fc)[3][NC], const float (&fpres)[6],
                                 const float (&acc)[NC], const float *g_cc, size_t g_stride, bool &reset )
{
#  pragma unroll
   for (int v=0; v<NC; v++)
   {
      const float2 df = p_bc( dt_dh2*acc[v] );
#     pragma unroll
      for (int d=0; d<3; d++) fc[d][v] = p_sub( fc[d][v], df );
   }
   bool bad = false;
#  pragma unroll
   for (int d=0; d<3; d++)
   {
#     pragma unroll
      for (int s=0; s<2; s++)
      {
         const float dd = s ? fc[d][0].y : fc[d][0].x, e = s ? fc[d][4].y : fc[d][4].x, p = fpres[2*d+s];
         bad |= !( dd >= FLT_MIN && dd <= FLT_MAX );
         bad |= !( e  >= FLT_MIN && e  <= FLT_MAX );
         bad |= !( p  >= 0.f     && p  <= FLT_MAX );
      }
   }
   reset = bad;
   if ( bad )
   {
#     pragma unroll
      for (int v=0; v<NC; v++)
      {
         const float c = g_cc[v*g_stride];
#        pragma unroll
         for (int d=0; d<3; d++) fc[d][v] = p_bc( c );
      }
   }
   else
   {
#     pragma unroll
      for (int d=0; d<3; d++)
      {
         fc[d][0] = make_float2( fmaxf( fc[d][0].x, ph.min_dens ), fmaxf( fc[d][0].y, ph.min_dens ) );
         fc[d][4] = floor_eint_pair<P>( ph, fc[d][0], fc[d][1], fc[d][2], fc[d][3], fc[d][4] );
#        pragma unroll
         for (int v=5; v<NC; v++)
            if ( ph.pfloor & ( 1u << v ) ) fc[d][v] = make_float2( fmaxf( fc[d][v].x, FLT_MIN ), fmaxf( fc[d][v].y, FLT_MIN ) );
      }
   }
}

} // namespace gb
