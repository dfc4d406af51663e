// Per-cell and per-face hydrodynamics of the MHM patch-group solver (ideal gas, no MHD).
//
// The reference evaluates these through EoS function pointers and rotates state vectors in
// memory (Hydro_Rotate3D, src/Model_Hydro/CPU_Hydro/CPU_Shared_FluUtility.cpp:93).  Here the face
// direction D is a template parameter, so rotation is compile-time index remapping, the gamma-law
// EoS is inlined, and the precision policy P decides which recoveries run in double.
//
// The branch structure of every routine is the reference's (wave-speed choices, star-region sign,
// rescue and reset conditions); the arithmetic is rearranged only where the result is the same up
// to round-off:
//   * a reciprocal 1/rho is formed once and multiplied instead of repeated divisions;
//   * the Hancock half-step fluxes are formed from the primitive face state (rho, v, P) that the
//     conserved face state was built from, instead of recovering v and P from it again;
//   * PLM face values skip the clamp to the neighbour values when the limiter bounds the slope by
//     theta*min(|dL|,|dR|) with theta < 2, for which the clamp can never act.
#pragma once
#include <type_traits>
#include "gb_common.cuh"

namespace gb {

template <typename R>
struct Phys {
   R gamma, gm1, inv_gm1;             // EoS_AuxArray_Flt[0..2] (src/EoS/Gamma/CPU_EoS_Gamma.cpp)
   R min_dens, min_pres, min_eint;
   R de_switch;
   R jeans_coeff = R(0);              // JeansMinPres_Coeff (used when jeans != 0)
   int jeans = 0;                     // JeansMinPres
   unsigned frac_mask = 0u;           // FracPassive: bit p = passive scalar p reconstructed as a mass
                                      // fraction (0 = FracPassive off)
   unsigned pfloor = 0u;              // PassiveFloor: bit v = variable v (v >= 5) floored at TINY_NUMBER
};

// ---------------------------------------------------------------------------------------------
// internal energy E - 1/2 |m|^2 / rho  (Hydro_Con2Eint, CPU_Shared_FluUtility.cpp:1259), with the
// reciprocal density ird given.
// P_MIXED does the recovery in double wherever the subtraction cancels: when the kinetic energy is
// at most E/4, the float result E - K carries a relative error below ~2.2 float epsilons (K's own
// ~5 eps error is divided by E - K >= 3K), i.e. within two float ulps of the double result, so the
// double evaluation is kept for K > E/4 (Mach >~ 1.3 for gamma = 5/3), negative or NaN input.
// ---------------------------------------------------------------------------------------------
// the double evaluation, out of line: it is the rare path of every call site
static __device__ __noinline__ float eint_con_double( float d, float a, float b, float c, float e )
{
   const double m2 = (double)a*(double)a + (double)b*(double)b + (double)c*(double)c;
   return (float)( (double)e - 0.5*m2*rcp_dd( (double)d ) );
}

template <int P, typename R>
GB_DEV R eint_con( R d, R ird, R a, R b, R c, R e )
{
   if constexpr ( P == P_MIXED )
   {
      const R ke = R(0.5)*( a*a + b*b + c*c )*ird;
      if ( ke <= R(0.25)*e ) return e - ke;
      return (R)eint_con_double( (float)d, (float)a, (float)b, (float)c, (float)e );
   }
   else
      return e - R(0.5)*( a*a + b*b + c*c )*ird;
}

// pressure with floor (Hydro_Con2Pres, CPU_Shared_FluUtility.cpp:1165)
template <int P, typename R>
GB_DEV R pres_con( const Phys<R> &ph, R d, R ird, R a, R b, R c, R e )
{
   return check_floor( eint_con<P>( d, ird, a, b, c, e )*ph.gm1, ph.min_pres );
}

// physical flux along D of a conserved state with known pressure and 1/rho
// (Hydro_Con2Flux, CPU_Shared_FluUtility.cpp:458)
template <int D, int NC, typename R>
GB_DEV void con2flux( const R *u, R ird, R pres, R *f )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   const R vx = ird*u[n];
   f[0]  = u[n];
   f[n]  = vx*u[n] + pres;
   f[t1] = vx*u[t1];
   f[t2] = vx*u[t2];
   f[4]  = vx*( u[4] + pres );
#  pragma unroll
   for (int v=5; v<NC; v++) f[v] = u[v]*vx;
}

// the same flux of a face state built from the primitive state w (velocity w[n], pressure w[4])
template <int D, int NC, typename R>
GB_DEV void pri_con2flux( const R *w, const R *u, R *f )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   const R vx = w[n], pres = w[4];
   f[0]  = u[n];
   f[n]  = vx*u[n] + pres;
   f[t1] = vx*u[t1];
   f[t2] = vx*u[t2];
   f[4]  = vx*( u[4] + pres );
#  pragma unroll
   for (int v=5; v<NC; v++) f[v] = u[v]*vx;
}

// conserved -> primitive (Hydro_Con2Pri, CPU_Shared_FluUtility.cpp:209)
template <int P, int NC, typename R>
GB_DEV void con2pri( const Phys<R> &ph, const R *u, R *w )
{
   const R ir = R(1)/u[0];
   w[0] = u[0];
   w[1] = u[1]*ir;
   w[2] = u[2]*ir;
   w[3] = u[3]*ir;
   w[4] = pres_con<P>( ph, u[0], ir, u[1], u[2], u[3], u[4] );
#  pragma unroll
   for (int v=5; v<NC; v++) w[v] = u[v];
}

// the cell-centred conversion of the data reconstruction (Hydro_Con2Pri as called by
// Hydro_DataReconstruction, CPU_Shared_DataReconstruction.cpp:323): con2pri, then the Jeans
// pressure floor P = max(P, JeansMinPres_Coeff*rho^2) and the mass fractions of the FracPassive
// scalars (CPU_Shared_FluUtility.cpp:272-296).  The Riemann solvers convert without either.
template <int P, int NC, typename R>
GB_DEV void con2pri_cc( const Phys<R> &ph, const R *u, R *w )
{
   con2pri<P,NC>( ph, u, w );
   if ( ph.jeans ) w[4] = check_floor( w[4], ph.jeans_coeff*( w[0]*w[0] ) );
   if constexpr ( NC > 5 )
   {
      if ( ph.frac_mask )
      {
         const R ir = R(1)/u[0];
#        pragma unroll
         for (int v=5; v<NC; v++) if ( ph.frac_mask & ( 1u << ( v - 5 ) ) ) w[v] *= ir;
      }
   }
}

// primitive -> conserved (Hydro_Pri2Con, CPU_Shared_FluUtility.cpp:343 + Hydro_ConEint2Etot :1299);
// the kinetic energy is formed as 1/2 rho v^2 from the primitive velocity; FracPassive scalars go
// back from mass fraction to mass density
template <int NC, typename R>
GB_DEV void pri2con( const Phys<R> &ph, const R *w, R *u )
{
   u[0] = w[0];
   u[1] = w[0]*w[1];
   u[2] = w[0]*w[2];
   u[3] = w[0]*w[3];
   u[4] = R(0.5)*w[0]*( w[1]*w[1] + w[2]*w[2] + w[3]*w[3] ) + w[4]*ph.inv_gm1;
#  pragma unroll
   for (int v=5; v<NC; v++) u[v] = w[v];
   if constexpr ( NC > 5 )
   {
      if ( ph.frac_mask )
      {
#        pragma unroll
         for (int v=5; v<NC; v++) if ( ph.frac_mask & ( 1u << ( v - 5 ) ) ) u[v] *= w[0];
      }
   }
}

// passive scalars of a Riemann flux are upwinded with the mass flux (e.g. HLLC.cpp:633-647)
template <int NC, typename R>
GB_DEV void passive_upwind( R *f, const R *L, const R *Rt, R irl, R irr )
{
   if constexpr ( NC > 5 )
   {
      if ( f[0] >= R(0) ) { const R vx = f[0]*irl;
#                           pragma unroll
                            for (int v=5; v<NC; v++) f[v] = L[v]*vx; }
      else                { const R vx = f[0]*irr;
#                           pragma unroll
                            for (int v=5; v<NC; v++) f[v] = Rt[v]*vx; }
   }
}

// ---------------------------------------------------------------------------------------------
// HLLE, Davis wave speeds (CPU_Shared_RiemannSolver_HLLE.cpp:302-700, HD version)
// ---------------------------------------------------------------------------------------------
template <int D, int P, int NC, typename R>
GB_DEV void riemann_hlle( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   const R irl = R(1)/L[0], irr = R(1)/Rt[0];
   const R ul = irl*L[n], ur = irr*Rt[n];
   const R pl = pres_con<P>( ph, L[0],  irl, L[n],  L[t1],  L[t2],  L[4]  );
   const R pr = pres_con<P>( ph, Rt[0], irr, Rt[n], Rt[t1], Rt[t2], Rt[4] );
   const R cfl = gsqrt( ph.gamma*pl*irl ), cfr = gsqrt( ph.gamma*pr*irr );
   R mvl = gmin( ul - cfl, ur - cfr );
   R mvr = gmax( ul + cfl, ur + cfr );
   mvl = gmin( mvl, R(0) );
   mvr = gmax( mvr, R(0) );
   R fl[NC], fr[NC];
   con2flux<D,NC>( L,  irl, pl, fl );
   con2flux<D,NC>( Rt, irr, pr, fr );
#  pragma unroll
   for (int v=0; v<5; v++) { fl[v] -= mvl*L[v];  fr[v] -= mvr*Rt[v]; }
   if ( mvl == R(0) && mvr == R(0) )
   {
#     pragma unroll
      for (int v=0; v<5; v++) fo[v] = fl[v];
   }
   else
   {
      const R id = R(1)/( mvr - mvl );
#     pragma unroll
      for (int v=0; v<5; v++) fo[v] = id*( mvr*fl[v] - mvl*fr[v] );
   }
   passive_upwind<NC>( fo, L, Rt, irl, irr );
}

// The HLLE solver on the rare paths (NaN rescue of HLLC, failed intermediate state of Roe) is kept
// out of line, with the states passed by value, so that it adds no code to the hot loops.
template <int NC, typename R> struct FaceState { R v[NC]; };

template <int D, int P, int NC, typename R>
__device__ __noinline__ FaceState<NC,R> riemann_hlle_rare( const Phys<R> ph, const FaceState<NC,R> L,
                                                           const FaceState<NC,R> Rt )
{
   FaceState<NC,R> f;
   riemann_hlle<D,P,NC>( ph, L.v, Rt.v, f.v );
   return f;
}

template <int D, int P, int NC, typename R>
GB_DEV void riemann_hlle_outlined( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   FaceState<NC,R> l, r;
#  pragma unroll
   for (int v=0; v<NC; v++) { l.v[v] = L[v];  r.v[v] = Rt[v]; }
   const FaceState<NC,R> f = riemann_hlle_rare<D,P,NC>( ph, l, r );
#  pragma unroll
   for (int v=0; v<NC; v++) fo[v] = f.v[v];
}

// ---------------------------------------------------------------------------------------------
// HLLC, Davis wave speeds (CPU_Shared_RiemannSolver_HLLC.cpp:392-655, HD version)
// ---------------------------------------------------------------------------------------------
template <int D, int P, int NC, typename R>
GB_DEV void riemann_hllc( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   const R irl = R(1)/L[0], irr = R(1)/Rt[0];
   const R ul = irl*L[n], ur = irr*Rt[n];
   const R pl = pres_con<P>( ph, L[0],  irl, L[n],  L[t1],  L[t2],  L[4]  );
   const R pr = pres_con<P>( ph, Rt[0], irr, Rt[n], Rt[t1], Rt[t2], Rt[4] );
   const R csl = gsqrt( ph.gamma*pl*irl ), csr = gsqrt( ph.gamma*pr*irr );
   const R wl1 = ul - csl, wl2 = ur - csr, wr1 = ul + csl, wr2 = ur + csr;
   const R wl = gmin( wl1, wl2 ), wr = gmax( wr1, wr2 );
   // star-region speed and pressure without u-W differences (HLLC.cpp:562-583)
   const R t1l = +L[0]*( ( wl1 < wl2 ) ? csl : ( ul - ur ) + csr );
   const R t1r = -Rt[0]*( ( wr2 > wr1 ) ? csr : ( ul - ur ) + csl );
   const R t2s = R(1)/( t1l - t1r );
   const R vs  = t2s*( pl - pr + t1l*ul - t1r*ur );
   const R ps  = check_floor( t2s*( t1l*( pr + t1r*ur ) - t1r*( pl + t1l*ul ) ), ph.min_pres );
   // upwind side: left if V_S >= 0 (HLLC.cpp:589-631)
   const bool left = ( vs >= R(0) );
   const R *U  = left ? L : Rt;
   const R  ir = left ? irl : irr;
   const R  p  = left ? pl : pr;
   const R  mv = left ? gmin( wl, R(0) ) : gmax( wr, R(0) );
   R f[NC], clr, cst;
   con2flux<D,NC>( U, ir, p, f );
#  pragma unroll
   for (int v=0; v<5; v++) f[v] -= mv*U[v];
   if ( left && vs == R(0) && mv == R(0) ) { clr = R(1); cst = R(0); }
   else { const R t4 = R(1)/( vs - mv );  clr = t4*vs;  cst = -t4*mv*ps; }
#  pragma unroll
   for (int v=0; v<5; v++) fo[v] = clr*f[v];
   fo[n] += cst;
   fo[4] += cst*vs;
   passive_upwind<NC>( fo, L, Rt, irl, irr );
}

// ---------------------------------------------------------------------------------------------
// Roe with the intermediate-state check falling back to HLLE
// (CPU_Shared_RiemannSolver_Roe.cpp:88-719, HD version; CHECK_INTERMEDIATE = HLLE, include/CUFLU.h:178-186).
// The reference defines CHECK_INTERMEDIATE only in builds whose RSOLVER is ROE, so the first-order
// Roe fluxes of Flu_Close run without the check in other builds (CHECK = false).
// ---------------------------------------------------------------------------------------------
template <int D, int P, int NC, typename R, bool CHECK = true>
GB_DEV void riemann_roe( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   const R irl = R(1)/L[0], irr = R(1)/Rt[0];
   const R pl = pres_con<P>( ph, L[0],  irl, L[n],  L[t1],  L[t2],  L[4]  );
   const R pr = pres_con<P>( ph, Rt[0], irr, Rt[n], Rt[t1], Rt[t2], Rt[4] );
   const R hl = irl*( L[4] + pl ), hr = irr*( Rt[4] + pr );
   const R sl = gsqrt( L[0] ), sr = gsqrt( Rt[0] );
   const R rho = sl*sr, irho = R(1)/rho;
   const R isl = R(1)/sl, isr = R(1)/sr, iss = R(1)/( sl + sr );
   const R u = iss*( isl*L[n]  + isr*Rt[n]  );
   const R v = iss*( isl*L[t1] + isr*Rt[t1] );
   const R w = iss*( isl*L[t2] + isr*Rt[t2] );
   const R V2 = u*u + v*v + w*w;
   const R H  = iss*( sl*hl + sr*hr );
   R gp = ph.gm1*( H - R(0.5)*V2 );
   gp = ph.gamma*irho*check_floor( gp*rho/ph.gamma, ph.min_pres );
   const R a2 = gp, a = gsqrt( a2 );
   R fl[NC], fr[NC];
   con2flux<D,NC>( L,  irl, pl, fl );
   con2flux<D,NC>( Rt, irr, pr, fr );
   if ( u - a >= R(0) ) {
#     pragma unroll
      for (int k=0; k<NC; k++) fo[k] = fl[k];
      return;
   }
   if ( u + a <= R(0) ) {
#     pragma unroll
      for (int k=0; k<NC; k++) fo[k] = fr[k];
      return;
   }
   // jumps and wave amplitudes in the rotated frame (index 0 density, 1 normal, 2/3 transverse, 4 energy)
   const R J0 = Rt[0] - L[0], J1 = Rt[n] - L[n], J2 = Rt[t1] - L[t1], J3 = Rt[t2] - L[t2], J4 = Rt[4] - L[4];
   R A[5];
   A[2] = J2 - v*J0;
   A[3] = J3 - w*J0;
   A[1] = ph.gm1/a2*( J0*( H - u*u ) + u*J1 - J4 + v*A[2] + w*A[3] );
   A[0] = R(0.5)/a*( J0*( u + a ) - J1 - a*A[1] );
   A[4] = J0 - A[0] - A[1];
   // right eigenvectors (columns): rows = (rho, m_n, m_t1, m_t2, E)
   const R RE[5][5] = { { R(1),    R(1),       R(0), R(0), R(1)    },
                        { u - a,   u,          R(0), R(0), u + a   },
                        { v,       v,          R(1), R(0), v       },
                        { w,       w,          R(0), R(1), w       },
                        { H - u*a, R(0.5)*V2,  v,    w,    H + u*a } };
   // the intermediate states must have positive density and pressure (Roe.cpp, section 8);
   // eigenvalues are (u-a, u, u, u, u+a): only the states after wave 0 and after wave 3 are distinct
   if constexpr ( CHECK )
   {
      R I0 = L[0], I1 = L[n], I2 = L[t1], I3 = L[t2], I4 = L[4];
#     pragma unroll
      for (int t=0; t<4; t++)
      {
         I0 += A[t]*RE[0][t];  I1 += A[t]*RE[1][t];  I2 += A[t]*RE[2][t];
         I3 += A[t]*RE[3][t];  I4 += A[t]*RE[4][t];
         if ( t == 0 || t == 3 )
         {
            const R ip = eint_con<P>( I0, R(1)/I0, I1, I2, I3, I4 )*ph.gm1;
            if ( I0 <= R(0) || ip <= R(0) ) { riemann_hlle_outlined<D,P,NC>( ph, L, Rt, fo ); return; }
         }
      }
   }
   const R ev[5] = { u - a, u, u, u, u + a };
#  pragma unroll
   for (int k=0; k<5; k++) A[k] *= gabs( ev[k] );
   const int map[5] = { 0, n, t1, t2, 4 };
#  pragma unroll
   for (int k=0; k<5; k++)
   {
      R s = fl[map[k]] + fr[map[k]];
#     pragma unroll
      for (int t=0; t<5; t++) s -= A[t]*RE[k][t];
      fo[map[k]] = R(0.5)*s;
   }
   passive_upwind<NC>( fo, L, Rt, irl, irr );
}

// ---------------------------------------------------------------------------------------------
// Exact solver (CPU_Shared_RiemannSolver_Exact.cpp:62-432, hydro, gamma law): the star pressure by
// bisection of f_L(p) + f_R(p) + (u_R - u_L) until |f| < MAX_ERROR (1e-14 in double, 1e-6 in
// float, include/Macro.h:1023-1031) or the midpoint equals a bound, then the sampled state at the
// face.  The reference's loops carry no count; here the bracket doubling stops after 2100 steps
// and the bisection after 2200, more than the exponent range of a double allows either to take on
// finite input, and a state that is not finite comes out as NaN flux (for the HLLE rescue).
// ---------------------------------------------------------------------------------------------
// Solve_f (:360-405)
template <typename R>
GB_DEV R exact_f( R rho, R p, R ps, const Phys<R> &ph )
{
   const R gm1 = ph.gamma - R(1), gp1 = ph.gamma + R(1);
   if ( ps > p )
   {
      const R A = R(2)/( rho*gp1 ), B = p*gm1/gp1;
      return ( ps - p )*gsqrt( A/( ps + B ) );
   }
   const R a = gsqrt( ph.gamma*p/rho );
   return R(2)*a*( gpow( ps/p, R(0.5)*gm1/ph.gamma ) - R(1) )/gm1;
}

// Set_Flux (:409-425) of a rotated primitive state
template <typename R>
GB_DEV void exact_set_flux( R *f, const R *w, const Phys<R> &ph )
{
   const R gm1 = ph.gamma - R(1);
   f[0] = w[0]*w[1];
   f[1] = w[0]*w[1]*w[1] + w[4];
   f[2] = w[0]*w[1]*w[2];
   f[3] = w[0]*w[1]*w[3];
   f[4] = w[1]*( R(0.5)*w[0]*( w[1]*w[1] + w[2]*w[2] + w[3]*w[3] ) + w[4]/gm1 + w[4] );
}

// d f / d p* of Solve_f (the shock and rarefaction branches of exact_f differentiated in p*):
// shock sqrt(A/(p*+B)) (1 - (p*-p)/(2(p*+B))), rarefaction (p*/p)^(-(gamma+1)/(2 gamma)) / (rho a)
template <typename R>
GB_DEV R exact_fprime( R rho, R p, R ps, const Phys<R> &ph )
{
   const R gm1 = ph.gamma - R(1), gp1 = ph.gamma + R(1);
   if ( ps > p )
   {
      const R A = R(2)/( rho*gp1 ), B = p*gm1/gp1;
      return gsqrt( A/( ps + B ) )*( R(1) - R(0.5)*( ps - p )/( ps + B ) );
   }
   const R a = gsqrt( ph.gamma*p/rho );
   return gpow( ps/p, -R(0.5)*gp1/ph.gamma )/( rho*a );
}

// the star pressure of the rotated primitive states L, Rr (CPU_Shared_RiemannSolver_Exact.cpp:
// 110-170): bracket, then bisection until |f| < max_err or the midpoint equals a bound
template <typename R>
GB_DEV R exact_pstar( const R *L, const R *Rr, const Phys<R> &ph, R max_err )
{
   const R du = Rr[1] - L[1];
   R f = R(0), ps, bound[2], cmp[2];
   bound[0] = gmin( L[4], Rr[4] );
   bound[1] = gmax( L[4], Rr[4] );
   for (int i=0; i<2; i++) cmp[i] = exact_f( L[0], L[4], bound[i], ph ) + exact_f( Rr[0], Rr[4], bound[i], ph ) + du;
   if ( cmp[0]*cmp[1] > R(0) )
   {
      if ( cmp[0] > R(0) ) { bound[1] = bound[0];  bound[0] = R(0); }
      else if ( cmp[1] < R(0) )
      {
         bound[0] = bound[1];
         bound[1] = R(2)*bound[0];
         for (int it=0; it<2100; it++)
         {
            for (int i=0; i<2; i++) cmp[i] = exact_f( L[0], L[4], bound[i], ph ) + exact_f( Rr[0], Rr[4], bound[i], ph ) + du;
            if ( !( cmp[0]*cmp[1] > R(0) ) ) break;
            bound[0] = bound[1];
            bound[1] = bound[0]*R(2);
         }
      }
   }
   int it = 0;
   do
   {
      ps = R(0.5)*( bound[0] + bound[1] );
      if ( ps == bound[0] || ps == bound[1] ) break;
      f = exact_f( L[0], L[4], ps, ph ) + exact_f( Rr[0], Rr[4], ps, ph ) + du;
      if ( f > R(0) ) bound[1] = ps;
      else            bound[0] = ps;
   }
   while ( gabs( f ) >= max_err && ++it < 2200 );
   return ps;
}

template <int D, int P, int NC, typename R>
GB_DEV void riemann_exact( const Phys<R> &ph, const R *Lc, const R *Rc, R *fo )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   typedef typename ScalarOf<R>::type S;
   const R max_err = sizeof(S) == 8 ? R(1.0e-14) : R(1.0e-6);
   // Gamma_m1 is EoS_AuxArray_Flt[1] here, while Solve_f and Set_Flux form Gamma - 1 themselves
   const R g = ph.gamma, gm1 = ph.gm1, gp1 = g + R(1), c = gm1/gp1;
   R wl[NC], wr[NC];
   con2pri<P,NC>( ph, Lc, wl );
   con2pri<P,NC>( ph, Rc, wr );
   // rotated primitive states: density, normal velocity, transverse velocities, pressure
   R L[5]  = { wl[0], wl[n], wl[t1], wl[t2], wl[4] };
   R Rr[5] = { wr[0], wr[n], wr[t1], wr[t2], wr[4] };
   R Ls[5], Rs[5];
   Ls[2] = L[2];  Ls[3] = L[3];  Rs[2] = Rr[2];  Rs[3] = Rr[3];
   if constexpr ( ScalarOf<R>::dual )
   {
      // derivatives (the adjoint): the root found on the values, as in the plain evaluation, and
      // its tangents from the implicit function theorem, dp* = -(dF at fixed p*) / (dF/dp*), since
      // the bisection midpoints carry the tangents of the bracket, not of the root
      const Phys<S> sph = value_phys( ph );
      S Lv[5], Rv[5];
#     pragma unroll
      for (int v=0; v<5; v++) { Lv[v] = L[v].v;  Rv[v] = Rr[v].v; }
      const S ps = exact_pstar( Lv, Rv, sph, S( sizeof(S) == 8 ? 1.0e-14 : 1.0e-6 ) );
      const R pc( (double)ps );
      const R F = exact_f( L[0], L[4], pc, ph ) + exact_f( Rr[0], Rr[4], pc, ph ) + ( Rr[1] - L[1] );
      const S Fp = exact_fprime( Lv[0], Lv[4], ps, sph ) + exact_fprime( Rv[0], Rv[4], ps, sph );
      Ls[4] = pc;
#     pragma unroll
      for (int k=0; k<ScalarOf<R>::ntan; k++) Ls[4].d[k] = -F.d[k]/Fp;
   }
   else Ls[4] = exact_pstar( L, Rr, ph, max_err );
   Rs[4] = Ls[4];
   Ls[1] = R(0.5)*( L[1] + Rr[1] ) + R(0.5)*( exact_f( Rr[0], Rr[4], Rs[4], ph ) - exact_f( L[0], L[4], Ls[4], ph ) );
   Rs[1] = Ls[1];
   if ( Ls[4] > L[4] ) { const R r = Ls[4]/L[4];  Ls[0] = L[0]*( ( r + c )/( c*r + R(1) ) ); }
   else
   {
      Ls[0] = L[0]*gpow( Ls[4]/L[4], R(1)/g );
      const R aL = gsqrt( g*L[4]/L[0] ), as = gsqrt( g*Ls[4]/Ls[0] );
      if ( L[1] < aL && Ls[1] > as )     // sonic rarefaction
      {
         Ls[0] = L[0]*gpow( R(2)/gp1 + c*L[1]/aL, R(2)/gm1 );
         Ls[1] = R(2)*( aL + R(0.5)*gm1*L[1] )/gp1;
         Ls[4] = L[4]*gpow( R(2)/gp1 + c*L[1]/aL, R(2)*g/gm1 );
      }
   }
   if ( Rs[4] > Rr[4] ) { const R r = Rs[4]/Rr[4];  Rs[0] = Rr[0]*( ( r + c )/( c*r + R(1) ) ); }
   else
   {
      Rs[0] = Rr[0]*gpow( Rs[4]/Rr[4], R(1)/g );
      const R aR = gsqrt( g*Rr[4]/Rr[0] ), as = gsqrt( g*Rs[4]/Rs[0] );
      if ( Rr[1] > -aR && Rs[1] < -as )  // sonic rarefaction
      {
         Rs[0] = Rr[0]*gpow( R(2)/gp1 - c*Rr[1]/aR, R(2)/gm1 );
         Rs[1] = R(2)*( -aR + R(0.5)*gm1*Rr[1] )/gp1;
         Rs[4] = Rr[4]*gpow( R(2)/gp1 - c*Rr[1]/aR, R(2)*g/gm1 );
      }
   }
   const R ev1 = Ls[1];
   R ev0, ev4;
   if ( L[4] < Ls[4] ) ev0 = L[1] - gsqrt( g*L[4]/L[0] )*gsqrt( R(0.5)/g*( gp1*Ls[4]/L[4] + gm1 ) );
   else                ev0 = L[1] - gsqrt( g*L[4]/L[0] );
   if ( Rr[4] < Rs[4] ) ev4 = Rr[1] + gsqrt( g*Rr[4]/Rr[0] )*gsqrt( R(0.5)/g*( gp1*Rs[4]/Rr[4] + gm1 ) );
   else                 ev4 = Rr[1] + gsqrt( g*Rr[4]/Rr[0] );
   R f[5];
   if ( gabs( ev1 ) < max_err ) { f[0] = R(0);  f[1] = Ls[4];  f[2] = R(0);  f[3] = R(0);  f[4] = R(0); }
   else if ( ev1 > R(0) ) exact_set_flux( f, ( ev0 > R(0) ) ? L : Ls, ph );
   else                   exact_set_flux( f, ( ev4 < R(0) ) ? Rr : Rs, ph );
   fo[0] = f[0];  fo[n] = f[1];  fo[t1] = f[2];  fo[t2] = f[3];  fo[4] = f[4];
   passive_upwind<NC>( fo, Lc, Rc, R(1)/Lc[0], R(1)/Rc[0] );
}

template <int D, int P, int NC>
GB_DEV void riemann_hllc_pair( const Phys<float> &ph, const float *L, const float *Rt, float *fo );

// dispatch + HLLE rescue on NaN (CPU_Shared_ComputeFlux.cpp:313-362; the reference has no rescue
// when the main solver is Roe or HLLE, include/CUFLU.h:193-208); float HLLC runs the float2 form
// of hydro_pair.cuh
template <int RS, int D, int P, int NC, typename R>
GB_DEV void riemann( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   if constexpr ( RS == RS_HLLC )
   {
      if constexpr ( std::is_same<R, float>::value ) riemann_hllc_pair<D,P,NC>( ph, L, Rt, fo );
      else                                           riemann_hllc<D,P,NC>( ph, L, Rt, fo );
      bool nan = false;
#     pragma unroll
      for (int v=0; v<NC; v++) nan |= ( fo[v] != fo[v] );
      if ( nan ) riemann_hlle_outlined<D,P,NC>( ph, L, Rt, fo );
   }
   else if constexpr ( RS == RS_EXACT )
   {
      riemann_exact<D,P,NC>( ph, L, Rt, fo );
      bool nan = false;
#     pragma unroll
      for (int v=0; v<NC; v++) nan |= ( fo[v] != fo[v] );
      if ( nan ) riemann_hlle_outlined<D,P,NC>( ph, L, Rt, fo );
   }
   else if constexpr ( RS == RS_ROE ) riemann_roe<D,P,NC>( ph, L, Rt, fo );
   else                               riemann_hlle<D,P,NC>( ph, L, Rt, fo );
}

// ---------------------------------------------------------------------------------------------
// slope limiters (Hydro_LimitSlope, CPU_Shared_DataReconstruction.cpp:1918-2032), one variable
// ---------------------------------------------------------------------------------------------
template <typename R>
GB_DEV R limit_slope( R cl, R cc, R cr, int lim, R coeff )
{
   R sl = cc - cl, sr = cr - cc;
   const R sc  = R(0.5)*( sl + sr );
   const R slr = sl*sr;
   if ( !( slr > R(0) ) ) return R(0);
   switch ( lim )
   {
      case LIM_CENTRAL:  return sc;
      case LIM_VANLEER:  return R(2)*slr/( sl + sr );
      case LIM_ALBADA:   return slr*( sl + sr )/( sl*sl + sr*sr );
      case LIM_VL_GMINMOD:
      {
         const R sa = R(2)*sl*sr/( sl + sr );
         sl *= coeff;  sr *= coeff;
         R s = gmin( gabs( sl ), gabs( sr ) );
         s = gmin( gabs( sc ), s );
         s = gmin( gabs( sa ), s );
         return s*gsign( sc );
      }
      case LIM_GMINMOD:
      default:
      {
         sl *= coeff;  sr *= coeff;
         R s = gmin( gabs( sl ), gabs( sr ) );
         s = gmin( gabs( sc ), s );
         return s*gsign( sc );
      }
   }
}

// the clamp of PLM face values to the neighbours is a no-op when |slope| <= theta*min(|dL|,|dR|)
// with theta < 2 (generalized MinMod and vanLeer+generalized MinMod)
GB_DEV bool plm_clamp_needed( int lim, double coeff )
{
   return !( ( lim == LIM_GMINMOD || lim == LIM_VL_GMINMOD ) && coeff < 2.0 );
}

// PLM face values of one variable (CPU_Shared_DataReconstruction.cpp:386-430): slope, then clamp
// each face value between the cell and its neighbour (reflected through the cell value)
template <typename R>
GB_DEV void plm_faces( R cl, R cc, R cr, int lim, R coeff, bool clamp, R &fl, R &fr )
{
   const R s = limit_slope( cl, cc, cr, lim, coeff );
   fl = cc - R(0.5)*s;
   if ( clamp )
   {
      const R mn = ( cc < cl ) ? cc : cl, mx = ( cc > cl ) ? cc : cl;
      fl = ( fl > mn ) ? fl : mn;
      fl = ( fl < mx ) ? fl : mx;
   }
   fr = R(2)*cc - fl;
   if ( clamp )
   {
      const R mn = ( cc < cr ) ? cc : cr, mx = ( cc > cr ) ? cc : cr;
      fr = ( fr > mn ) ? fr : mn;
      fr = ( fr < mx ) ? fr : mx;
   }
   fl = R(2)*cc - fr;
}

// the limiters of limit_slope applied to given left / right / centred (/ van Leer) slopes
template <typename R>
GB_DEV R limit_slopes( R sl, R sr, R sc, R sa, int lim, R coeff )
{
   const R slr = sl*sr;
   if ( !( slr > R(0) ) ) return R(0);
   switch ( lim )
   {
      case LIM_CENTRAL:  return sc;
      case LIM_VANLEER:  return R(2)*slr/( sl + sr );
      case LIM_ALBADA:   return slr*( sl + sr )/( sl*sl + sr*sr );
      case LIM_VL_GMINMOD:
      {
         sl *= coeff;  sr *= coeff;
         R s = gmin( gabs( sl ), gabs( sr ) );
         s = gmin( gabs( sc ), s );
         s = gmin( gabs( sa ), s );
         return s*gsign( sc );
      }
      case LIM_GMINMOD:
      default:
      {
         sl *= coeff;  sr *= coeff;
         R s = gmin( gabs( sl ), gabs( sr ) );
         s = gmin( gabs( sc ), s );
         return s*gsign( sc );
      }
   }
}

// the limited slope vector of the cell cc between cl and cr in its characteristic variables, gamma-law
// EoS, no MHD (Hydro_LimitSlope with Hydro_Pri2Char / Hydro_Char2Pri, CPU_Shared_DataReconstruction.cpp:
// 1436-1576 and :1918-2035): the left, right, centred (and van Leer) slopes of the cell's primitive
// variables are projected onto the characteristic variables of the cell (its own rho and P), limited
// there, and projected back; passive scalars (index >= 5) are limited as they are
template <int D, int NC, typename R>
GB_DEV void char_limited_slopes( const Phys<R> &ph, const R *cl, const R *cc, const R *cr, int lim, R coeff,
                                 R (&s)[NC] )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   R sl[NC], sr[NC], sc[NC], sa[NC];
#  pragma unroll
   for (int v=0; v<NC; v++)
   {
      sl[v] = cc[v] - cl[v];
      sr[v] = cr[v] - cc[v];
      sc[v] = R(0.5)*( sl[v] + sr[v] );
      sa[v] = ( sl[v]*sr[v] > R(0) ) ? R(2)*sl[v]*sr[v]/( sl[v] + sr[v] ) : R(0);
   }
   const R dens = cc[0], pres = cc[4];
   const R a2  = ph.gamma*pres/dens;                     // EoS_DensPres2CSqr, gamma law
   const R ia2 = R(1)/a2, ia = gsqrt( ia2 ), a = gsqrt( a2 );
   // characteristic variables in the rotated order (0, 4: acoustic; 1: entropy; 2, 3: shear)
   auto pri2char = [&]( R *s ) {
      const R q0 = s[0], qn = s[n], qt1 = s[t1], qt2 = s[t2], q4 = s[4];
      s[0] = -R(0.5)*dens*ia*qn + R(0.5)*ia2*q4;
      s[1] = q0 - ia2*q4;
      s[2] = qt1;
      s[3] = qt2;
      s[4] = +R(0.5)*dens*ia*qn + R(0.5)*ia2*q4;
   };
   pri2char( sl );  pri2char( sr );  pri2char( sc );
   if ( lim == LIM_VL_GMINMOD ) pri2char( sa );
#  pragma unroll
   for (int v=0; v<NC; v++) s[v] = limit_slopes( sl[v], sr[v], sc[v], sa[v], lim, coeff );
   {
      const R c0 = s[0], c1 = s[1], c2 = s[2], c3 = s[3], c4 = s[4];
      s[0]  = c0 + c1 + c4;
      s[n]  = a/dens*( -c0 + c4 );
      s[t1] = c2;
      s[t2] = c3;
      s[4]  = a2*( c0 + c4 );
   }
}

// PLM face values of one variable from its limited slope s (CPU_Shared_DataReconstruction.cpp:386-430):
// the left face value is clamped between the cell and its left neighbour, the right one (reflected
// through the cell value) between the cell and its right neighbour, and the left one reflected back
template <typename R>
GB_DEV void plm_clamped_faces( R cl, R cc, R cr, R s, R &fl, R &fr )
{
   R l = cc - R(0.5)*s;
   R mn = ( cc < cl ) ? cc : cl, mx = ( cc > cl ) ? cc : cl;
   l = ( l > mn ) ? l : mn;
   l = ( l < mx ) ? l : mx;
   R r = R(2)*cc - l;
   mn = ( cc < cr ) ? cc : cr;  mx = ( cc > cr ) ? cc : cr;
   r = ( r > mn ) ? r : mn;
   r = ( r < mx ) ? r : mx;
   fr = r;
   fl = R(2)*cc - r;
}

// PLM face values with CHAR_RECONSTRUCTION from the slopes of char_limited_slopes, clamped between
// the cell and its neighbours (which here can act)
template <int D, int NC, typename R>
GB_DEV void plm_faces_char( const Phys<R> &ph, const R *cl, const R *cc, const R *cr, int lim, R coeff,
                            R (&fl)[NC], R (&fr)[NC] )
{
   R s[NC];
   char_limited_slopes<D,NC>( ph, cl, cc, cr, lim, coeff, s );
#  pragma unroll
   for (int v=0; v<NC; v++) plm_clamped_faces( cl[v], cc[v], cr[v], s[v], fl[v], fr[v] );
}

// PPM with CHAR_RECONSTRUCTION: the limited slopes of the left, centre and right cells, each limited
// in its own characteristic variables (the slope pass of Hydro_DataReconstruction PPM,
// CPU_Shared_DataReconstruction.cpp:884-907, through Hydro_LimitSlope :1918-2035)
template <int D, int NC, typename R>
GB_DEV void ppm_char_slopes( const Phys<R> &ph, const R *ll, const R *l, const R *c, const R *r, const R *rr,
                             int lim, R coeff, R *sl, R *sc, R *sr )
{
   R t[NC];
   char_limited_slopes<D,NC>( ph, ll, l, c, lim, coeff, t );
#  pragma unroll
   for (int v=0; v<NC; v++) sl[v] = t[v];
   char_limited_slopes<D,NC>( ph, l, c, r, lim, coeff, t );
#  pragma unroll
   for (int v=0; v<NC; v++) sc[v] = t[v];
   char_limited_slopes<D,NC>( ph, c, r, rr, lim, coeff, t );
#  pragma unroll
   for (int v=0; v<NC; v++) sr[v] = t[v];
}

// PPM face values of one variable from the limited slopes of the left/centre/right cells
// (CPU_Shared_DataReconstruction.cpp:1065-1140, non-ATHENA limiters)
template <typename R>
GB_DEV void ppm_faces( R cl, R cc, R cr, R dl, R dc, R dr, int lim, R &fl, R &fr )
{
   fl = R(0.5)*( cc + cl ) - R(1)/R(6)*( dc - dl );
   fr = R(0.5)*( cc + cr ) - R(1)/R(6)*( dr - dc );
   if ( lim == LIM_CENTRAL )
   {
      if ( ( cc - fl )*( fl - cl ) < R(0) ) fl = R(0.5)*( cc + cl );
      if ( ( cr - fr )*( fr - cc ) < R(0) ) fr = R(0.5)*( cc + cr );
   }
   const R dfc  = fr - fl;
   const R dfc6 = R(6)*( cc - R(0.5)*( fl + fr ) );
   if ( ( fr - cc )*( cc - fl ) <= R(0) ) { fl = cc;  fr = cc; }
   else if ( dfc*dfc6 > +dfc*dfc ) fl = R(3)*cc - R(2)*fr;
   else if ( dfc*dfc6 < -dfc*dfc ) fr = R(3)*cc - R(2)*fl;
   R mn = ( cc < cl ) ? cc : cl, mx = ( cc > cl ) ? cc : cl;
   fl = ( fl > mn ) ? fl : mn;
   fl = ( fl < mx ) ? fl : mx;
   mn = ( cc < cr ) ? cc : cr;  mx = ( cc > cr ) ? cc : cr;
   fr = ( fr > mn ) ? fr : mn;
   fr = ( fr < mx ) ? fr : mx;
}

// Hydro_CheckMinEintInEngy (CPU_Shared_FluUtility.cpp:822).  P_MIXED first tests the float
// estimate: when it clears the floor by more than its own round-off the double recovery would
// leave E unchanged as well, so it is only computed near the floor.
template <int P, typename R>
GB_DEV R floor_eint_in_engy( const Phys<R> &ph, R d, R mx, R my, R mz, R e )
{
   const R ird = R(1)/d;
   if constexpr ( P == P_MIXED )
   {
      const R ke  = R(0.5)*( mx*mx + my*my + mz*mz )*ird;
      const R ein = e - ke;
      if ( ein > ph.min_eint + R(16)*Lim<R>::eps()*( gabs( e ) + gabs( ke ) ) ) return e;
   }
   const R ein  = eint_con<P>( d, ird, mx, my, mz, e );
   const R eout = check_floor( ein, ph.min_eint );
   return ( ein == eout ) ? e : e - ein + eout;
}

// Hydro_IsUnphysical, UNPHY_MODE_CONS, EOS_GAMMA, no MHD (CPU_Shared_FluUtility.cpp:843-960);
// passive scalars are floored (dual-energy field) when NC > 5
template <int P, int NC, typename R>
GB_DEV bool is_unphysical( const R *u, unsigned pfloor )
{
   // each test is written as the range a physical value lies in, so that a NaN (for which every
   // comparison is false) fails it without a test of its own
   bool ok = true;
#  pragma unroll
   for (int v=0; v<NC; v++)
   {
      if ( v >= 1 && v <= 3 ) ok &= ( u[v] >= -Lim<R>::huge() && u[v] <= Lim<R>::huge() );
      else if ( v < 5 )       ok &= ( u[v] > R(0) && u[v] <= Lim<R>::huge() );
      else                    ok &= ( u[v] >= -Lim<R>::huge() && u[v] <= Lim<R>::huge() ) &&
                                    !( u[v] < R(0) && ( pfloor & ( 1u << v ) ) );
   }
   const R ei = eint_con<P>( u[0], R(1)/u[0], u[1], u[2], u[3], u[4] );
   ok &= ( ei >= R(-3)*u[4]*Lim<R>::eps() && ei <= Lim<R>::huge() );
   return !ok;
}

// Hydro_NormalizePassive (CPU_Shared_FluUtility.cpp:1536-1561): the listed passive scalars (idx:
// passive indices, no repeats) are rescaled so that they sum to the gas density; the sum runs in
// list order.  The element of each list entry is picked with unrolled selects, so the state stays
// in registers.
template <int NC, typename R>
GB_DEV void normalize_passive( R dens, R *u, int nnorm, const int *idx )
{
   R sum = R(0);
#  pragma unroll
   for (int k=0; k<NC-5; k++)
   {
      if ( k < nnorm )
      {
         R val = R(0);
#        pragma unroll
         for (int v=5; v<NC; v++) if ( idx[k] == v - 5 ) val = u[v];
         sum += val;
      }
   }
   const R norm = dens/sum;
#  pragma unroll
   for (int k=0; k<NC-5; k++)
   {
      if ( k < nnorm )
      {
#        pragma unroll
         for (int v=5; v<NC; v++) if ( idx[k] == v - 5 ) u[v] *= norm;
      }
   }
}

// dual-energy fix, DE_ENPY (Hydro_DualEnergyFix, CPU_Shared_DualEnergy.cpp:64-119, CheckMinPres off)
// P_MIXED selects the branch and forms the corrected energy in double.
template <int P, typename R>
GB_DEV void dual_energy_fix( const Phys<R> &ph, R d, R mx, R my, R mz, R &etot, R &dual, char &st )
{
   typedef typename std::conditional<P == P_MIXED, double, R>::type T;
   dual = gmax( dual, Lim<R>::tiny() );
   T eint;
   if constexpr ( P == P_MIXED )
      eint = (double)etot - 0.5*( (double)mx*mx + (double)my*my + (double)mz*mz )*rcp_dd( (double)d );
   else
      eint = eint_con<P>( d, R(1)/d, mx, my, mz, etot );
   const T enth = (T)etot - eint;
   const T gm1 = (T)ph.gm1;
   if ( eint/enth < (T)ph.de_switch )
   {
      const T pres = (T)dual*gpow( (T)d, gm1 );
      etot = (R)( enth + pres*(T)ph.inv_gm1 );
      st   = DE_BY_DUAL;
   }
   else
   {
      const T pres = eint*gm1;
      dual = gmax( (R)( pres*gpow( (T)d, -gm1 ) ), Lim<R>::tiny() );
      st   = DE_BY_ETOT;
   }
}

} // namespace gb

// float2 forms of the face-state and Riemann routines (riemann_hllc_pair, used by riemann<> above)
#include "hydro_pair.cuh"
