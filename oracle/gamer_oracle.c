/* Test infrastructure only — the oracle.  Never linked into the product.
 *
 * A plain-C, single-threaded restatement of GAMER's patch-group MHM fluid solver
 * (hydro, ideal gas, no MHD) used as the CPU checker of the CUDA path.  Each function cites the
 * reference routine it restates (paths relative to the GAMER source tree).  The arithmetic is
 * written in the same order as the reference so that, built with -ffp-contract=off, the results
 * agree bit for bit with the reference's own CPU_FluidSolver (checked by tests/test_oracle.py
 * against the reference compiled from source by oracle/build_ref.sh).
 *
 * Covered: MHM (src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_MHM.cpp:265-589)
 *          PLM (CPU_Shared_DataReconstruction.cpp:189-689) and PPM (:704-1395, non-ATHENA limiters)
 *          limiters vanLeer / GMinMod / vanAlbada / VL+GMinMod / central (:1918-2032), in primitive
 *                   or, with CHAR_RECONSTRUCTION (PLM), characteristic variables (:1400-1580)
 *          Hancock predictor with MHM_CHECK_PREDICT (:2064-2160)
 *          Riemann: HLLC (CPU_Shared_RiemannSolver_HLLC.cpp:392-655), HLLE (..._HLLE.cpp:302-700),
 *                   Roe with the HLLE intermediate-state check (..._Roe.cpp:88-719),
 *                   exact (..._Exact.cpp:62-432)
 *          HLLE rescue on NaN fluxes (CPU_Shared_ComputeFlux.cpp:313-362)
 *          coarse-fine flux planes (CPU_Shared_ComputeFlux.cpp:391-450)
 *          full-step update + dual energy DE_ENPY (CPU_Shared_FullStepUpdate.cpp:64-271,
 *                   CPU_Shared_DualEnergy.cpp:64-119)
 *          MinMod-coefficient retry loop (CPU_FluidSolver_MHM.cpp:496-584)
 *          MHM_RP half step (CPU_FluidSolver_MHM.cpp:593-950), PLM
 *          EoS: constant gamma (src/EoS/Gamma/CPU_EoS_Gamma.cpp)
 *
 * Build:  ORACLE_FP64 selects double ("FLOAT8"), otherwise float.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#ifdef ORACLE_FP64
typedef double real;
#  define SQRT(a) sqrt(a)
#  define FABS(a) fabs(a)
#  define FMAX(a,b) fmax(a,b)
#  define FMIN(a,b) fmin(a,b)
#  define POW(a,b) pow(a,b)
#  define TINY_NUMBER DBL_MIN
#  define HUGE_NUMBER DBL_MAX
#  define MACHINE_EPSILON DBL_EPSILON
#  define PPM_ROUND_ERR 1.e-12
#  define EXPORT(name) gor64_##name
#else
typedef float real;
#  define SQRT(a) sqrtf(a)
#  define FABS(a) fabsf(a)
#  define FMAX(a,b) fmaxf(a,b)
#  define FMIN(a,b) fminf(a,b)
#  define POW(a,b) powf(a,b)
#  define TINY_NUMBER FLT_MIN
#  define HUGE_NUMBER FLT_MAX
#  define MACHINE_EPSILON FLT_EPSILON
#  define PPM_ROUND_ERR 1.e-6
#  define EXPORT(name) gor32_##name
#endif

#define SQR(a)  ((a)*(a))
#define SIGN(a) ( ((a) < (real)0.0) ? (real)-1.0 : (real)+1.0 )
#define PS1 8
#define PS2 16
#define NCMAX 8            /* 5 fluid + up to 2 user passive scalars + optional dual-energy variable */

/* limiter ids follow include/Typedef.h:184-194 */
enum { LIM_VANLEER = 1, LIM_GMINMOD = 2, LIM_ALBADA = 3, LIM_VL_GMINMOD = 4, LIM_CENTRAL = 6 };
/* Riemann solver ids follow include/Macro.h (EXACT 1, ROE 2, HLLE 3, HLLC 4, HLLD 5) */
enum { RS_EXACT = 1, RS_ROE = 2, RS_HLLE = 3, RS_HLLC = 4 };
enum { LR_PLM = 1, LR_PPM = 2 };
#define DE_UPDATED_BY_ETOT     '0'
#define DE_UPDATED_BY_DUAL     '1'
#define DE_UPDATED_BY_MIN_PRES '2'

typedef struct {
   int  lr;             /* LR_PLM / LR_PPM */
   int  rsolver;        /* RS_HLLC / RS_HLLE / RS_ROE */
   int  dual;           /* 1 = DE_ENPY dual energy, NCOMP = 6 */
   int  char_rec;       /* 1 = CHAR_RECONSTRUCTION (PLM) */
   int  rp;             /* 1 = FLU_SCHEME MHM_RP (Riemann-predictor half step, PLM) */
   int  limiter;
   real minmod_coeff;
   int  minmod_maxiter;
   real dt, dh;
   real min_dens, min_pres, min_eint, de_switch;
   real gamma, gamma_m1, _gamma_m1;
} Cfg;

static int  g_nc;     /* number of variables: 5 + user passive scalars + dual-energy field */
static long g_floor;  /* PassiveFloor: bit v set for the floored passive scalars (the dual-energy
                         field, include/Macro.h:302-305: DUAL = NCOMP_TOTAL - 1) */
#define FLOORED(v) ( ( g_floor >> (v) ) & 1L )

/* ---------------------------------------------------------------------------------------------
 * EoS (src/EoS/Gamma/CPU_EoS_Gamma.cpp)
 * ------------------------------------------------------------------------------------------- */
static real eos_eint2pres( const Cfg *c, real eint )         { return eint*c->gamma_m1; }
static real eos_pres2eint( const Cfg *c, real pres )         { return pres*c->_gamma_m1; }
static real eos_pres2csqr( const Cfg *c, real dens, real p ) { return c->gamma*p/dens; }

/* CPU_Shared_FluUtility.cpp:1170 (Hydro_CheckMinPres) */
static real check_min( real in, real mn ) { return ( in == in ) ? FMAX( in, mn ) : in; }

/* CPU_Shared_FluUtility.cpp:1259 (Hydro_Con2Eint, no MHD) */
static real con2eint( real d, real mx, real my, real mz, real e )
{
   return e - (real)0.5*( SQR(mx) + SQR(my) + SQR(mz) ) / d;
}

/* CPU_Shared_FluUtility.cpp:1165 (Hydro_Con2Pres) */
static real con2pres( const Cfg *c, real d, real mx, real my, real mz, real e, int check, real minp )
{
   real p = eos_eint2pres( c, con2eint( d, mx, my, mz, e ) );
   if ( check ) p = check_min( p, minp );
   return p;
}

/* CPU_Shared_FluUtility.cpp:1299 (Hydro_ConEint2Etot) */
static real coneint2etot( real d, real mx, real my, real mz, real eint )
{
   real etot = (real)0.5*( SQR(mx) + SQR(my) + SQR(mz) ) / d;
   return etot + eint;
}

/* CPU_Shared_FluUtility.cpp:822 (Hydro_CheckMinEintInEngy) */
static real check_min_eint_in_engy( real d, real mx, real my, real mz, real e, real mineint )
{
   const real ein  = con2eint( d, mx, my, mz, e );
   const real eout = check_min( ein, mineint );
   return ( ein == eout ) ? e : e - ein + eout;
}

/* rotation x->(x,y,z) (CPU_Shared_FluUtility.cpp:93, Hydro_Rotate3D) */
static void rotate( real *a, int xyz, int fwd )
{
   real t0 = a[1], t1 = a[2], t2 = a[3];
   if ( xyz == 0 ) return;
   if ( (xyz == 1 && fwd) || (xyz == 2 && !fwd) ) { a[1] = t1; a[2] = t2; a[3] = t0; }
   else                                          { a[1] = t2; a[2] = t0; a[3] = t1; }
}

/* CPU_Shared_FluUtility.cpp:209 (Hydro_Con2Pri) */
static void con2pri( const Cfg *c, const real *in, real *out )
{
   const real _rho = (real)1.0/in[0];
   out[0] = in[0];
   out[1] = in[1]*_rho;
   out[2] = in[2]*_rho;
   out[3] = in[3]*_rho;
   out[4] = con2pres( c, in[0], in[1], in[2], in[3], in[4], 1, c->min_pres );
   for (int v=5; v<g_nc; v++) out[v] = in[v];
}

/* CPU_Shared_FluUtility.cpp:343 (Hydro_Pri2Con) */
static void pri2con( const Cfg *c, const real *in, real *out )
{
   for (int v=5; v<g_nc; v++) out[v] = in[v];
   out[0] = in[0];
   out[1] = in[0]*in[1];
   out[2] = in[0]*in[2];
   out[3] = in[0]*in[3];
   out[4] = coneint2etot( out[0], out[1], out[2], out[3], eos_pres2eint( c, in[4] ) );
}

/* CPU_Shared_FluUtility.cpp:458 (Hydro_Con2Flux); pres != NULL gives the pressure directly */
static void con2flux( const Cfg *c, int xyz, real *flux, const real *in, const real *pres )
{
   real r[5];
   for (int v=0; v<5; v++) r[v] = in[v];
   rotate( r, xyz, 1 );
   const real p   = ( pres == NULL ) ? con2pres( c, r[0], r[1], r[2], r[3], r[4], 1, c->min_pres ) : *pres;
   const real _rho = (real)1.0 / r[0];
   const real vx  = _rho*r[1];
   flux[0] = r[1];
   flux[1] = vx*r[1] + p;
   flux[2] = vx*r[2];
   flux[3] = vx*r[3];
   flux[4] = vx*( r[4] + p );
   for (int v=5; v<g_nc; v++) flux[v] = in[v]*vx;
   rotate( flux, xyz, 0 );
}

/* ---------------------------------------------------------------------------------------------
 * Riemann solvers
 * ------------------------------------------------------------------------------------------- */
/* CPU_Shared_RiemannSolver_HLLE.cpp:302-700 (HD, Davis wave speeds) */
static void riemann_hlle( const Cfg *c, int xyz, real *fo, const real *lin, const real *rin )
{
   real L[NCMAX], R[NCMAX], FL[NCMAX], FR[NCMAX];
   for (int v=0; v<g_nc; v++) { L[v] = lin[v]; R[v] = rin[v]; }
   rotate( L, xyz, 1 );  rotate( R, xyz, 1 );
   const real _rl = (real)1.0/L[0], _rr = (real)1.0/R[0];
   const real ul = _rl*L[1], ur = _rr*R[1];
   real pl = con2pres( c, L[0], L[1], L[2], L[3], L[4], 1, c->min_pres );
   real pr = con2pres( c, R[0], R[1], R[2], R[3], R[4], 1, c->min_pres );
   const real a2l = eos_pres2csqr( c, L[0], pl ), a2r = eos_pres2csqr( c, R[0], pr );
   const real cfl = SQRT( a2l ), cfr = SQRT( a2r );
   real maxvl = FMIN( ul-cfl, ur-cfr );
   real maxvr = FMAX( ul+cfl, ur+cfr );
   maxvl = FMIN( maxvl, (real)0.0 );
   maxvr = FMAX( maxvr, (real)0.0 );
   con2flux( c, 0, FL, L, &pl );
   con2flux( c, 0, FR, R, &pr );
   for (int v=0; v<5; v++) { FL[v] -= maxvl*L[v];  FR[v] -= maxvr*R[v]; }
   if ( maxvl == (real)0.0 && maxvr == (real)0.0 )
      for (int v=0; v<5; v++) fo[v] = FL[v];
   else
   {
      const real _d = (real)1.0 / ( maxvr - maxvl );
      for (int v=0; v<5; v++) fo[v] = _d*( maxvr*FL[v] - maxvl*FR[v] );
   }
   if ( g_nc > 5 )
   {
      if ( fo[0] >= (real)0.0 ) { const real vx = fo[0]*_rl; for (int v=5; v<g_nc; v++) fo[v] = L[v]*vx; }
      else                      { const real vx = fo[0]*_rr; for (int v=5; v<g_nc; v++) fo[v] = R[v]*vx; }
   }
   rotate( fo, xyz, 0 );
}

/* CPU_Shared_RiemannSolver_HLLC.cpp:392-655 (HD, Davis wave speeds) */
static void riemann_hllc( const Cfg *c, int xyz, real *fo, const real *lin, const real *rin )
{
   real L[NCMAX], R[NCMAX], F[NCMAX];
   for (int v=0; v<g_nc; v++) { L[v] = lin[v]; R[v] = rin[v]; }
   rotate( L, xyz, 1 );  rotate( R, xyz, 1 );
   const real _rl = (real)1.0 / L[0], _rr = (real)1.0 / R[0];
   const real ul = _rl*L[1], ur = _rr*R[1];
   real pl = con2pres( c, L[0], L[1], L[2], L[3], L[4], 1, c->min_pres );
   real pr = con2pres( c, R[0], R[1], R[2], R[3], R[4], 1, c->min_pres );
   const real csl = SQRT( eos_pres2csqr( c, L[0], pl ) );
   const real csr = SQRT( eos_pres2csqr( c, R[0], pr ) );
   const real wl1 = ul - csl, wl2 = ur - csr, wr1 = ul + csl, wr2 = ur + csr;
   const real wl = FMIN( wl1, wl2 ), wr = FMAX( wr1, wr2 );
   const real t1l = +L[0]*( ( wl1 < wl2 ) ? csl : (ul-ur)+csr );
   const real t1r = -R[0]*( ( wr2 > wr1 ) ? csr : (ul-ur)+csl );
   const real t2  = (real)1.0 / ( t1l - t1r );
   const real vs  = t2*( pl - pr + t1l*ul - t1r*ur );
   real ps = t2*( t1l*( pr + t1r*ur ) - t1r*( pl + t1l*ul ) );
   ps = check_min( ps, c->min_pres );
   real clr, cs;
   if ( vs >= (real)0.0 )
   {
      const real mvl = FMIN( wl, (real)0.0 );
      con2flux( c, 0, F, L, &pl );
      for (int v=0; v<5; v++) F[v] -= mvl*L[v];
      if ( vs == (real)0.0 && mvl == (real)0.0 ) { clr = (real)1.0; cs = (real)0.0; }
      else { const real t4 = (real)1.0 / ( vs - mvl ); clr = t4*vs; cs = -t4*mvl*ps; }
   }
   else
   {
      const real mvr = FMAX( wr, (real)0.0 );
      con2flux( c, 0, F, R, &pr );
      for (int v=0; v<5; v++) F[v] -= mvr*R[v];
      const real t4 = (real)1.0 / ( vs - mvr );
      clr = t4*vs;  cs = -t4*mvr*ps;
   }
   for (int v=0; v<5; v++) fo[v] = clr*F[v];
   fo[1] += cs;
   fo[4] += cs*vs;
   if ( g_nc > 5 )
   {
      if ( fo[0] >= (real)0.0 ) { const real vx = fo[0]*_rl; for (int v=5; v<g_nc; v++) fo[v] = L[v]*vx; }
      else                      { const real vx = fo[0]*_rr; for (int v=5; v<g_nc; v++) fo[v] = R[v]*vx; }
   }
   rotate( fo, xyz, 0 );
}

/* CPU_Shared_RiemannSolver_Roe.cpp:88-719 (HD; CHECK_INTERMEDIATE = HLLE, include/CUFLU.h:178-186) */
static void riemann_roe( const Cfg *c, int xyz, real *fo, const real *lin, const real *rin )
{
   real L[NCMAX], R[NCMAX], FL[NCMAX], FR[NCMAX];
   for (int v=0; v<g_nc; v++) { L[v] = lin[v]; R[v] = rin[v]; }
   rotate( L, xyz, 1 );  rotate( R, xyz, 1 );
   const real gamma = c->gamma, gm1 = c->gamma_m1;
   const real _rl = (real)1.0 / L[0], _rr = (real)1.0 / R[0];
   const real pl = con2pres( c, L[0], L[1], L[2], L[3], L[4], 1, c->min_pres );
   const real pr = con2pres( c, R[0], R[1], R[2], R[3], R[4], 1, c->min_pres );
   const real hl = _rl*( L[4] + pl ), hr = _rr*( R[4] + pr );
   const real sl = SQRT( L[0] ), sr = SQRT( R[0] );
   const real rho = sl*sr, _rho = (real)1.0/rho;
   const real _sl = (real)1.0/sl, _sr = (real)1.0/sr, _ss = (real)1.0/(sl + sr);
   const real u = _ss*( _sl*L[1] + _sr*R[1] );
   const real v = _ss*( _sl*L[2] + _sr*R[2] );
   const real w = _ss*( _sl*L[3] + _sr*R[3] );
   const real V2 = u*u + v*v + w*w;
   const real H  = _ss*( sl*hl + sr*hr );
   real gp = gm1*( H - (real)0.5*V2 );
   gp = gamma*_rho*check_min( gp*rho/gamma, c->min_pres );
   const real a2 = gp;
   const real a  = SQRT( a2 );
   const real ev[5] = { u-a, u, u, u, u+a };
   con2flux( c, 0, FL, L, &pl );
   con2flux( c, 0, FR, R, &pr );
   if ( ev[0] >= (real)0.0 ) { for (int k=0; k<g_nc; k++) fo[k] = FL[k]; rotate( fo, xyz, 0 ); return; }
   if ( ev[4] <= (real)0.0 ) { for (int k=0; k<g_nc; k++) fo[k] = FR[k]; rotate( fo, xyz, 0 ); return; }
   const real RE[5][5] = { { (real)1.0,  (real)1.0,        (real)0.0, (real)0.0, (real)1.0 },
                           { u-a,        u,                (real)0.0, (real)0.0, u+a       },
                           { v,          v,                (real)1.0, (real)0.0, v         },
                           { w,          w,                (real)0.0, (real)1.0, w         },
                           { H-u*a,      (real)0.5*V2,     v,         w,         H+u*a     } };
   real J[5], A[5];
   for (int k=0; k<5; k++) J[k] = R[k] - L[k];
   A[2] = J[2] - v*J[0];
   A[3] = J[3] - w*J[0];
   A[1] = gm1/a2*( J[0]*(H-SQR(u)) + u*J[1] - J[4] + v*A[2] + w*A[3] );
   A[0] = (real)0.5/a*( J[0]*(u+a) - J[1] - a*A[1] );
   A[4] = J[0] - A[0] - A[1];
   /* intermediate-state check (Roe.cpp, section 8) */
   real I[5];
   for (int k=0; k<5; k++) I[k] = L[k];
   for (int t=0; t<4; t++)
   {
      for (int k=0; k<5; k++) I[k] += A[t]*RE[k][t];
      if ( ev[t+1] > ev[t] )
      {
         const real ip = con2pres( c, I[0], I[1], I[2], I[3], I[4], 0, (real)0.0 );
         if ( I[0] <= (real)0.0 || ip <= (real)0.0 )
         {
            riemann_hlle( c, 0, fo, L, R );
            rotate( fo, xyz, 0 );
            return;
         }
      }
   }
   for (int k=0; k<5; k++) A[k] *= FABS( ev[k] );
   for (int k=0; k<5; k++)
   {
      fo[k] = FL[k] + FR[k];
      for (int t=0; t<5; t++) fo[k] -= A[t]*RE[k][t];
      fo[k] *= (real)0.5;
   }
   if ( g_nc > 5 )
   {
      if ( fo[0] >= (real)0.0 ) { const real vx = fo[0]*_rl; for (int k=5; k<g_nc; k++) fo[k] = L[k]*vx; }
      else                      { const real vx = fo[0]*_rr; for (int k=5; k<g_nc; k++) fo[k] = R[k]*vx; }
   }
   rotate( fo, xyz, 0 );
}

/* CPU_Shared_RiemannSolver_Exact.cpp:360-405 (Solve_f) */
static real exact_solve_f( real rho, real p, real p_star, real Gamma )
{
   const real Gamma_m1 = Gamma - (real)1.0;
   const real Gamma_p1 = Gamma + (real)1.0;
   real f;
   if ( p_star > p )
   {
      const real A = (real)2.0/( rho*Gamma_p1 );
      const real B = p*Gamma_m1/Gamma_p1;
      const real Temp = A/(p_star+B);
      f = (p_star-p)*SQRT( Temp );
   }
   else
   {
      const real a  = SQRT( Gamma*p/rho );
      const real cr = p_star/p;
      f = (real)2.0*a*(  POW( cr, (real)0.5*Gamma_m1/Gamma ) - (real)1.0  ) / Gamma_m1;
   }
   return f;
}

/* CPU_Shared_RiemannSolver_Exact.cpp:409-425 (Set_Flux, rotated primitive state) */
static void exact_set_flux( real *flux, const real *val, real Gamma )
{
   const real Gamma_m1 = Gamma - (real)1.0;
   flux[0] = val[0]*val[1];
   flux[1] = val[0]*val[1]*val[1] + val[4];
   flux[2] = val[0]*val[1]*val[2];
   flux[3] = val[0]*val[1]*val[3];
   flux[4] = val[1]*(  (real)0.5*val[0]*( val[1]*val[1] + val[2]*val[2] + val[3]*val[3] )
                      + val[4]/Gamma_m1 + val[4]  );
}

/* CPU_Shared_RiemannSolver_Exact.cpp:62-357 (Hydro_RiemannSolver_Exact, MAX_ERROR of
 * include/Macro.h:1023-1031): star pressure by bisection, then the sampled state */
static void riemann_exact( const Cfg *c, int xyz, real *fo, const real *lin, const real *rin )
{
#  ifdef ORACLE_FP64
   const real max_error = 1.0e-14;
#  else
   const real max_error = 1.0e-06f;
#  endif
   const real Gamma = c->gamma, Gamma_m1 = c->gamma_m1, Gamma_p1 = Gamma + (real)1.0;
   const real cc = Gamma_m1 / Gamma_p1;
   real eival[5], Ls[5], Rs[5], L[NCMAX], R[NCMAX];
   con2pri( c, lin, L );
   con2pri( c, rin, R );
   rotate( L, xyz, 1 );
   rotate( R, xyz, 1 );
   Ls[2] = L[2];  Ls[3] = L[3];  Rs[2] = R[2];  Rs[3] = R[3];
   {
      const real du = R[1] - L[1];
      real f = (real)0.0, f_L, f_R, bound[2], compare[2];
      bound[0] = FMIN( L[4], R[4] );
      bound[1] = FMAX( L[4], R[4] );
      for (int i=0; i<2; i++)
      {
         f_L = exact_solve_f( L[0], L[4], bound[i], Gamma );
         f_R = exact_solve_f( R[0], R[4], bound[i], Gamma );
         compare[i] = f_L + f_R + du;
      }
      if ( compare[0]*compare[1] > (real)0.0 )
      {
         if ( compare[0] > (real)0.0 ) { bound[1] = bound[0];  bound[0] = (real)0.0; }
         else if ( compare[1] < (real)0.0 )
         {
            int cont;
            bound[0] = bound[1];
            bound[1] = (real)2.0*bound[0];
            do
            {
               for (int i=0; i<2; i++)
               {
                  f_L = exact_solve_f( L[0], L[4], bound[i], Gamma );
                  f_R = exact_solve_f( R[0], R[4], bound[i], Gamma );
                  compare[i] = f_L + f_R + du;
               }
               cont = ( compare[0]*compare[1] > (real)0.0 );
               if ( cont ) { bound[0] = bound[1];  bound[1] = bound[0]*(real)2.0; }
            }
            while ( cont );
         }
      }
      do
      {
         Ls[4] = (real)0.5*( bound[0] + bound[1] );
         if ( Ls[4] == bound[0] || Ls[4] == bound[1] ) break;
         f_L = exact_solve_f( L[0], L[4], Ls[4], Gamma );
         f_R = exact_solve_f( R[0], R[4], Ls[4], Gamma );
         f   = f_L + f_R + du;
         if ( f > (real)0.0 ) bound[1] = Ls[4];
         else                 bound[0] = Ls[4];
      }
      while ( FABS(f) >= max_error );
   }
   Rs[4] = Ls[4];
   {
      const real f_L = exact_solve_f( L[0], L[4], Ls[4], Gamma );
      const real f_R = exact_solve_f( R[0], R[4], Rs[4], Gamma );
      Ls[1] = (real)0.5*( L[1] + R[1] ) + (real)0.5*( f_R - f_L );
   }
   Rs[1] = Ls[1];
   if ( Ls[4] > L[4] ) { const real r = Ls[4] / L[4];  Ls[0] = L[0]*(  ( r + cc ) / ( cc*r + (real)1.0 )  ); }
   else
   {
      Ls[0] = L[0]*POW( Ls[4]/L[4], (real)1.0/Gamma );
      const real a_L = SQRT( Gamma * L[4] / L[0] ), a_s = SQRT( Gamma * Ls[4] / Ls[0] );
      if ( L[1] < a_L  &&  Ls[1] > a_s )
      {
         Ls[0] = L[0]*POW(  (real)2.0/Gamma_p1 + cc*L[1]/a_L, (real)2.0/Gamma_m1  );
         Ls[1] = (real)2.0*( a_L + (real)0.5*Gamma_m1*L[1] ) / Gamma_p1;
         Ls[4] = L[4]*POW(  (real)2.0/Gamma_p1 + cc*L[1]/a_L, (real)2.0*Gamma/Gamma_m1  );
      }
   }
   if ( Rs[4] > R[4] ) { const real r = Rs[4] / R[4];  Rs[0] = R[0]*(  ( r + cc ) / ( cc * r + (real)1.0 )  ); }
   else
   {
      Rs[0] = R[0]*POW( Rs[4]/R[4], (real)1.0/Gamma );
      const real a_R = SQRT( Gamma * R[4] / R[0] ), a_s = SQRT( Gamma * Rs[4] / Rs[0] );
      if ( R[1] > -a_R  &&  Rs[1] < -a_s )
      {
         Rs[0] = R[0]*POW (  (real)2.0/Gamma_p1 - cc*R[1]/a_R, (real)2.0/Gamma_m1  );
         Rs[1] = (real)2.0*( -a_R + (real)0.5*Gamma_m1*R[1] ) / Gamma_p1;
         Rs[4] = R[4]*POW (  (real)2.0/Gamma_p1 - cc*R[1]/a_R, (real)2.0*Gamma/Gamma_m1 );
      }
   }
   eival[1] = Ls[1];  eival[2] = Ls[1];  eival[3] = Ls[1];
   if ( L[4] < Ls[4] )
   {
      const real Temp = (real)0.5/Gamma*( Gamma_p1*Ls[4]/L[4] + Gamma_m1 );
      eival[0] = L[1] - SQRT( Gamma*L[4]/L[0] )*SQRT( Temp );
   }
   else eival[0] = L[1] - SQRT ( Gamma*L[4]/L[0] );
   if ( R[4] < Rs[4] )
   {
      const real Temp = (real)0.5/Gamma*( Gamma_p1*Rs[4]/R[4] + Gamma_m1 );
      eival[4] = R[1] + SQRT( Gamma*R[4]/R[0] )*SQRT( Temp );
   }
   else eival[4] = R[1] + SQRT ( Gamma*R[4]/R[0] );
   if ( FABS( eival[1] ) < max_error )
   {
      fo[0] = (real)0.0;  fo[1] = Ls[4];  fo[2] = (real)0.0;  fo[3] = (real)0.0;  fo[4] = (real)0.0;
   }
   else if ( eival[1] > (real)0.0 ) exact_set_flux( fo, ( eival[0] > (real)0.0 ) ? L : Ls, Gamma );
   else                             exact_set_flux( fo, ( eival[4] < (real)0.0 ) ? R : Rs, Gamma );
   if ( g_nc > 5 )
   {
      if ( fo[0] >= (real)0.0 ) { const real vx = fo[0] / lin[0]; for (int v=5; v<g_nc; v++) fo[v] = lin[v]*vx; }
      else                      { const real vx = fo[0] / rin[0]; for (int v=5; v<g_nc; v++) fo[v] = rin[v]*vx; }
   }
   rotate( fo, xyz, 0 );
}

static void riemann( const Cfg *c, int xyz, real *fo, const real *l, const real *r )
{
   if      ( c->rsolver == RS_HLLC  ) riemann_hllc ( c, xyz, fo, l, r );
   else if ( c->rsolver == RS_ROE   ) riemann_roe  ( c, xyz, fo, l, r );
   else if ( c->rsolver == RS_EXACT ) riemann_exact( c, xyz, fo, l, r );
   else                               riemann_hlle ( c, xyz, fo, l, r );
   /* rescue with HLLE on NaN (CPU_Shared_ComputeFlux.cpp:313-362; none when RSOLVER is ROE or HLLE) */
   if ( c->rsolver == RS_HLLC || c->rsolver == RS_EXACT )
      for (int v=0; v<g_nc; v++)
         if ( fo[v] != fo[v] ) { riemann_hlle( c, xyz, fo, l, r ); break; }
}

/* ---------------------------------------------------------------------------------------------
 * Characteristic variables of the gamma-law hydro system, CHAR_RECONSTRUCTION
 * (CPU_Shared_DataReconstruction.cpp:1400-1580, Hydro_Pri2Char / Hydro_Char2Pri, no MHD): the
 * primitive slope is rotated along xyz and projected on the left eigenvectors of the cell's own
 * (rho, P); passive scalars are left as they are
 * ------------------------------------------------------------------------------------------- */
static void pri2char( const Cfg *c, real *io, real dens, real pres, int xyz )
{
   real t[5];
   for (int v=0; v<5; v++) t[v] = io[v];
   rotate( t, xyz, 1 );
   const real a2  = eos_pres2csqr( c, dens, pres );
   const real _a2 = (real)1.0 / a2;
   const real _a  = SQRT( _a2 );
   io[0] = -(real)0.5*dens*_a*t[1] + (real)0.5*_a2*t[4];
   io[1] = t[0] - _a2*t[4];
   io[2] = t[2];
   io[3] = t[3];
   io[4] = +(real)0.5*dens*_a*t[1] + (real)0.5*_a2*t[4];
}

static void char2pri( const Cfg *c, real *io, real dens, real pres, int xyz )
{
   real t[5];
   for (int v=0; v<5; v++) t[v] = io[v];
   const real a2 = eos_pres2csqr( c, dens, pres );
   const real a  = SQRT( a2 );
   io[0] = t[0] + t[1] + t[4];
   io[1] = a/dens*( -t[0] + t[4] );
   io[2] = t[2];
   io[3] = t[3];
   io[4] = a2*( t[0] + t[4] );
   rotate( io, xyz, 0 );
}

/* ---------------------------------------------------------------------------------------------
 * Slope limiter (CPU_Shared_DataReconstruction.cpp:1918-2032); with c->char_rec the slopes are
 * limited in characteristic variables of direction xyz
 * ------------------------------------------------------------------------------------------- */
static void limit_slope_c( const Cfg *c, const real *L, const real *C, const real *R, int lim, real coeff,
                           int xyz, real *out );

static void limit_slope( const real *L, const real *C, const real *R, int lim, real coeff, real *out )
{
   limit_slope_c( NULL, L, C, R, lim, coeff, 0, out );
}

static void limit_slope_c( const Cfg *c, const real *L, const real *C, const real *R, int lim, real coeff,
                           int xyz, real *out )
{
   real sl[NCMAX], sr[NCMAX], sc[NCMAX], sa[NCMAX];
   for (int v=0; v<g_nc; v++)
   {
      sl[v] = C[v] - L[v];
      sr[v] = R[v] - C[v];
      sc[v] = (real)0.5*( sl[v] + sr[v] );
   }
   if ( lim == LIM_VL_GMINMOD )
      for (int v=0; v<g_nc; v++)
         sa[v] = ( sl[v]*sr[v] > (real)0.0 ) ? (real)2.0*sl[v]*sr[v]/( sl[v] + sr[v] ) : (real)0.0;
   const int ch = ( c != NULL && c->char_rec );
   if ( ch )
   {
      pri2char( c, sl, C[0], C[4], xyz );
      pri2char( c, sr, C[0], C[4], xyz );
      pri2char( c, sc, C[0], C[4], xyz );
      if ( lim == LIM_VL_GMINMOD ) pri2char( c, sa, C[0], C[4], xyz );
   }
   for (int v=0; v<g_nc; v++)
   {
      const real slr = sl[v]*sr[v];
      if ( slr > (real)0.0 )
      {
         switch ( lim )
         {
            case LIM_CENTRAL:  out[v] = sc[v];  break;
            case LIM_VANLEER:  out[v] = (real)2.0*slr/( sl[v] + sr[v] );  break;
            case LIM_GMINMOD:
               sl[v] *= coeff;  sr[v] *= coeff;
               out[v]  = FMIN( FABS( sl[v] ), FABS( sr[v] ) );
               out[v]  = FMIN( FABS( sc[v] ), out[v] );
               out[v] *= SIGN( sc[v] );
               break;
            case LIM_ALBADA:
               out[v] = slr*( sl[v] + sr[v] ) / ( sl[v]*sl[v] + sr[v]*sr[v] );
               break;
            case LIM_VL_GMINMOD:
               sl[v] *= coeff;  sr[v] *= coeff;
               out[v]  = FMIN( FABS( sl[v] ), FABS( sr[v] ) );
               out[v]  = FMIN( FABS( sc[v] ), out[v] );
               out[v]  = FMIN( FABS( sa[v] ), out[v] );
               out[v] *= SIGN( sc[v] );
               break;
            default: out[v] = (real)0.0;
         }
      }
      else out[v] = (real)0.0;
   }
   if ( ch ) char2pri( c, out, C[0], C[4], xyz );
}

/* ---------------------------------------------------------------------------------------------
 * Per-patch-group solver
 * ------------------------------------------------------------------------------------------- */
typedef struct {
   int  nxt, ghost, lr_ghost, nfc;     /* FLU_NXT, FLU_GHOST_SIZE, LR_GHOST_SIZE, N_FC_VAR */
   real *pri;                          /* [NC][nxt^3]          */
   real *slope;                        /* [3][NC][(nfc+2)^3]   (PPM) */
   real *fc;                           /* [6][NC][nfc^3]       */
   real *flux;                         /* [3][NC][nflx^3], nflx = PS2+1 */
} Work;

#define IDX3(i,j,k,ni,nj) ( ((k)*(nj) + (j))*(ni) + (i) )

/* CPU_Shared_DataReconstruction.cpp:2064-2160 (Hydro_HancockPredict, MHM_CHECK_PREDICT on) */
static void hancock( const Cfg *c, real fcon[6][NCMAX], const real fpri[6][NCMAX],
                     const real *cc_in, int n3, int cc_idx )
{
   const real dt_dh2 = (real)0.5*c->dt/c->dh;
   real F[6][NCMAX];
   for (int f=0; f<6; f++) con2flux( c, f/2, F[f], fcon[f], NULL );
   for (int v=0; v<g_nc; v++)
   {
      const real df = dt_dh2*( F[1][v] - F[0][v] + F[3][v] - F[2][v] + F[5][v] - F[4][v] );
      for (int f=0; f<6; f++) fcon[f][v] -= df;
   }
   int reset = 0;
   for (int f=0; f<6; f++)
   {
      if ( fcon[f][0] < TINY_NUMBER || fcon[f][0] > HUGE_NUMBER || fcon[f][0] != fcon[f][0] ) reset = 1;
      if ( fcon[f][4] < TINY_NUMBER || fcon[f][4] > HUGE_NUMBER || fcon[f][4] != fcon[f][4] ) reset = 1;
      if ( fpri[f][4] < (real)0.0   || fpri[f][4] > HUGE_NUMBER || fpri[f][4] != fpri[f][4] ) reset = 1;
      if ( reset )
      {
         for (int ff=0; ff<6; ff++)
         for (int v=0; v<g_nc; v++) fcon[ff][v] = cc_in[ v*n3 + cc_idx ];
         break;
      }
      fcon[f][0] = FMAX( fcon[f][0], c->min_dens );
      fcon[f][4] = check_min_eint_in_engy( fcon[f][0], fcon[f][1], fcon[f][2], fcon[f][3], fcon[f][4], c->min_eint );
      for (int v=5; v<g_nc; v++) if ( FLOORED(v) ) fcon[f][v] = FMAX( fcon[f][v], TINY_NUMBER );
   }
}

/* PLM: CPU_Shared_DataReconstruction.cpp:189-689; PPM: :704-1395 */
static void reconstruct( const Cfg *c, const real *cc_in, Work *w, real coeff )
{
   /* MHM_RP reconstructs from the half-step primitive variables, N_HF_VAR = FLU_NXT - 2 per side,
      already in w->pri (CPU_Shared_DataReconstruction.cpp:205-209, Con2Pri_No) */
   const int N = c->rp ? w->nxt - 2 : w->nxt, NG = w->lr_ghost, NF = w->nfc, NS = NF + 2;
   const int N3 = N*N*N, NF3 = NF*NF*NF, NS3 = NS*NS*NS;
   const int dcc[3] = { 1, N, N*N }, dsl[3] = { 1, NS, NS*NS };

   /* 0. conserved -> primitive */
   for (int idx=0; idx<N3 && !c->rp; idx++)
   {
      real con[NCMAX], pri[NCMAX];
      for (int v=0; v<g_nc; v++) con[v] = cc_in[v*N3 + idx];
      con2pri( c, con, pri );
      for (int v=0; v<g_nc; v++) w->pri[v*N3 + idx] = pri[v];
   }

   /* 1. PPM slopes */
   if ( c->lr == LR_PPM )
   {
      for (int idx=0; idx<NS3; idx++)
      {
         const int i = NG - 1 + idx%NS, j = NG - 1 + (idx%(NS*NS))/NS, k = NG - 1 + idx/(NS*NS);
         const int icc = IDX3( i, j, k, N, N );
         real C[NCMAX], L[NCMAX], R[NCMAX], S[NCMAX];
         for (int v=0; v<g_nc; v++) C[v] = w->pri[v*N3 + icc];
         for (int d=0; d<3; d++)
         {
            for (int v=0; v<g_nc; v++) { L[v] = w->pri[v*N3 + icc - dcc[d]];  R[v] = w->pri[v*N3 + icc + dcc[d]]; }
            limit_slope( L, C, R, c->limiter, coeff, S );
            for (int v=0; v<g_nc; v++) w->slope[ (d*g_nc + v)*NS3 + idx ] = S[v];
         }
      }
   }

   /* 2. face values + Hancock */
   for (int idx_fc=0; idx_fc<NF3; idx_fc++)
   {
      const int ifc = idx_fc%NF, jfc = (idx_fc%(NF*NF))/NF, kfc = idx_fc/(NF*NF);
      const int icc = IDX3( ifc+NG, jfc+NG, kfc+NG, N, N );
      const int isl = IDX3( ifc+1, jfc+1, kfc+1, NS, NS );
      real C[NCMAX], L[NCMAX], R[NCMAX], S[NCMAX];
      real fpri[6][NCMAX], fcon[6][NCMAX];
      for (int v=0; v<g_nc; v++) C[v] = w->pri[v*N3 + icc];
      for (int d=0; d<3; d++)
      {
         const int fL = 2*d, fR = fL + 1;
         for (int v=0; v<g_nc; v++) { L[v] = w->pri[v*N3 + icc - dcc[d]];  R[v] = w->pri[v*N3 + icc + dcc[d]]; }
         if ( c->lr == LR_PLM )
         {
            limit_slope_c( c, L, C, R, c->limiter, coeff, d, S );
            for (int v=0; v<g_nc; v++)
            {
               fpri[fL][v] = C[v] - (real)0.5*S[v];
               fpri[fR][v] = C[v] + (real)0.5*S[v];
            }
            for (int v=0; v<g_nc; v++)
            {
               real mn, mx;
               mn = ( C[v] < L[v] ) ? C[v] : L[v];
               mx = ( C[v] > L[v] ) ? C[v] : L[v];
               fpri[fL][v] = ( fpri[fL][v] > mn ) ? fpri[fL][v] : mn;
               fpri[fL][v] = ( fpri[fL][v] < mx ) ? fpri[fL][v] : mx;
               fpri[fR][v] = (real)2.0*C[v] - fpri[fL][v];
               mn = ( C[v] < R[v] ) ? C[v] : R[v];
               mx = ( C[v] > R[v] ) ? C[v] : R[v];
               fpri[fR][v] = ( fpri[fR][v] > mn ) ? fpri[fR][v] : mn;
               fpri[fR][v] = ( fpri[fR][v] < mx ) ? fpri[fR][v] : mx;
               fpri[fL][v] = (real)2.0*C[v] - fpri[fR][v];
            }
         }
         else   /* PPM, non-ATHENA limiters */
         {
            for (int v=0; v<g_nc; v++)
            {
               const real dl = w->slope[ (d*g_nc + v)*NS3 + isl - dsl[d] ];
               const real dr = w->slope[ (d*g_nc + v)*NS3 + isl + dsl[d] ];
               const real dc = w->slope[ (d*g_nc + v)*NS3 + isl          ];
               real fl = (real)0.5*( C[v] + L[v] ) - (real)1.0/(real)6.0*( dc - dl );
               real fr = (real)0.5*( C[v] + R[v] ) - (real)1.0/(real)6.0*( dr - dc );
               if ( c->limiter == LIM_CENTRAL )
               {
                  if ( (C[v]-fl)*(fl-L[v]) < (real)0.0 ) fl = (real)0.5*( C[v] + L[v] );
                  if ( (R[v]-fr)*(fr-C[v]) < (real)0.0 ) fr = (real)0.5*( C[v] + R[v] );
               }
               const real dfc  = fr - fl;
               const real dfc6 = (real)6.0*( C[v] - (real)0.5*( fl + fr ) );
               if ( ( fr - C[v] )*( C[v] - fl ) <= (real)0.0 ) { fl = C[v]; fr = C[v]; }
               else if ( dfc*dfc6 > +dfc*dfc ) fl = (real)3.0*C[v] - (real)2.0*fr;
               else if ( dfc*dfc6 < -dfc*dfc ) fr = (real)3.0*C[v] - (real)2.0*fl;
               real mn, mx;
               mn = ( C[v] < L[v] ) ? C[v] : L[v];
               mx = ( C[v] > L[v] ) ? C[v] : L[v];
               fl = ( fl > mn ) ? fl : mn;
               fl = ( fl < mx ) ? fl : mx;
               mn = ( C[v] < R[v] ) ? C[v] : R[v];
               mx = ( C[v] > R[v] ) ? C[v] : R[v];
               fr = ( fr > mn ) ? fr : mn;
               fr = ( fr < mx ) ? fr : mx;
               fpri[fL][v] = fl;
               fpri[fR][v] = fr;
            }
         }
         pri2con( c, fpri[fL], fcon[fL] );
         pri2con( c, fpri[fR], fcon[fR] );
      }
      if ( !c->rp ) hancock( c, fcon, fpri, cc_in, N3, icc );
      for (int f=0; f<6; f++)
      for (int v=0; v<g_nc; v++) w->fc[ (f*g_nc + v)*NF3 + idx_fc ] = fcon[f][v];
   }
}

/* CPU_Shared_ComputeFlux.cpp:113-376 (NSkip_N = 0, NSkip_T = 1 for hydro MHM) */
static void compute_flux( const Cfg *c, Work *w )
{
   const int NF = w->nfc, NF3 = NF*NF*NF, NX = PS2 + 1, NX3 = NX*NX*NX;
   const int dfc[3] = { 1, NF, NF*NF };
   for (int d=0; d<3; d++)
   {
      int s[3] = { 1, 1, 1 }, e[3] = { NF-2, NF-2, NF-2 };
      s[d] = 0;  e[d] = NF - 1;
      for (int k=0; k<e[2]; k++)
      for (int j=0; j<e[1]; j++)
      for (int i=0; i<e[0]; i++)
      {
         const int ifx = IDX3( i, j, k, NX, NX );
         const int ifc = IDX3( i+s[0], j+s[1], k+s[2], NF, NF );
         real L[NCMAX], R[NCMAX], F[NCMAX];
         for (int v=0; v<g_nc; v++)
         {
            L[v] = w->fc[ ((2*d+1)*g_nc + v)*NF3 + ifc          ];
            R[v] = w->fc[ ((2*d  )*g_nc + v)*NF3 + ifc + dfc[d] ];
         }
         riemann( c, d, F, L, R );
         for (int v=0; v<g_nc; v++) w->flux[ (d*g_nc + v)*NX3 + ifx ] = F[v];
      }
   }
}

/* CPU_Shared_ComputeFlux.cpp:391-450 (Hydro_StoreIntFlux) */
static void store_int_flux( const Work *w, real *out )
{
   const int NX = PS2 + 1, NX3 = NX*NX*NX;
   for (int idx=0; idx<PS2*PS2; idx++)
   {
      const int a = idx%PS2, b = idx/PS2;
      const int src[9][2] = { {0, IDX3(0,a,b,NX,NX)}, {0, IDX3(PS1,a,b,NX,NX)}, {0, IDX3(PS2,a,b,NX,NX)},
                              {1, IDX3(a,0,b,NX,NX)}, {1, IDX3(a,PS1,b,NX,NX)}, {1, IDX3(a,PS2,b,NX,NX)},
                              {2, IDX3(a,b,0,NX,NX)}, {2, IDX3(a,b,PS1,NX,NX)}, {2, IDX3(a,b,PS2,NX,NX)} };
      for (int p=0; p<9; p++)
      for (int v=0; v<g_nc; v++)
         out[ (p*g_nc + v)*PS2*PS2 + idx ] = w->flux[ (src[p][0]*g_nc + v)*NX3 + src[p][1] ];
   }
}

/* CPU_Shared_DualEnergy.cpp:64-119 (Hydro_DualEnergyFix, DE_ENPY, CheckMinPres off) */
static void dual_energy_fix( const Cfg *c, real d, real mx, real my, real mz, real *etot, real *dual, char *st )
{
   *dual = FMAX( *dual, TINY_NUMBER );
   real eint = con2eint( d, mx, my, mz, *etot );
   const real enth = *etot - eint;
   real pres;
   if ( eint/enth < c->de_switch )
   {
      pres  = *dual*POW( d, c->gamma_m1 );
      eint  = pres*c->_gamma_m1;
      *etot = enth + eint;
      *st   = DE_UPDATED_BY_DUAL;
   }
   else
   {
      pres  = eint*c->gamma_m1;
      *dual = FMAX( pres*POW( d, -c->gamma_m1 ), TINY_NUMBER );
      *st   = DE_UPDATED_BY_ETOT;
   }
}

/* CPU_Shared_FluUtility.cpp:843 (Hydro_IsUnphysical, UNPHY_MODE_CONS, EOS_GAMMA, no MHD) */
static int is_unphysical( const real *u )
{
   int bad = 0;
   for (int v=0; v<g_nc; v++)
   {
      if ( u[v] != u[v] ) bad = 1;
      if ( v >= 1 && v <= 3 ) { if ( u[v] < -HUGE_NUMBER || u[v] > HUGE_NUMBER ) bad = 1; }
      else if ( v < 5 )       { if ( u[v] <= (real)0.0 || u[v] > HUGE_NUMBER ) bad = 1; }
      else                    { if ( u[v] < (real)0.0 && FLOORED(v) ) bad = 1;
                                if ( u[v] < -HUGE_NUMBER || u[v] > HUGE_NUMBER ) bad = 1; }
   }
   const real eint = con2eint( u[0], u[1], u[2], u[3], u[4] );
   if ( eint < (real)-3.0*u[4]*MACHINE_EPSILON || eint > HUGE_NUMBER || eint != eint ) bad = 1;
   return bad;
}

/* CPU_Shared_FullStepUpdate.cpp:64-271; returns 1 if any output cell is unphysical */
static int full_step_update( const Cfg *c, const real *in, const Work *w, real *out, char *de )
{
   const int N = w->nxt, N3 = N*N*N, G = w->ghost, NX = PS2 + 1, NX3 = NX*NX*NX;
   const int dfx[3] = { 1, NX, NX*NX };
   const real dt_dh = c->dt/c->dh;
   int fail = 0;
   for (int idx=0; idx<PS2*PS2*PS2; idx++)
   {
      const int i = idx%PS2, j = (idx%(PS2*PS2))/PS2, k = idx/(PS2*PS2);
      const int ifx = IDX3( i, j, k, NX, NX );
      const int iin = IDX3( i+G, j+G, k+G, N, N );
      real df[3][NCMAX], u[NCMAX];
      for (int d=0; d<3; d++)
      for (int v=0; v<g_nc; v++)
         df[d][v] = w->flux[ (d*g_nc + v)*NX3 + ifx + dfx[d] ] - w->flux[ (d*g_nc + v)*NX3 + ifx ];
      for (int v=0; v<g_nc; v++) u[v] = in[v*N3 + iin] - dt_dh*( df[0][v] + df[1][v] + df[2][v] );
      for (int v=5; v<g_nc; v++) if ( FLOORED(v) ) u[v] = FMAX( u[v], TINY_NUMBER );
      if ( c->dual )
      {
         const int DI = g_nc - 1;
         const real ekin = (real)0.5*( SQR(u[1]) + SQR(u[2]) + SQR(u[3]) )/u[0];
         if ( u[0] > (real)0.0 && u[4]*(real)2.0 > ekin )
            dual_energy_fix( c, u[0], u[1], u[2], u[3], &u[4], &u[DI], &de[idx] );
      }
      for (int v=0; v<g_nc; v++) out[v*PS2*PS2*PS2 + idx] = u[v];
      if ( is_unphysical( u ) ) fail = 1;
   }
   return fail;
}

/* MHM_RP half step (CPU_FluidSolver_MHM.cpp:593-800 Hydro_RiemannPredict_Flux, :807-950
 * Hydro_RiemannPredict, hydro): first-order Riemann fluxes between the input cells, then the input
 * advanced by dt/2 with them on the inner (FLU_NXT-2)^3 cells, floored, and converted to the
 * primitive variables the reconstruction starts from (w->pri, stride FLU_NXT-2).
 * hf: scratch of 3*NCMAX*(FLU_NXT-1)^3 reals. */
static void riemann_predict( const Cfg *c, const real *cc, Work *w, real *hf )
{
   const int N = w->nxt, N3 = N*N*N, NH = N - 1, NH3 = NH*NH*NH, NV = N - 2, NV3 = NV*NV*NV;
   const int dcc[3] = { 1, N, N*N }, dhf[3] = { 1, NH, NH*NH };
   for (int d=0; d<3; d++)
   {
      const int is = ( d == 0 ) ? 0 : 1, js = ( d == 1 ) ? 0 : 1, ks = ( d == 2 ) ? 0 : 1;
      const int ni = ( d == 0 ) ? NH : NH - 1, nj = ( d == 1 ) ? NH : NH - 1, nk = ( d == 2 ) ? NH : NH - 1;
      for (int k=0; k<nk; k++)
      for (int j=0; j<nj; j++)
      for (int i=0; i<ni; i++)
      {
         const int ihf = IDX3( i, j, k, NH, NH );
         const int icc = IDX3( i+is, j+js, k+ks, N, N );
         real L[NCMAX], R[NCMAX], F[NCMAX];
         for (int v=0; v<g_nc; v++) { L[v] = cc[ v*N3 + icc ];  R[v] = cc[ v*N3 + icc + dcc[d] ]; }
         riemann( c, d, F, L, R );
         for (int v=0; v<g_nc; v++) hf[ (d*g_nc + v)*NH3 + ihf ] = F[v];
      }
   }
   const real dt_dh2 = (real)0.5*c->dt/c->dh;
   for (int k=0; k<NV; k++)
   for (int j=0; j<NV; j++)
   for (int i=0; i<NV; i++)
   {
      const int ihf = IDX3( i, j, k, NH, NH ), icc = IDX3( i+1, j+1, k+1, N, N );
      real dflux[3][NCMAX], con[NCMAX], pri[NCMAX];
      for (int d=0; d<3; d++)
      for (int v=0; v<g_nc; v++)
         dflux[d][v] = hf[ (d*g_nc + v)*NH3 + ihf + dhf[d] ] - hf[ (d*g_nc + v)*NH3 + ihf ];
      for (int v=0; v<g_nc; v++)
         con[v] = cc[ v*N3 + icc ] - dt_dh2*( dflux[0][v] + dflux[1][v] + dflux[2][v] );
      con[0] = FMAX( con[0], c->min_dens );
      con[4] = check_min_eint_in_engy( con[0], con[1], con[2], con[3], con[4], c->min_eint );
      for (int v=5; v<g_nc; v++) if ( FLOORED(v) ) con[v] = FMAX( con[v], TINY_NUMBER );
      con2pri( c, con, pri );
      for (int v=0; v<g_nc; v++) w->pri[ v*NV3 + IDX3( i, j, k, NV, NV ) ] = pri[v];
   }
}

/* Solve npg patch groups.  Shapes: in[npg][nc][nxt^3], out[npg][nc][16^3], flux[npg][9][nc][16^2],
 * de[npg][16^3].  lr: 1 PLM / 2 PPM; rsolver: 1 EXACT / 2 ROE / 3 HLLE / 4 HLLC.  nxt may exceed the scheme's
 * minimum (20 for PLM, 22 for PPM): the extra outer layers are ignored, as with a larger
 * FLU_GHOST_SIZE.  char_rec: CHAR_RECONSTRUCTION (PLM only). */
static int solve_impl( const real *in, real *out, real *flux, char *de, int npg, int nxt,
                       int lr, int rsolver, int dual, int limiter, double minmod_coeff, int minmod_maxiter,
                       double dt, double dh, double min_dens, double min_pres, double min_eint,
                       double de_switch, double gamma, int char_rec, int rp, int npass )
{
   Cfg c;
   c.lr = lr;  c.rsolver = rsolver;  c.dual = dual;  c.limiter = limiter;  c.char_rec = char_rec;  c.rp = rp;
   if ( rp && lr != LR_PLM ) return -1;
   c.minmod_coeff = (real)minmod_coeff;  c.minmod_maxiter = minmod_maxiter;
   c.dt = (real)dt;  c.dh = (real)dh;
   c.min_dens = (real)min_dens;  c.min_pres = (real)min_pres;  c.min_eint = (real)min_eint;
   c.de_switch = (real)de_switch;
   /* EoS_SetAuxArray_Gamma: the constants are formed in double and then cast to real */
   c.gamma = (real)gamma;  c.gamma_m1 = (real)(gamma - 1.0);  c._gamma_m1 = (real)(1.0/(gamma - 1.0));
   g_nc = 5 + npass + ( dual ? 1 : 0 );
   g_floor = dual ? ( 1L << ( g_nc - 1 ) ) : 0L;
   if ( npass < 0 || g_nc > NCMAX ) return -1;

   const int need = ( lr == LR_PPM || rp ) ? 22 : 20;
   if ( nxt < need || ( (nxt - need) & 1 ) ) return -1;
   const int shift = ( nxt - need )/2;     /* outer layers not read by the scheme */
   const int N = need, N3 = N*N*N, NF = PS2 + 2, NS = NF + 2, NX = PS2 + 1;
   Work w;
   w.nxt = N;  w.ghost = N/2 - PS2/2;  w.lr_ghost = ( lr == LR_PPM ) ? 2 : 1;  w.nfc = NF;
   w.pri   = (real*)malloc( sizeof(real)*NCMAX*N3 );
   w.slope = (real*)malloc( sizeof(real)*3*NCMAX*NS*NS*NS );
   w.fc    = (real*)malloc( sizeof(real)*6*NCMAX*NF*NF*NF );
   w.flux  = (real*)malloc( sizeof(real)*3*NCMAX*NX*NX*NX );
   real *cc = (real*)malloc( sizeof(real)*NCMAX*N3 );
   real *hf = rp ? (real*)malloc( sizeof(real)*3*NCMAX*(N-1)*(N-1)*(N-1) ) : NULL;
   const int NIN = nxt, NIN3 = NIN*NIN*NIN;

   for (int p=0; p<npg; p++)
   {
      /* cut the central N^3 window when nxt exceeds the scheme's size */
      for (int v=0; v<g_nc; v++)
      for (int k=0; k<N; k++)
      for (int j=0; j<N; j++)
      for (int i=0; i<N; i++)
         cc[ v*N3 + IDX3(i,j,k,N,N) ] = in[ ((size_t)p*g_nc + v)*NIN3 + IDX3(i+shift,j+shift,k+shift,NIN,NIN) ];

      if ( rp ) riemann_predict( &c, cc, &w, hf );
      int iter = 0, fail;
      do {
         real coeff = ( c.minmod_maxiter == 0 ) ? c.minmod_coeff
                    : c.minmod_coeff - (real)iter*c.minmod_coeff/(real)c.minmod_maxiter;
         coeff = FMAX( coeff, (real)0.0 );
         reconstruct( &c, cc, &w, coeff );
         compute_flux( &c, &w );
         if ( flux != NULL ) store_int_flux( &w, flux + (size_t)p*9*g_nc*PS2*PS2 );
         fail = full_step_update( &c, cc, &w, out + (size_t)p*g_nc*PS2*PS2*PS2,
                                  ( de != NULL ) ? de + (size_t)p*PS2*PS2*PS2 : NULL );
         iter++;
      } while ( fail && iter <= c.minmod_maxiter );
   }
   free( w.pri );  free( w.slope );  free( w.fc );  free( w.flux );  free( cc );  free( hf );
   return 0;
}

int EXPORT(solve_mhm)( const real *in, real *out, real *flux, char *de, int npg, int nxt,
                       int lr, int rsolver, int dual, int limiter, double minmod_coeff, int minmod_maxiter,
                       double dt, double dh, double min_dens, double min_pres, double min_eint,
                       double de_switch, double gamma, int char_rec )
{
   return solve_impl( in, out, flux, de, npg, nxt, lr, rsolver, dual, limiter, minmod_coeff, minmod_maxiter,
                      dt, dh, min_dens, min_pres, min_eint, de_switch, gamma, char_rec, 0, 0 );
}

/* The same with FLU_SCHEME = MHM_RP (PLM; FLU_NXT = 22, or more with the central window read). */
int EXPORT(solve_mhm_rp)( const real *in, real *out, real *flux, char *de, int npg, int nxt,
                          int rsolver, int dual, int limiter, double minmod_coeff, int minmod_maxiter,
                          double dt, double dh, double min_dens, double min_pres, double min_eint,
                          double de_switch, double gamma )
{
   return solve_impl( in, out, flux, de, npg, nxt, LR_PLM, rsolver, dual, limiter, minmod_coeff, minmod_maxiter,
                      dt, dh, min_dens, min_pres, min_eint, de_switch, gamma, 0, 1, 0 );
}

/* The same with npass user passive scalars (NCOMP_PASSIVE_USER) before the dual-energy field:
 * in[npg][5+npass(+1)][nxt^3], reconstructed as densities and upwinded with the mass flux, not
 * floored. */
int EXPORT(solve_mhm_passive)( const real *in, real *out, real *flux, char *de, int npg, int nxt,
                               int lr, int rsolver, int dual, int npass, int limiter, double minmod_coeff,
                               int minmod_maxiter, double dt, double dh, double min_dens, double min_pres,
                               double min_eint, double de_switch, double gamma )
{
   return solve_impl( in, out, flux, de, npg, nxt, lr, rsolver, dual, limiter, minmod_coeff, minmod_maxiter,
                      dt, dh, min_dens, min_pres, min_eint, de_switch, gamma, 0, 0, npass );
}
