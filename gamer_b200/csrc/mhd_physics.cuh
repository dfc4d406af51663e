// Per-cell and per-face MHD of the CTU patch-group solver (ideal gas, 8 variables: rho, m, E, B).
//
// Variables are stored unrotated: 0 rho, 1..3 momentum, 4 total energy (incl. 1/2 B^2), 5..7 B.
// Face direction D is a template parameter; "n/t1/t2" index the normal and transverse components
// (Dir<D>) of momentum (+0) and of B (+4).  The branch structure follows the reference routines
// cited per function.
#pragma once
#include "hydro_physics.cuh"
#include "hydro_pair.cuh"

namespace gb {

constexpr int NM = 8;            // NCOMP_TOTAL_PLUS_MAG with MHD, no passive scalars
constexpr int MO = 5;            // MAG_OFFSET

template <int D> struct MDir {
   static constexpr int n  = 1 + D,              t1 = 1 + ( D + 1 ) % 3,  t2 = 1 + ( D + 2 ) % 3;
   static constexpr int bn = MO + D,             b1 = MO + ( D + 1 ) % 3, b2 = MO + ( D + 2 ) % 3;
};

// Hydro_Con2Eint with the magnetic energy (CPU_Shared_FluUtility.cpp:1259)
template <int P, typename R>
GB_DEV R eint_con_mhd( R d, R ird, R a, R b, R c, R e, R emag )
{
   if constexpr ( P == P_MIXED )
   {
      // float where the subtraction cannot cancel (kinetic + magnetic <= E/4), double elsewhere
      // (the bound of eint_con in hydro_physics.cuh)
      const R ke = R(0.5)*( a*a + b*b + c*c )*ird;
      if ( ke + emag <= R(0.25)*e ) return e - ke - emag;
      const double m2 = (double)a*(double)a + (double)b*(double)b + (double)c*(double)c;
      return (R)( (double)e - 0.5*m2*rcp_dd( (double)d ) - (double)emag );
   }
   else
      return e - R(0.5)*( a*a + b*b + c*c )*ird - emag;
}

template <typename R> GB_DEV R emag_of( const R *u ) { return R(0.5)*( u[5]*u[5] + u[6]*u[6] + u[7]*u[7] ); }

// Hydro_Con2Pri with MHD (CPU_Shared_FluUtility.cpp:209): B copied, pressure floored
template <int P, typename R>
GB_DEV void mhd_con2pri( const Phys<R> &ph, const R *u, R *w )
{
   const R ir = R(1)/u[0];
   w[0] = u[0];
   w[1] = u[1]*ir;  w[2] = u[2]*ir;  w[3] = u[3]*ir;
   w[4] = check_floor( eint_con_mhd<P>( u[0], ir, u[1], u[2], u[3], u[4], emag_of( u ) )*ph.gm1, ph.min_pres );
   w[5] = u[5];  w[6] = u[6];  w[7] = u[7];
}

// Hydro_Pri2Con with MHD (CPU_Shared_FluUtility.cpp:343)
template <typename R>
GB_DEV void mhd_pri2con( const Phys<R> &ph, const R *w, R *u )
{
   u[0] = w[0];
   u[1] = w[0]*w[1];  u[2] = w[0]*w[2];  u[3] = w[0]*w[3];
   u[4] = R(0.5)*( u[1]*u[1] + u[2]*u[2] + u[3]*u[3] )/u[0] + w[4]*ph.inv_gm1 + emag_of( w );
   u[5] = w[5];  u[6] = w[6];  u[7] = w[7];
}

// Hydro_Con2Flux with MHD terms (CPU_Shared_FluUtility.cpp:458-548), pressure given
template <int D, typename R>
GB_DEV void mhd_con2flux( const R *u, R ird, R pres, R *f )
{
   typedef MDir<D> M;
   const R Bx = u[M::bn], By = u[M::b1], Bz = u[M::b2];
   const R emag = R(0.5)*( Bx*Bx + By*By + Bz*Bz );
   const R vx = ird*u[M::n], vy = ird*u[M::t1], vz = ird*u[M::t2];
   f[0]     = u[M::n];
   f[M::n]  = vx*u[M::n] + pres;
   f[M::t1] = vx*u[M::t1];
   f[M::t2] = vx*u[M::t2];
   f[4]     = vx*( u[4] + pres );
   f[M::n]  += emag - Bx*Bx;
   f[M::t1] -= Bx*By;
   f[M::t2] -= Bx*Bz;
   f[4]     += vx*emag - Bx*( Bx*vx + By*vy + Bz*vz );
   f[M::bn]  = R(0);
   f[M::b1]  = By*vx - Bx*vy;
   f[M::b2]  = Bz*vx - Bx*vz;
}

// fast magnetosonic speed squared (HLLE/HLLD, e.g. CPU_Shared_RiemannSolver_HLLD.cpp:150-190)
template <typename R>
GB_DEV R fast_speed2( R a2, R cax2, R cat2 )
{
   const R ca2_plus_a2 = cat2 + cax2 + a2;
   const R ca2_min_a2  = cat2 + cax2 - a2;
   const R cf2_min_cs2 = gsqrt( ca2_min_a2*ca2_min_a2 + R(4)*a2*cat2 );
   if ( cat2 == R(0) ) return ( cax2 >= a2 ) ? cax2 : a2;
   if ( cax2 == R(0) ) return a2 + cat2;
   return R(0.5)*( ca2_plus_a2 + cf2_min_cs2 );
}

// HLLE for MHD, Davis wave speeds (CPU_Shared_RiemannSolver_HLLE.cpp:302-700, MHD branch)
template <int D, int P, typename R>
GB_DEV void hlle_mhd( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   typedef MDir<D> M;
   const R irl = R(1)/L[0], irr = R(1)/Rt[0];
   const R ul = irl*L[M::n], ur = irr*Rt[M::n];
   const R bx2l = L[M::bn]*L[M::bn], bx2r = Rt[M::bn]*Rt[M::bn];
   const R bt2l = L[M::b1]*L[M::b1] + L[M::b2]*L[M::b2], bt2r = Rt[M::b1]*Rt[M::b1] + Rt[M::b2]*Rt[M::b2];
   const R eml = R(0.5)*( bx2l + bt2l ), emr = R(0.5)*( bx2r + bt2r );
   const R pl = check_floor( eint_con_mhd<P>( L[0],  irl, L[M::n],  L[M::t1],  L[M::t2],  L[4],  eml )*ph.gm1, ph.min_pres );
   const R pr = check_floor( eint_con_mhd<P>( Rt[0], irr, Rt[M::n], Rt[M::t1], Rt[M::t2], Rt[4], emr )*ph.gm1, ph.min_pres );
   const R a2l = ph.gamma*pl*irl, a2r = ph.gamma*pr*irr;
   const R cfl = gsqrt( fast_speed2( a2l, bx2l*irl, bt2l*irl ) );
   const R cfr = gsqrt( fast_speed2( a2r, bx2r*irr, bt2r*irr ) );
   R mvl = gmin( ul - cfl, ur - cfr ), mvr = gmax( ul + cfl, ur + cfr );
   mvl = gmin( mvl, R(0) );
   mvr = gmax( mvr, R(0) );
   R fl[NM], fr[NM];
   mhd_con2flux<D>( L,  irl, pl, fl );
   mhd_con2flux<D>( Rt, irr, pr, fr );
   const int w7[7] = { 0, M::n, M::t1, M::t2, 4, M::b1, M::b2 };
#  pragma unroll
   for (int k=0; k<7; k++) { fl[w7[k]] -= mvl*L[w7[k]];  fr[w7[k]] -= mvr*Rt[w7[k]]; }
   if ( mvl == R(0) && mvr == R(0) )
   {
#     pragma unroll
      for (int k=0; k<7; k++) fo[w7[k]] = fl[w7[k]];
   }
   else
   {
      const R id = R(1)/( mvr - mvl );
#     pragma unroll
      for (int k=0; k<7; k++) fo[w7[k]] = id*( mvr*fl[w7[k]] - mvl*fr[w7[k]] );
   }
   fo[M::bn] = R(0);
}

// Roe's solver for MHD with the Eulerian Y factor (Hydro_RiemannSolver_Roe with MHD and EULERY,
// CPU_Shared_RiemannSolver_Roe.cpp:83-719; Stone et al. 2008, ApJS 178, 137, appendix B), without
// the intermediate-state check, which the reference compiles in only when the patch-group solver
// itself is Roe.  The 7 waves are (rho, m_n, m_t1, m_t2, E, B_t1, B_t2) along D; the longitudinal
// field is L's (equal to Rt's at a face) and its flux is zero.
template <int D, int P, typename R>
GB_DEV void roe_mhd( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   typedef MDir<D> M;
   const int w7[7] = { 0, M::n, M::t1, M::t2, 4, M::b1, M::b2 };
   const R half = R(0.5), one = R(1), two = R(2);
   const R gm1 = ph.gm1, gm2 = ph.gamma - two;
   const R irl = one/L[0], irr = one/Rt[0];
   const R Bx = L[M::bn], ByL = L[M::b1], BzL = L[M::b2], ByR = Rt[M::b1], BzR = Rt[M::b2];
   const R eml = half*( Bx*Bx + ByL*ByL + BzL*BzL );
   const R emr = half*( Bx*Bx + ByR*ByR + BzR*BzR );
   const R pl = check_floor( eint_con_mhd<P>( L[0],  irl, L[M::n],  L[M::t1],  L[M::t2],  L[4],  eml )*gm1, ph.min_pres );
   const R pr = check_floor( eint_con_mhd<P>( Rt[0], irr, Rt[M::n], Rt[M::t1], Rt[M::t2], Rt[4], emr )*gm1, ph.min_pres );
   const R hl = irl*( L[4] + pl + eml ), hr = irr*( Rt[4] + pr + emr );

   const R sl = gsqrt( L[0] ), sr = gsqrt( Rt[0] );
   const R rho = sl*sr, irho = one/rho;
   const R isl = one/sl, isr = one/sr, iss = one/( sl + sr );
   const R u  = iss*( isl*L[M::n]  + isr*Rt[M::n]  );
   const R v  = iss*( isl*L[M::t1] + isr*Rt[M::t1] );
   const R w  = iss*( isl*L[M::t2] + isr*Rt[M::t2] );
   const R V2 = u*u + v*v + w*w;
   const R H  = iss*( sl*hl + sr*hr );

   const R rho_sqrt = gsqrt( rho ), irho_sqrt = one/rho_sqrt;
   const R By = iss*( sl*ByR + sr*ByL ), Bz = iss*( sl*BzR + sr*BzL );
   const R Bn2 = By*By + Bz*Bz, Bn = gsqrt( Bn2 );
   const R B2 = Bx*Bx + Bn2, B2_rho = B2*irho;
   const R S = gsign( Bx );
   const R dBy = ByR - ByL, dBz = BzR - BzL;
   const R X = half*( dBy*dBy + dBz*dBz )*( iss*iss )*gm2;
   const R Y = half*( L[0] + Rt[0] )*irho*gm2;
   const R gm1_mY = gm1 - Y;
   const R Bn_star = gsqrt( gm1_mY )*Bn;
   R beta_y, beta_z, beta_ys, beta_zs;
   if ( Bn == R(0) ) { beta_y = one;  beta_z = R(0); }
   else              { const R i = one/Bn;  beta_y = By*i;  beta_z = Bz*i; }
   if ( Bn_star == R(0) ) { beta_ys = one;  beta_zs = R(0); }
   else                   { const R i = one/Bn_star;  beta_ys = By*i;  beta_zs = Bz*i; }
   const R beta_ns2 = beta_ys*beta_ys + beta_zs*beta_zs;

   R gp = gm1*( H - half*V2 );
   gp -= gm1*B2_rho;
   gp = ph.gamma*irho*check_floor( gp*rho/ph.gamma, ph.min_pres );
   const R a2 = gp - X, a = gsqrt( a2 );

   const R cax2 = Bx*Bx*irho, cax = gsqrt( cax2 );
   const R cat2 = ( gm1 - Y )*Bn2*irho;
   const R ca2_plus_a2 = cat2 + cax2 + a2, ca2_min_a2 = cat2 + cax2 - a2;
   const R cf2_min_cs2 = gsqrt( ca2_min_a2*ca2_min_a2 + R(4)*a2*cat2 );
   R cf2, cs2;
   if ( cat2 == R(0) )
   {
      if      ( cax2 == a2 ) { cf2 = a2;    cs2 = a2;   }
      else if ( cax2 >  a2 ) { cf2 = cax2;  cs2 = a2;   }
      else                   { cf2 = a2;    cs2 = cax2; }
   }
   else
   {
      if ( cax2 == R(0) ) { cf2 = a2 + cat2;  cs2 = R(0); }
      else                { cf2 = half*( ca2_plus_a2 + cf2_min_cs2 );  cs2 = a2*cax2/cf2; }
   }
   const R cf = gsqrt( cf2 ), cs = gsqrt( cs2 );
   const R a2_min_cs2 = a2 - cs2, cf2_min_a2 = cf2 - a2;
   R af, as;
   if      ( cf2_min_cs2 == R(0) ) { af = one;   as = R(0); }
   else if ( a2_min_cs2 <= R(0) )  { af = R(0);  as = one;  }
   else if ( cf2_min_a2 <= R(0) )  { af = one;   as = R(0); }
   else { const R i = one/cf2_min_cs2;  af = gsqrt( a2_min_cs2*i );  as = gsqrt( cf2_min_a2*i ); }

   const R ev[7] = { u - cf, u - cax, u - cs, u, u + cs, u + cax, u + cf };
   R fl[NM], fr[NM];
   mhd_con2flux<D>( L,  irl, pl, fl );
   mhd_con2flux<D>( Rt, irr, pr, fr );
   if ( ev[0] >= R(0) )
   {
#     pragma unroll
      for (int k=0; k<NM; k++) fo[k] = fl[k];
      return;
   }
   if ( ev[6] <= R(0) )
   {
#     pragma unroll
      for (int k=0; k<NM; k++) fo[k] = fr[k];
      return;
   }

   // right eigenvectors (columns of RE) and left eigenvectors (rows of LE), eqs. A13-A17, B28-B30
   R RE[7][7], LE[7][7];
   const R Af = a*af*rho_sqrt, As = a*as*rho_sqrt, Cff = cf*af, Css = cs*as, Qf = Cff*S, Qs = Css*S;
   RE[0][0] = af;  RE[0][1] = R(0);  RE[0][2] = as;  RE[0][3] = one;  RE[0][4] = as;  RE[0][5] = R(0);  RE[0][6] = af;
   const R u_af = u*af, u_as = u*as;
   RE[1][0] = u_af - Cff;  RE[1][1] = R(0);  RE[1][2] = u_as - Css;  RE[1][3] = u;
   RE[1][4] = u_as + Css;  RE[1][5] = R(0);  RE[1][6] = u_af + Cff;
   const R v_af = v*af, v_as = v*as, Qs_bys = Qs*beta_ys, Qf_bys = Qf*beta_ys;
   RE[2][0] = v_af + Qs_bys;  RE[2][1] = -beta_z;  RE[2][2] = v_as - Qf_bys;  RE[2][3] = v;
   RE[2][4] = v_as + Qf_bys;  RE[2][5] = beta_z;   RE[2][6] = v_af - Qs_bys;
   const R w_af = w*af, w_as = w*as, Qs_bzs = Qs*beta_zs, Qf_bzs = Qf*beta_zs;
   RE[3][0] = w_af + Qs_bzs;  RE[3][1] = beta_y;   RE[3][2] = w_as - Qf_bzs;  RE[3][3] = w;
   RE[3][4] = w_as + Qf_bzs;  RE[3][5] = -beta_y;  RE[3][6] = w_af - Qs_bzs;
   const R Hp = H - B2_rho, u_cf = u*cf, u_cs = u*cs;
   const R v_by_w_bz = v*beta_ys + w*beta_zs;
   const R Qs_vw = Qs*v_by_w_bz, Qf_vw = Qf*v_by_w_bz;
   const R Bn_b2_rho = Bn_star*beta_ns2*irho;
   const R As_Bn = As*Bn_b2_rho, Af_Bn = Af*Bn_b2_rho;
   RE[4][0] = af*( Hp - u_cf ) + Qs_vw + As_Bn;
   RE[4][1] = -( v*beta_z - w*beta_y );
   RE[4][2] = as*( Hp - u_cs ) - Qf_vw - Af_Bn;
   RE[4][3] = half*V2 + X/gm1;
   RE[4][4] = as*( Hp + u_cs ) + Qf_vw - Af_Bn;
   RE[4][5] = -RE[4][1];
   RE[4][6] = af*( Hp + u_cf ) - Qs_vw + As_Bn;
   const R bys_rho = beta_ys*irho;
   RE[5][0] = As*bys_rho;  RE[5][1] = -S*beta_z*irho_sqrt;  RE[5][2] = -Af*bys_rho;  RE[5][3] = R(0);
   RE[5][4] = RE[5][2];    RE[5][5] = RE[5][1];             RE[5][6] = RE[5][0];
   const R bzs_rho = beta_zs*irho;
   RE[6][0] = As*bzs_rho;  RE[6][1] = S*beta_y*irho_sqrt;   RE[6][2] = -Af*bzs_rho;  RE[6][3] = R(0);
   RE[6][4] = RE[6][2];    RE[6][5] = RE[6][1];             RE[6][6] = RE[6][0];

   const R Qy = beta_ys/beta_ns2, Qz = beta_zs/beta_ns2;
   const R nh = half/a2, nb = nh*gm1;
   const R Cff_h = nh*Cff, Css_h = nh*Css, Af_h = nh*Af, As_h = nh*As, Qf_h = nh*Qf, Qs_h = nh*Qs, X_h = nh*X;
   const R af_b = nb*af, as_b = nb*as;
   const R af_V2_Hp = af_b*( V2 - Hp ), as_V2_Hp = as_b*( V2 - Hp );
   const R v_Qy_w_Qz = v*Qy + w*Qz;
   const R Qf_vQ = Qf_h*v_Qy_w_Qz, Qs_vQ = Qs_h*v_Qy_w_Qz;
   const R Bn_rho = Bn_star*irho;
   const R Af_Bn_rho = Af_h*Bn_rho, As_Bn_rho = As_h*Bn_rho;
   LE[0][0] = af_V2_Hp + Cff_h*( cf + u ) - Qs_vQ - As_Bn_rho;
   LE[1][0] = half*( v*beta_z - w*beta_y );
   LE[2][0] = as_V2_Hp + Css_h*( cs + u ) + Qf_vQ + Af_Bn_rho;
   LE[3][0] = one - nb*V2 + two*X_h;
   LE[4][0] = as_V2_Hp + Css_h*( cs - u ) - Qf_vQ + Af_Bn_rho;
   LE[5][0] = -LE[1][0];
   LE[6][0] = af_V2_Hp + Cff_h*( cf - u ) + Qs_vQ - As_Bn_rho;
   const R u_af_b = u*af_b, u_as_b = u*as_b;
   LE[0][1] = -u_af_b - Cff_h;  LE[1][1] = R(0);  LE[2][1] = -u_as_b - Css_h;  LE[3][1] = two*nb*u;
   LE[4][1] = -u_as_b + Css_h;  LE[5][1] = R(0);  LE[6][1] = -u_af_b + Cff_h;
   const R v_af_b = v*af_b, v_as_b = v*as_b, Qs_Qy = Qs_h*Qy, Qf_Qy = Qf_h*Qy;
   LE[0][2] = -v_af_b + Qs_Qy;  LE[1][2] = -half*beta_z;  LE[2][2] = -v_as_b - Qf_Qy;  LE[3][2] = two*nb*v;
   LE[4][2] = -v_as_b + Qf_Qy;  LE[5][2] = -LE[1][2];     LE[6][2] = -v_af_b - Qs_Qy;
   const R w_af_b = w*af_b, w_as_b = w*as_b, Qs_Qz = Qs_h*Qz, Qf_Qz = Qf_h*Qz;
   LE[0][3] = -w_af_b + Qs_Qz;  LE[1][3] = half*beta_y;   LE[2][3] = -w_as_b - Qf_Qz;  LE[3][3] = two*nb*w;
   LE[4][3] = -w_as_b + Qf_Qz;  LE[5][3] = -LE[1][3];     LE[6][3] = -w_af_b - Qs_Qz;
   LE[0][4] = af_b;  LE[1][4] = R(0);  LE[2][4] = as_b;  LE[3][4] = -gm1/a2;
   LE[4][4] = as_b;  LE[5][4] = R(0);  LE[6][4] = af_b;
   LE[0][5] = As_h*Qy - af_b*By;  LE[1][5] = -half*S*beta_z*rho_sqrt;  LE[2][5] = -Af_h*Qy - as_b*By;
   LE[3][5] = two*nb*By;  LE[4][5] = LE[2][5];  LE[5][5] = LE[1][5];  LE[6][5] = LE[0][5];
   LE[0][6] = As_h*Qz - af_b*Bz;  LE[1][6] = half*S*beta_y*rho_sqrt;   LE[2][6] = -Af_h*Qz - as_b*Bz;
   LE[3][6] = two*nb*Bz;  LE[4][6] = LE[2][6];  LE[5][6] = LE[1][6];  LE[6][6] = LE[0][6];

   // wave amplitudes of the jump (the structure of the left eigenvectors, eq. B31-B37)
   R J[7], A[7];
#  pragma unroll
   for (int k=0; k<7; k++) J[k] = Rt[ w7[k] ] - L[ w7[k] ];
   A[0] = LE[0][0]*J[0] + LE[0][1]*J[1] + LE[0][2]*J[2] + LE[0][3]*J[3];
   A[1] = LE[1][0]*J[0]                 + LE[1][2]*J[2] + LE[1][3]*J[3];
   A[2] = LE[2][0]*J[0] + LE[2][1]*J[1] + LE[2][2]*J[2] + LE[2][3]*J[3];
   A[3] = LE[3][0]*J[0] + LE[3][1]*J[1] + LE[3][2]*J[2] + LE[3][3]*J[3]
        + LE[3][4]*J[4] + LE[3][5]*J[5] + LE[3][6]*J[6];
   A[4] = LE[4][0]*J[0] + LE[4][1]*J[1] + LE[4][2]*J[2] + LE[4][3]*J[3];
   A[5] = -A[1];
   A[6] = LE[6][0]*J[0] + LE[6][1]*J[1] + LE[6][2]*J[2] + LE[6][3]*J[3];
   const R t0 = LE[0][4]*J[4] + LE[0][5]*J[5] + LE[0][6]*J[6];
   const R t1 =                 LE[1][5]*J[5] + LE[1][6]*J[6];
   const R t2 = LE[2][4]*J[4] + LE[2][5]*J[5] + LE[2][6]*J[6];
   A[0] += t0;  A[1] += t1;  A[2] += t2;  A[4] += t2;  A[5] += t1;  A[6] += t0;

#  pragma unroll
   for (int k=0; k<7; k++) A[k] *= gabs( ev[k] );
#  pragma unroll
   for (int r=0; r<7; r++)
   {
      R f = fl[ w7[r] ] + fr[ w7[r] ];
#     pragma unroll
      for (int t=0; t<7; t++) f -= A[t]*RE[r][t];
      fo[ w7[r] ] = f*half;
   }
   fo[M::bn] = R(0);
}

// HLLD, Davis wave speeds (CPU_Shared_RiemannSolver_HLLD.cpp:65-440)
template <int D, int P, typename R>
GB_DEV void hlld( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   typedef MDir<D> M;
   const R maxerr = ( sizeof(R) == 8 ) ? R(1.0e-14) : R(1.0e-06);     // MAX_ERROR (include/Macro.h)
   const R maxerr2 = maxerr*maxerr;
   const R Bx = L[M::bn], ByL = L[M::b1], BzL = L[M::b2], ByR = Rt[M::b1], BzR = Rt[M::b2];
   const R iBx = R(1)/Bx, Bx2 = Bx*Bx, iBx2 = iBx*iBx;
   // primitive states (rotated components named explicitly)
   R wl[NM], wr[NM];
   mhd_con2pri<P>( ph, L, wl );
   mhd_con2pri<P>( ph, Rt, wr );
   const R rl = wl[0], rr = wr[0];
   const R uL = wl[M::n], vL = wl[M::t1], zL = wl[M::t2], uR = wr[M::n], vR = wr[M::t1], zR = wr[M::t2];
   const R pL = wl[4], pR = wr[4];
   const R irl = R(1)/L[0], irr = R(1)/Rt[0];
   const R btl2 = ByL*ByL + BzL*BzL, btr2 = ByR*ByR + BzR*BzR;
   const R b2l = R(0.5)*( Bx2 + btl2 ), b2r = R(0.5)*( Bx2 + btr2 );
   const R ptl = pL + b2l, ptr = pR + b2r;
   const R cfl = gsqrt( fast_speed2( ph.gamma*pL/L[0], Bx2*irl, btl2*irl ) );
   const R cfr = gsqrt( fast_speed2( ph.gamma*pR/Rt[0], Bx2*irr, btr2*irr ) );
   const R S0 = gmin( uL - cfl, uR - cfr );
   const R S4 = gmax( uL + cfl, uR + cfr );
   R fl[NM], fr[NM];
   mhd_con2flux<D>( L,  irl, pL, fl );
   mhd_con2flux<D>( Rt, irr, pR, fr );
   if ( S0 >= R(0) ) {
#     pragma unroll
      for (int v=0; v<NM; v++) fo[v] = fl[v];
      return;
   }
   if ( S4 <= R(0) ) {
#     pragma unroll
      for (int v=0; v<NM; v++) fo[v] = fr[v];
      return;
   }
   const R sdl = S0 - uL, sdr = S4 - uR;
   const R t1 = sdl*rl, t2 = sdr*rr;
   const R S2 = ( t2*uR - t1*uL - ptr + ptl )/( t2 - t1 );
   const R sdml = S0 - S2, sdmr = S4 - S2;
   const R sl_sml = sdl/sdml, sr_smr = sdr/sdmr;
   // star states in the rotated frame: [0 rho, 1 mn, 2 mt1, 3 mt2, 4 E, 5 Bn, 6 Bt1, 7 Bt2]
   R Ls[NM], Rs[NM], Lds[NM], Rds[NM];
   Ls[0] = L[0]*sl_sml;
   Rs[0] = Rt[0]*sr_smr;
   const R sqls = gsqrt( Ls[0] ), sqrs = gsqrt( Rs[0] );
   const R S1 = S2 - gabs( Bx )/sqls;
   const R S3 = S2 + gabs( Bx )/sqrs;
   const R pts = ptl + rl*sdl*( sdl - sdml );
   Ls[1] = Ls[0]*S2;
   Ls[5] = Bx;
   R tmp = gmin( b2l, b2r );
   const R critbx = ( tmp == R(0) ) ? R(0) : gabs( R(0.5)*Bx2/tmp );
   R crit = ( critbx < maxerr2 ) ? L[0]*sdl*sdml : L[0]*sdl*sdml*iBx2 - R(1);
   if ( gabs( crit ) < maxerr ) {
      Ls[2] = Ls[0]*vL;  Ls[3] = Ls[0]*zL;  Ls[6] = ByL;  Ls[7] = BzL;
   }
   else if ( critbx < maxerr2 ) {
      Ls[2] = Ls[0]*vL;  Ls[3] = Ls[0]*zL;  Ls[6] = ByL*sl_sml;  Ls[7] = BzL*sl_sml;
   }
   else {
      const R ic = R(1)/crit;
      R q = ( sdl - sdml )*iBx*ic;
      Ls[2] = Ls[0]*( vL - ByL*q );
      Ls[3] = Ls[0]*( zL - BzL*q );
      q = ( L[0]*sdl*sdl - Bx2 )*iBx2*ic;
      Ls[6] = ByL*q;  Ls[7] = BzL*q;
   }
   const R vbl = ( Ls[1]*Ls[5] + Ls[2]*Ls[6] + Ls[3]*Ls[7] )/Ls[0];
   Ls[4] = ( sdl*L[4] - ptl*uL + pts*S2 + Bx*( uL*Bx + vL*ByL + zL*BzL - vbl ) )/sdml;
   const R irls = R(1)/Ls[0];
   const R vyls = irls*Ls[2], vzls = irls*Ls[3];
   Rs[1] = Rs[0]*S2;
   Rs[5] = Bx;
   crit = ( critbx < maxerr2 ) ? Rt[0]*sdr*sdmr : Rt[0]*sdr*sdmr*iBx2 - R(1);
   if ( gabs( crit ) < maxerr ) {
      Rs[2] = Rs[0]*vR;  Rs[3] = Rs[0]*zR;  Rs[6] = ByR;  Rs[7] = BzR;
   }
   else if ( critbx < maxerr2 ) {
      Rs[2] = Rs[0]*vR;  Rs[3] = Rs[0]*zR;  Rs[6] = ByR*sr_smr;  Rs[7] = BzR*sr_smr;
   }
   else {
      const R ic = R(1)/crit;
      R q = ( sdr - sdmr )*iBx*ic;
      Rs[2] = Rs[0]*( vR - ByR*q );
      Rs[3] = Rs[0]*( zR - BzR*q );
      q = ( Rt[0]*sdr*sdr - Bx2 )*iBx2*ic;
      Rs[6] = ByR*q;  Rs[7] = BzR*q;
   }
   const R vbr = ( Rs[1]*Rs[5] + Rs[2]*Rs[6] + Rs[3]*Rs[7] )/Rs[0];
   Rs[4] = ( sdr*Rt[4] - ptr*uR + pts*S2 + Bx*( uR*Bx + vR*ByR + zR*BzR - vbr ) )/sdmr;
   const R irrs = R(1)/Rs[0];
   const R vyrs = irrs*Rs[2], vzrs = irrs*Rs[3];
   if ( critbx < maxerr2 )
   {
#     pragma unroll
      for (int v=0; v<NM; v++) { Lds[v] = Ls[v];  Rds[v] = Rs[v]; }
   }
   else
   {
      const R isum = R(1)/( sqls + sqrs );
      const R sg = gsign( Bx );
      Lds[0] = Ls[0];  Rds[0] = Rs[0];
      Lds[1] = Ls[1];  Rds[1] = Rs[1];
      tmp = isum*( sqls*vyls + sqrs*vyrs + sg*( Rs[6] - Ls[6] ) );
      Lds[2] = Lds[0]*tmp;  Rds[2] = Rds[0]*tmp;
      tmp = isum*( sqls*vzls + sqrs*vzrs + sg*( Rs[7] - Ls[7] ) );
      Lds[3] = Lds[0]*tmp;  Rds[3] = Rds[0]*tmp;
      tmp = isum*( sqls*Rs[6] + sqrs*Ls[6] + sg*sqls*sqrs*( vyrs - vyls ) );
      Lds[6] = tmp;  Rds[6] = tmp;
      tmp = isum*( sqls*Rs[7] + sqrs*Ls[7] + sg*sqls*sqrs*( vzrs - vzls ) );
      Lds[7] = tmp;  Rds[7] = tmp;
      Lds[5] = Ls[5];  Rds[5] = Rs[5];
      tmp = S2*Bx + ( Lds[2]*Lds[6] + Lds[3]*Lds[7] )/Lds[0];
      Lds[4] = Ls[4] - sqls*sg*( vbl - tmp );
      Rds[4] = Rs[4] + sqrs*sg*( vbr - tmp );
   }
   // map rotated star components to the storage positions
   const int map[NM] = { 0, M::n, M::t1, M::t2, 4, M::bn, M::b1, M::b2 };
   if ( S1 >= R(0) )
   {
#     pragma unroll
      for (int k=0; k<5; k++) fo[map[k]] = fl[map[k]] + S0*( Ls[k] - L[map[k]] );
      fo[M::b1] = fl[M::b1] + S0*( Ls[6] - ByL );
      fo[M::b2] = fl[M::b2] + S0*( Ls[7] - BzL );
   }
   else if ( S2 >= R(0) )
   {
      const R c = S1 - S0;
#     pragma unroll
      for (int k=0; k<5; k++) fo[map[k]] = fl[map[k]] - S0*L[map[k]] - c*Ls[k] + S1*Lds[k];
      fo[M::b1] = fl[M::b1] - S0*ByL - c*Ls[6] + S1*Lds[6];
      fo[M::b2] = fl[M::b2] - S0*BzL - c*Ls[7] + S1*Lds[7];
   }
   else if ( S3 > R(0) )
   {
      const R c = S3 - S4;
#     pragma unroll
      for (int k=0; k<5; k++) fo[map[k]] = fr[map[k]] - S4*Rt[map[k]] - c*Rs[k] + S3*Rds[k];
      fo[M::b1] = fr[M::b1] - S4*ByR - c*Rs[6] + S3*Rds[6];
      fo[M::b2] = fr[M::b2] - S4*BzR - c*Rs[7] + S3*Rds[7];
   }
   else
   {
#     pragma unroll
      for (int k=0; k<5; k++) fo[map[k]] = fr[map[k]] + S4*( Rs[k] - Rt[map[k]] );
      fo[M::b1] = fr[M::b1] + S4*( Rs[6] - ByR );
      fo[M::b2] = fr[M::b2] + S4*( Rs[7] - BzR );
   }
   fo[M::bn] = R(0);
}

// the double evaluation of eint_con_mhd<P_MIXED>, out of line: the rare path of the packed HLLD
static __device__ __noinline__ float eint_mhd_double( float d, float a, float b, float c, float e, float emag )
{
   const double m2 = (double)a*(double)a + (double)b*(double)b + (double)c*(double)c;
   return (float)( (double)e - 0.5*m2*rcp_dd( (double)d ) - (double)emag );
}

// HLLD for the float policies with the work of the left and right state as the two lanes of
// float2 (packed add/mul/fma.rn.f32x2, hydro_pair.cuh): primitive recovery, fluxes, fast speeds,
// the star states and their energies.  The branches (early exits, the three cases of the star
// transverse components, the weak-Bx double star, the four flux regions) are hlld's, per lane where
// they are per state (CPU_Shared_RiemannSolver_HLLD.cpp:65-440).
template <int D, int P>
GB_DEV void hlld_pair( const Phys<float> &ph, const float *L, const float *Rt, float *fo )
{
   typedef MDir<D> M;
   constexpr int n = M::n, t1 = M::t1, t2 = M::t2;
   const float maxerr = 1.0e-06f, maxerr2 = maxerr*maxerr;                // MAX_ERROR (include/Macro.h)
   const float Bx = L[M::bn];
   const float2 By = make_float2( L[M::b1], Rt[M::b1] ), Bz = make_float2( L[M::b2], Rt[M::b2] );
   const float iBx = 1.f/Bx, Bx2 = Bx*Bx, iBx2 = iBx*iBx;
   const float2 rho = make_float2( L[0], Rt[0] );
   const float2 ir  = make_float2( 1.f/L[0], 1.f/Rt[0] );
   const float2 mm[3] = { make_float2( L[1], Rt[1] ), make_float2( L[2], Rt[2] ), make_float2( L[3], Rt[3] ) };
   const float2 en = make_float2( L[4], Rt[4] );
   // mhd_con2pri: pressure from E - 1/2 m^2/rho - 1/2 B^2 (storage order), floored
   float2 pres;
   {
      const float2 b5 = make_float2( L[5], Rt[5] ), b6 = make_float2( L[6], Rt[6] ), b7 = make_float2( L[7], Rt[7] );
      const float2 em = p_mul( p_bc( 0.5f ), p_fma( b7, b7, p_fma( b6, b6, p_mul( b5, b5 ) ) ) );
      const float2 k2 = p_fma( mm[2], mm[2], p_fma( mm[1], mm[1], p_mul( mm[0], mm[0] ) ) );
      const float2 ke = p_mul( p_mul( p_bc( 0.5f ), k2 ), ir );
      float2 ei = p_sub( p_sub( en, ke ), em );
      if constexpr ( P == P_MIXED )
      {
         if ( !( ke.x + em.x <= 0.25f*en.x ) ) ei.x = eint_mhd_double( L[0],  L[1],  L[2],  L[3],  L[4],  em.x );
         if ( !( ke.y + em.y <= 0.25f*en.y ) ) ei.y = eint_mhd_double( Rt[0], Rt[1], Rt[2], Rt[3], Rt[4], em.y );
      }
      const float2 pr = p_mul( ei, p_bc( ph.gm1 ) );
      pres = make_float2( check_floor( pr.x, ph.min_pres ), check_floor( pr.y, ph.min_pres ) );
   }
   const float2 un = p_mul( mm[n-1], ir ), vt = p_mul( mm[t1-1], ir ), zt = p_mul( mm[t2-1], ir );
   const float2 bt2 = p_fma( Bz, Bz, p_mul( By, By ) );
   const float2 b2  = p_mul( p_bc( 0.5f ), p_add( p_bc( Bx2 ), bt2 ) );
   const float2 pt  = p_add( pres, b2 );
   const float2 a2  = p_mul( p_mul( p_bc( ph.gamma ), pres ), ir );
   const float2 cax = p_mul( p_bc( Bx2 ), ir ), cat = p_mul( bt2, ir );
   const float2 cf  = make_float2( sqrtf( fast_speed2( a2.x, cax.x, cat.x ) ), sqrtf( fast_speed2( a2.y, cax.y, cat.y ) ) );
   const float2 wm = p_sub( un, cf ), wp = p_add( un, cf );
   const float S0 = fminf( wm.x, wm.y ), S4 = fmaxf( wp.x, wp.y );
   // mhd_con2flux of both states
   float2 f[NM];
   {
      const float2 emag = p_mul( p_bc( 0.5f ), p_fma( Bz, Bz, p_fma( By, By, p_bc( Bx*Bx ) ) ) );
      const float2 mn = mm[n-1], m1 = mm[t1-1], m2 = mm[t2-1];
      const float2 nbx = p_bc( -Bx );
      f[0]    = mn;
      f[n]    = p_add( p_fma( un, mn, pres ), p_fma( nbx, p_bc( Bx ), emag ) );
      f[t1]   = p_fma( nbx, By, p_mul( un, m1 ) );
      f[t2]   = p_fma( nbx, Bz, p_mul( un, m2 ) );
      const float2 dot = p_fma( Bz, zt, p_fma( By, vt, p_mul( p_bc( Bx ), un ) ) );
      f[4]    = p_fma( nbx, dot, p_fma( un, emag, p_mul( un, p_add( en, pres ) ) ) );
      f[M::bn] = p_bc( 0.f );
      f[M::b1] = p_fma( nbx, vt, p_mul( By, un ) );
      f[M::b2] = p_fma( nbx, zt, p_mul( Bz, un ) );
   }
   if ( S0 >= 0.f ) {
#     pragma unroll
      for (int v=0; v<NM; v++) fo[v] = f[v].x;
      return;
   }
   if ( S4 <= 0.f ) {
#     pragma unroll
      for (int v=0; v<NM; v++) fo[v] = f[v].y;
      return;
   }
   const float2 S04 = make_float2( S0, S4 );
   const float2 sd  = p_sub( S04, un );                         // (S0 - uL, S4 - uR)
   const float2 tt  = p_mul( sd, rho );
   const float S2 = ( tt.y*un.y - tt.x*un.x - pt.y + pt.x )/( tt.y - tt.x );
   const float2 sdm = p_sub( S04, p_bc( S2 ) );
   const float2 ssm = make_float2( sd.x/sdm.x, sd.y/sdm.y );
   // star states in the rotated frame: [0 rho, 1 mn, 2 mt1, 3 mt2, 4 E, 5 Bn, 6 Bt1, 7 Bt2]
   const float2 s0 = p_mul( rho, ssm );
   const float2 sq = make_float2( sqrtf( s0.x ), sqrtf( s0.y ) );
   const float S1 = S2 - fabsf( Bx )/sq.x;
   const float S3 = S2 + fabsf( Bx )/sq.y;
   const float pts = pt.x + rho.x*sd.x*( sd.x - sdm.x );
   const float2 s1 = p_mul( s0, p_bc( S2 ) );
   const float tmn = fminf( b2.x, b2.y );
   const float critbx = ( tmn == 0.f ) ? 0.f : fabsf( 0.5f*Bx2/tmn );
   const bool weak = ( critbx < maxerr2 );
   const float2 csd  = p_mul( p_mul( rho, sd ), sdm );
   const float2 crit = weak ? csd : p_fma( csd, p_bc( iBx2 ), p_bc( -1.f ) );
   float2 s2, s3, s6, s7;
   if ( weak )
   {
      s2 = p_mul( s0, vt );  s3 = p_mul( s0, zt );
      s6 = p_mul( By, ssm ); s7 = p_mul( Bz, ssm );
   }
   else
   {
      const float2 ic = make_float2( 1.f/crit.x, 1.f/crit.y );
      float2 q = p_mul( p_mul( p_sub( sd, sdm ), p_bc( iBx ) ), ic );
      const float2 nq = p_mul( q, p_bc( -1.f ) );
      s2 = p_mul( s0, p_fma( By, nq, vt ) );
      s3 = p_mul( s0, p_fma( Bz, nq, zt ) );
      q = p_mul( p_mul( p_sub( p_mul( p_mul( rho, sd ), sd ), p_bc( Bx2 ) ), p_bc( iBx2 ) ), ic );
      s6 = p_mul( By, q );  s7 = p_mul( Bz, q );
   }
   if ( fabsf( crit.x ) < maxerr ) { s2.x = s0.x*vt.x;  s3.x = s0.x*zt.x;  s6.x = By.x;  s7.x = Bz.x; }
   if ( fabsf( crit.y ) < maxerr ) { s2.y = s0.y*vt.y;  s3.y = s0.y*zt.y;  s6.y = By.y;  s7.y = Bz.y; }
   const float2 vbn = p_fma( s3, s7, p_fma( s2, s6, p_mul( s1, p_bc( Bx ) ) ) );
   const float2 vb  = make_float2( vbn.x/s0.x, vbn.y/s0.y );
   const float2 ub  = p_fma( zt, Bz, p_fma( vt, By, p_mul( un, p_bc( Bx ) ) ) );
   float2 e4 = p_mul( sd, en );
   e4 = p_fma( pt, p_mul( un, p_bc( -1.f ) ), e4 );
   e4 = p_fma( p_bc( pts ), p_bc( S2 ), e4 );
   e4 = p_fma( p_bc( Bx ), p_sub( ub, vb ), e4 );
   const float2 s4 = make_float2( e4.x/sdm.x, e4.y/sdm.y );
   const float2 irs = make_float2( 1.f/s0.x, 1.f/s0.y );
   const float2 vys = p_mul( irs, s2 ), vzs = p_mul( irs, s3 );
   // double star (Lds/Rds)
   float2 d2 = s2, d3 = s3, d4 = s4, d6 = s6, d7 = s7;
   if ( !weak )
   {
      const float isum = 1.f/( sq.x + sq.y );
      const float sg = ( Bx < 0.f ) ? -1.f : 1.f;
      float tm = isum*( sq.x*vys.x + sq.y*vys.y + sg*( s6.y - s6.x ) );
      d2 = p_mul( s0, p_bc( tm ) );
      tm = isum*( sq.x*vzs.x + sq.y*vzs.y + sg*( s7.y - s7.x ) );
      d3 = p_mul( s0, p_bc( tm ) );
      tm = isum*( sq.x*s6.y + sq.y*s6.x + sg*sq.x*sq.y*( vys.y - vys.x ) );
      d6 = p_bc( tm );
      tm = isum*( sq.x*s7.y + sq.y*s7.x + sg*sq.x*sq.y*( vzs.y - vzs.x ) );
      d7 = p_bc( tm );
      tm = S2*Bx + ( d2.x*d6.x + d3.x*d7.x )/s0.x;
      d4 = make_float2( s4.x - sq.x*sg*( vb.x - tm ), s4.y + sq.y*sg*( vb.y - tm ) );
   }
   // fluxes of the four regions, rotated star components mapped to the storage positions
   const int map[5] = { 0, n, t1, t2, 4 };
   const float2 st[5] = { s0, s1, s2, s3, s4 }, dst[5] = { s0, s1, d2, d3, d4 };
   if ( S1 >= 0.f )
   {
#     pragma unroll
      for (int k=0; k<5; k++) fo[map[k]] = f[map[k]].x + S0*( st[k].x - L[map[k]] );
      fo[M::b1] = f[M::b1].x + S0*( s6.x - By.x );
      fo[M::b2] = f[M::b2].x + S0*( s7.x - Bz.x );
   }
   else if ( S2 >= 0.f )
   {
      const float c = S1 - S0;
#     pragma unroll
      for (int k=0; k<5; k++) fo[map[k]] = f[map[k]].x - S0*L[map[k]] - c*st[k].x + S1*dst[k].x;
      fo[M::b1] = f[M::b1].x - S0*By.x - c*s6.x + S1*d6.x;
      fo[M::b2] = f[M::b2].x - S0*Bz.x - c*s7.x + S1*d7.x;
   }
   else if ( S3 > 0.f )
   {
      const float c = S3 - S4;
#     pragma unroll
      for (int k=0; k<5; k++) fo[map[k]] = f[map[k]].y - S4*Rt[map[k]] - c*st[k].y + S3*dst[k].y;
      fo[M::b1] = f[M::b1].y - S4*By.y - c*s6.y + S3*d6.y;
      fo[M::b2] = f[M::b2].y - S4*Bz.y - c*s7.y + S3*d7.y;
   }
   else
   {
#     pragma unroll
      for (int k=0; k<5; k++) fo[map[k]] = f[map[k]].y + S4*( st[k].y - Rt[map[k]] );
      fo[M::b1] = f[M::b1].y + S4*( s6.y - By.y );
      fo[M::b2] = f[M::b2].y + S4*( s7.y - Bz.y );
   }
   fo[M::bn] = 0.f;
}

// HLLD with the HLLE rescue on NaN (CPU_Shared_ComputeFlux.cpp:313-362; RSOLVER_RESCUE = HLLE)
template <int D, int P, typename R>
GB_DEV void riemann_mhd( const Phys<R> &ph, const R *L, const R *Rt, R *fo )
{
   if constexpr ( std::is_same<R, float>::value ) hlld_pair<D,P>( ph, L, Rt, fo );
   else                                           hlld<D,P>( ph, L, Rt, fo );
   bool nan = false;
#  pragma unroll
   for (int v=0; v<NM; v++) nan |= ( fo[v] != fo[v] );
   if ( nan ) hlle_mhd<D,P>( ph, L, Rt, fo );
}

// MHD eigen-system along D of a primitive state (MHD_GetEigenSystem, CPU_Shared_DataReconstruction.cpp:1611-1893).
// Rows/columns are in the rotated 7-wave ordering (rho, vn, vt1, vt2, P, Bt1, Bt2); entries that the
// reference leaves at their constant initial values (0 or 1) are set here explicitly.
template <int D, typename R>
GB_DEV void mhd_eigen( const Phys<R> &ph, const R *w, R (&ev)[7], R (&LE)[7][7], R (&RE)[7][7] )
{
   typedef MDir<D> M;
   const R rho = w[0], irho = R(1)/rho;
   const R a2 = ph.gamma*w[4]/rho, a = gsqrt( a2 ), ia = R(1)/a, ia2 = ia*ia;
   const R Bx = w[M::bn], By = w[M::b1], Bz = w[M::b2];
   const R bn2 = By*By + Bz*Bz, bn = gsqrt( bn2 );
   const R cax2 = Bx*Bx*irho, cax = gsqrt( cax2 ), cat2 = bn2*irho;
   const R tsum = cax2 + cat2 + a2, tdif = cax2 + cat2 - a2;
   const R cf2_min_cs2 = gsqrt( tdif*tdif + R(4)*a2*cat2 );
   R cf2, cs2;
   if ( cat2 == R(0) )
   {
      if      ( cax2 == a2 ) { cf2 = a2;    cs2 = a2;   }
      else if ( cax2 >  a2 ) { cf2 = cax2;  cs2 = a2;   }
      else                   { cf2 = a2;    cs2 = cax2; }
   }
   else
   {
      if ( cax2 == R(0) ) { cf2 = a2 + cat2;  cs2 = R(0); }
      else                { cf2 = R(0.5)*( tsum + cf2_min_cs2 );  cs2 = a2*cax2/cf2; }
   }
   const R cf = gsqrt( cf2 ), cs = gsqrt( cs2 );
   const R vn = w[M::n];
   ev[0] = vn - cf;  ev[1] = vn - cax;  ev[2] = vn - cs;  ev[3] = vn;
   ev[4] = vn + cs;  ev[5] = vn + cax;  ev[6] = vn + cf;
   const R S = gsign( Bx );
   const R sqr = gsqrt( rho ), isqr = R(1)/sqr;
   const R a2_min_cs2 = a2 - cs2, cf2_min_a2 = cf2 - a2;
   R by, bz, af, as;
   if ( bn == R(0) ) { by = R(1);  bz = R(0); }
   else              { const R ibn = R(1)/bn;  by = By*ibn;  bz = Bz*ibn; }
   if      ( cf2_min_cs2 == R(0) ) { af = R(1);  as = R(0); }
   else if ( a2_min_cs2 <= R(0) )  { af = R(0);  as = R(1); }
   else if ( cf2_min_a2 <= R(0) )  { af = R(1);  as = R(0); }
   else { const R i = R(1)/cf2_min_cs2;  af = gsqrt( a2_min_cs2*i );  as = gsqrt( cf2_min_a2*i ); }
   const R Af = a*af*sqr, As = a*as*sqr, Cff = cf*af, Css = cs*as, Qf = Cff*S, Qs = Css*S;
   const R S_sqr = S*sqr;
#  pragma unroll
   for (int r=0; r<7; r++)
#     pragma unroll
      for (int c=0; c<7; c++) { RE[r][c] = R(0);  LE[r][c] = R(0); }
   RE[0][0] =  rho*af;  RE[0][1] = -Cff;  RE[0][2] =  Qs*by;  RE[0][3] =  Qs*bz;
   RE[0][4] =  RE[0][0]*a2;  RE[0][5] =  As*by;  RE[0][6] =  As*bz;
   RE[1][2] = -bz;  RE[1][3] =  by;  RE[1][5] = -S_sqr*bz;  RE[1][6] =  S_sqr*by;
   RE[2][0] =  rho*as;  RE[2][1] = -Css;  RE[2][2] = -Qf*by;  RE[2][3] = -Qf*bz;
   RE[2][4] =  RE[2][0]*a2;  RE[2][5] = -Af*by;  RE[2][6] = -Af*bz;
   RE[3][0] = R(1);
   RE[4][0] =  RE[2][0];  RE[4][1] = -RE[2][1];  RE[4][2] = -RE[2][2];  RE[4][3] = -RE[2][3];
   RE[4][4] =  RE[2][4];  RE[4][5] =  RE[2][5];  RE[4][6] =  RE[2][6];
   RE[5][2] = -RE[1][2];  RE[5][3] = -RE[1][3];  RE[5][5] =  RE[1][5];  RE[5][6] =  RE[1][6];
   RE[6][0] =  RE[0][0];  RE[6][1] = -RE[0][1];  RE[6][2] = -RE[0][2];  RE[6][3] = -RE[0][3];
   RE[6][4] =  RE[0][4];  RE[6][5] =  RE[0][5];  RE[6][6] =  RE[0][6];
   const R N = R(0.5)*ia2, Nby = N*by, Nbz = N*bz, As_r = As*irho, Af_r = Af*irho, S_isqr = S*isqr;
   LE[0][1] = -N*Cff;  LE[0][2] =  Nby*Qs;  LE[0][3] =  Nbz*Qs;  LE[0][4] =  N*af*irho;
   LE[0][5] =  Nby*As_r;  LE[0][6] =  Nbz*As_r;
   LE[1][2] = -R(0.5)*bz;  LE[1][3] =  R(0.5)*by;  LE[1][5] =  LE[1][2]*S_isqr;  LE[1][6] =  LE[1][3]*S_isqr;
   LE[2][1] = -N*Css;  LE[2][2] = -Nby*Qf;  LE[2][3] = -Nbz*Qf;  LE[2][4] =  N*as*irho;
   LE[2][5] = -Nby*Af_r;  LE[2][6] = -Nbz*Af_r;
   LE[3][0] = R(1);  LE[3][4] = -ia2;
   LE[4][1] = -LE[2][1];  LE[4][2] = -LE[2][2];  LE[4][3] = -LE[2][3];  LE[4][4] =  LE[2][4];
   LE[4][5] =  LE[2][5];  LE[4][6] =  LE[2][6];
   LE[5][2] = -LE[1][2];  LE[5][3] = -LE[1][3];  LE[5][5] =  LE[1][5];  LE[5][6] =  LE[1][6];
   LE[6][1] = -LE[0][1];  LE[6][2] = -LE[0][2];  LE[6][3] = -LE[0][3];  LE[6][4] =  LE[0][4];
   LE[6][5] =  LE[0][5];  LE[6][6] =  LE[0][6];
}


// MHD slopes limited in the 7-wave characteristic variables of the cell (Hydro_LimitSlope with MHD and
// CHAR_RECONSTRUCTION, CPU_Shared_DataReconstruction.cpp:1918-2030, through Hydro_Pri2Char:1436-1486 and
// Hydro_Char2Pri:1513-1576).  LE / RE are the cell's eigenvectors along D (mhd_eigen).  The normal B
// carries no wave: its slope is zero.  The left / right / centred (and van Leer) primitive slopes go
// to wave amplitudes with the rows of LE, where the structure of the left eigenvectors pairs the fast
// (0, 6) and slow (2, 4) modes as f +- b of their fluid and magnetic parts; each amplitude is limited
// on its own, and the limited amplitudes go back with the columns of RE, the pressure from the
// density through the entropy mode (P = a^2 (rho - entropy amplitude)).
template <int D, typename R>
GB_DEV void mhd_char_limited_slopes( const Phys<R> &ph, const R (&LE)[7][7], const R (&RE)[7][7],
                                     const R *cl, const R *cc, const R *cr, int lim, R coeff, R (&s)[NM] )
{
   typedef MDir<D> M;
   const int wv[7] = { 0, M::n, M::t1, M::t2, 4, M::b1, M::b2 };   // wave-ordered primitive -> storage
   R sl[7], sr[7], sc[7], sa[7];
#  pragma unroll
   for (int q=0; q<7; q++)
   {
      const R l = cc[wv[q]] - cl[wv[q]], r = cr[wv[q]] - cc[wv[q]];
      sl[q] = l;  sr[q] = r;
      sc[q] = R(0.5)*( l + r );
      sa[q] = ( l*r > R(0) ) ? R(2)*l*r/( l + r ) : R(0);
   }
   auto to_waves = [&]( R (&t)[7] ) {
      const R f0 = LE[0][1]*t[1] + LE[0][2]*t[2] + LE[0][3]*t[3];
      const R b0 = LE[0][4]*t[4] + LE[0][5]*t[5] + LE[0][6]*t[6];
      const R f2 = LE[2][1]*t[1] + LE[2][2]*t[2] + LE[2][3]*t[3];
      const R b2 = LE[2][4]*t[4] + LE[2][5]*t[5] + LE[2][6]*t[6];
      const R w1 = LE[1][2]*t[2] + LE[1][3]*t[3] + LE[1][5]*t[5] + LE[1][6]*t[6];
      const R w5 = LE[5][2]*t[2] + LE[5][3]*t[3] + LE[5][5]*t[5] + LE[5][6]*t[6];
      const R w3 = t[0] + LE[3][4]*t[4];
      t[0] = f0 + b0;   t[1] = w1;   t[2] = f2 + b2;   t[3] = w3;
      t[4] = -f2 + b2;  t[5] = w5;   t[6] = -f0 + b0;
   };
   to_waves( sl );  to_waves( sr );  to_waves( sc );
   if ( lim == LIM_VL_GMINMOD ) to_waves( sa );
   R w[7];
#  pragma unroll
   for (int m=0; m<7; m++) w[m] = limit_slopes( sl[m], sr[m], sc[m], sa[m], lim, coeff );
   const R a2 = ph.gamma*cc[4]/cc[0];
   const R rho = RE[0][0]*w[0] + RE[2][0]*w[2] + w[3] + RE[4][0]*w[4] + RE[6][0]*w[6];
   s[0]    = rho;
   s[M::n] = RE[0][1]*w[0] + RE[2][1]*w[2] + RE[4][1]*w[4] + RE[6][1]*w[6];
#  pragma unroll
   for (int q=2; q<4; q++)
      s[wv[q]] = RE[0][q]*w[0] + RE[1][q]*w[1] + RE[2][q]*w[2] + RE[4][q]*w[4] + RE[5][q]*w[5] + RE[6][q]*w[6];
   s[4] = ( rho - w[3] )*a2;
   s[M::bn] = R(0);
#  pragma unroll
   for (int q=5; q<7; q++)
      s[wv[q]] = RE[0][q]*w[0] + RE[1][q]*w[1] + RE[2][q]*w[2] + RE[4][q]*w[4] + RE[5][q]*w[5] + RE[6][q]*w[6];
}

} // namespace gb
