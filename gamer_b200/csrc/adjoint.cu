// Adjoint kernels of the MHM + PLM step and the periodic-box gather/scatter used by K-step runs.
// See adjoint.cuh for the derivation and the symbol names.
#include <cstring>
#include <new>
#include "../../include/gamer_b200_fluid.h"
#include "adjoint.cuh"

namespace gb {

constexpr int OUT3 = PS2*PS2*PS2;

GB_DEV int cc_index( int i, int j, int k ) { return ( k*ADJ_N + j )*ADJ_N + i; }

// items of one patch group per grid.y index (blockIdx.y = patch group of the chunk), 32-bit indices
#define ADJ_PG_LOOP( r, per ) \
   const int pg = blockIdx.y; \
   for (int r = blockIdx.x*blockDim.x + threadIdx.x; r < ( per ); r += gridDim.x*blockDim.x)
GB_DEV int fc_index( int i, int j, int k ) { return ( k*ADJ_F + j )*ADJ_F + i; }

// primitive variables of input cell (i,j,k) of patch group window u
template <int P, typename R>
GB_DEV void load_pri( const Phys<R> &ph, const R *u, int i, int j, int k, R *w )
{
   R c[ADJ_NC];
   const int idx = cc_index( i, j, k );
#  pragma unroll
   for (int v=0; v<ADJ_NC; v++) c[v] = u[v*ADJ_N3 + idx];
   con2pri<P,ADJ_NC>( ph, c, w );
}

// face primitive states of one fc cell along D from the stencil, with the branch codes
template <int D, typename R>
GB_DEV void adj_faces( const R *wl, const R *wc, const R *wr, R coeff, R *fl, R *fr, int *br )
{
#  pragma unroll
   for (int v=0; v<ADJ_NC; v++)
   {
      const R s = gminmod_branch( wl[v], wc[v], wr[v], coeff, br[v] );
      // no clamp acts for generalized MinMod with theta < 2 (see plm_clamp_needed)
      fl[v] = wc[v] - R(0.5)*s;
      fr[v] = R(2)*wc[v] - fl[v];
      fl[v] = R(2)*wc[v] - fr[v];
   }
}

// ---- A1: forward recompute of the face states with the tape ---------------------------------
template <typename R, int P>
__global__ void adj_forward_kernel( const __grid_constant__ AdjArgs<R> a )
{
   ADJ_PG_LOOP( f, ADJ_F3 )
   {
      const int i = f % ADJ_F, j = ( f / ADJ_F ) % ADJ_F, k = f / ( ADJ_F*ADJ_F );
      const R *u = a.in + (size_t)pg*ADJ_NC*ADJ_N3;
      const int ci = i + 1, cj = j + 1, ck = k + 1;
      R wc[ADJ_NC], wm[ADJ_NC], wp[ADJ_NC], fpri[6][ADJ_NC], fcon[6][ADJ_NC], acc[ADJ_NC];
      int br[ADJ_NC];
      load_pri<P>( a.ph, u, ci, cj, ck, wc );
      uint8_t *tape = a.tape + (size_t)pg*3*ADJ_NC*ADJ_F3;
#     pragma unroll
      for (int d=0; d<3; d++)
      {
         load_pri<P>( a.ph, u, ci - ( d == 0 ), cj - ( d == 1 ), ck - ( d == 2 ), wm );
         load_pri<P>( a.ph, u, ci + ( d == 0 ), cj + ( d == 1 ), ck + ( d == 2 ), wp );
         if      ( d == 0 ) adj_faces<0>( wm, wc, wp, a.coeff, fpri[0], fpri[1], br );
         else if ( d == 1 ) adj_faces<1>( wm, wc, wp, a.coeff, fpri[2], fpri[3], br );
         else               adj_faces<2>( wm, wc, wp, a.coeff, fpri[4], fpri[5], br );
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++) tape[( d*ADJ_NC + v )*ADJ_F3 + f] = (uint8_t)br[v];
      }
#     pragma unroll
      for (int d=0; d<3; d++)
      {
         R fL[ADJ_NC], fR[ADJ_NC];
         pri2con<ADJ_NC>( a.ph, fpri[2*d], fcon[2*d] );
         pri2con<ADJ_NC>( a.ph, fpri[2*d+1], fcon[2*d+1] );
         if      ( d == 0 ) { pri_con2flux<0,ADJ_NC>( fpri[0], fcon[0], fL );  pri_con2flux<0,ADJ_NC>( fpri[1], fcon[1], fR ); }
         else if ( d == 1 ) { pri_con2flux<1,ADJ_NC>( fpri[2], fcon[2], fL );  pri_con2flux<1,ADJ_NC>( fpri[3], fcon[3], fR ); }
         else               { pri_con2flux<2,ADJ_NC>( fpri[4], fcon[4], fL );  pri_con2flux<2,ADJ_NC>( fpri[5], fcon[5], fR ); }
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++) acc[v] = ( d == 0 ) ? fR[v] - fL[v] : ( acc[v] + fR[v] ) - fL[v];
      }
      const R k2 = R(0.5)*a.dt/a.dh;
      bool bad = false;
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++)
      {
         const R df = k2*acc[v];
#        pragma unroll
         for (int q=0; q<6; q++) fcon[q][v] -= df;
      }
#     pragma unroll
      for (int q=0; q<6; q++)
      {
         const R d = fcon[q][0], en = fcon[q][4], p = fpri[q][4];
         bad |= ( d < Lim<R>::tiny() || d > Lim<R>::huge() || d != d );
         bad |= ( en < Lim<R>::tiny() || en > Lim<R>::huge() || en != en );
         bad |= ( p < R(0) || p > Lim<R>::huge() || p != p );
      }
      if ( bad )
      {
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++)
         {
            const R c = u[v*ADJ_N3 + cc_index( ci, cj, ck )];
#           pragma unroll
            for (int q=0; q<6; q++) fcon[q][v] = c;
         }
      }
      else
      {
#        pragma unroll
         for (int q=0; q<6; q++)
         {
            fcon[q][0] = gmax( fcon[q][0], a.ph.min_dens );
            fcon[q][4] = floor_eint_in_engy<P>( a.ph, fcon[q][0], fcon[q][1], fcon[q][2], fcon[q][3], fcon[q][4] );
         }
      }
      a.tape[(size_t)a.npg*3*ADJ_NC*ADJ_F3 + (size_t)pg*ADJ_F3 + f] = bad ? 1 : 0;
      R *q = a.q + (size_t)pg*6*ADJ_NC*ADJ_F3;
#     pragma unroll
      for (int qq=0; qq<6; qq++)
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++) q[( qq*ADJ_NC + v )*ADJ_F3 + f] = fcon[qq][v];
   }
}

// ---- HLLC vector-Jacobian product by a reverse sweep --------------------------------------------
// (dF/dL)^T fbar and (dF/dR)^T fbar of riemann_hllc (CPU_Shared_RiemannSolver_HLLC.cpp:392-655, HD
// version, no passive scalars, pressures from E - 1/2 |m|^2/rho) in one backward pass over the
// same evaluation, about three flux evaluations instead of the ten of forward-mode tangents.  Every
// branch (wave-speed choices, floors, upwind side, the V_S = 0 special case) is the one the forward
// sweep takes, and each min/max/floor passes its adjoint to the operand it selected, as the
// dual-number evaluation does.  Returns false when the flux is NaN: the HLLE rescue applies there,
// and the caller differentiates that face with dual numbers.
template <int D, typename R>
GB_DEV bool hllc_vjp( const Phys<R> &ph, const R *L, const R *Rt, const double *fbar, double *lb, double *rb )
{
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   // ---- forward sweep
   const R irl = R(1)/L[0], irr = R(1)/Rt[0];
   const R ul = irl*L[n], ur = irr*Rt[n];
   const R m2l = L[n]*L[n] + L[t1]*L[t1] + L[t2]*L[t2], m2r = Rt[n]*Rt[n] + Rt[t1]*Rt[t1] + Rt[t2]*Rt[t2];
   const R plr = ( L[4]  - R(0.5)*m2l*irl )*ph.gm1;
   const R prr = ( Rt[4] - R(0.5)*m2r*irr )*ph.gm1;
   const bool fll = ( plr == plr ) && ( ph.min_pres > plr ), flr = ( prr == prr ) && ( ph.min_pres > prr );
   const R pl = fll ? ph.min_pres : plr, pr = flr ? ph.min_pres : prr;
   const R csl = gsqrt( ph.gamma*pl*irl ), csr = gsqrt( ph.gamma*pr*irr );
   const R wl1 = ul - csl, wl2 = ur - csr, wr1 = ul + csl, wr2 = ur + csr;
   const R wl = ( wl2 < wl1 ) ? wl2 : wl1, wr = ( wr2 > wr1 ) ? wr2 : wr1;
   const bool sl = ( wl1 < wl2 ), sr = ( wr2 > wr1 );
   const R Al = sl ? csl : ( ul - ur ) + csr;
   const R Ar = sr ? csr : ( ul - ur ) + csl;
   const R t1l = L[0]*Al, t1r = -Rt[0]*Ar;
   const R t2s = R(1)/( t1l - t1r );
   const R S   = pl - pr + t1l*ul - t1r*ur;
   const R vs  = t2s*S;
   const R Xr  = pr + t1r*ur, Xl = pl + t1l*ul;
   const R Q   = t1l*Xr - t1r*Xl;
   const R psr = t2s*Q;
   const bool fls = ( psr == psr ) && ( ph.min_pres > psr );
   const R ps  = fls ? ph.min_pres : psr;
   const bool left = ( vs >= R(0) );
   const R *U = left ? L : Rt;
   const R ir = left ? irl : irr, p = left ? pl : pr;
   const bool mvon = left ? !( R(0) < wl ) : !( R(0) > wr );
   const R mv = mvon ? ( left ? wl : wr ) : R(0);
   const R vx = ir*U[n];
   R f[5];
   f[0]  = U[n]           - mv*U[0];
   f[n]  = vx*U[n] + p    - mv*U[n];
   f[t1] = vx*U[t1]       - mv*U[t1];
   f[t2] = vx*U[t2]       - mv*U[t2];
   f[4]  = vx*( U[4] + p ) - mv*U[4];
   const bool special = left && vs == R(0) && mv == R(0);
   R clr = R(1), cst = R(0), t4 = R(0);
   if ( !special ) { t4 = R(1)/( vs - mv );  clr = t4*vs;  cst = -t4*mv*ps; }
   bool nan = false;
#  pragma unroll
   for (int v=0; v<5; v++)
   {
      R fo = clr*f[v];
      if ( v == n ) fo += cst;
      if ( v == 4 ) fo += cst*vs;
      nan |= ( fo != fo );
   }
   if ( nan ) return false;

   // ---- reverse sweep
   R fob[5];
#  pragma unroll
   for (int v=0; v<5; v++) fob[v] = (R)fbar[v];
   R clrb = R(0), fb[5];
#  pragma unroll
   for (int v=0; v<5; v++) { clrb += fob[v]*f[v];  fb[v] = fob[v]*clr; }
   const R cstb = fob[n] + fob[4]*vs;
   R vsb = fob[4]*cst, mvb = R(0), psb = R(0);
   if ( !special )
   {
      const R t4b = clrb*vs - cstb*mv*ps;
      vsb += clrb*t4;
      mvb -= cstb*t4*ps;
      psb -= cstb*t4*mv;
      const R db = -t4b*t4*t4;
      vsb += db;  mvb -= db;
   }
   R Ub[5];
#  pragma unroll
   for (int v=0; v<5; v++) { mvb -= fb[v]*U[v];  Ub[v] = -fb[v]*mv; }
   const R vxb = fb[n]*U[n] + fb[t1]*U[t1] + fb[t2]*U[t2] + fb[4]*( U[4] + p );
   Ub[n]  += fb[0] + fb[n]*vx + vxb*ir;
   Ub[t1] += fb[t1]*vx;
   Ub[t2] += fb[t2]*vx;
   Ub[4]  += fb[4]*vx;
   const R pb = fb[n] + fb[4]*vx, irb = vxb*U[n];
   R lr[5], rr[5], irlb = R(0), irrb = R(0), plb = R(0), prb = R(0), wlb = R(0), wrb = R(0);
#  pragma unroll
   for (int v=0; v<5; v++) { lr[v] = left ? Ub[v] : R(0);  rr[v] = left ? R(0) : Ub[v]; }
   if ( left ) { irlb += irb;  plb += pb;  if ( mvon ) wlb += mvb; }
   else        { irrb += irb;  prb += pb;  if ( mvon ) wrb += mvb; }
   // ps = floor( t2s*Q ), Q = t1l*Xr - t1r*Xl
   const R psrb = fls ? R(0) : psb;
   R t2sb = psrb*Q;
   const R Qb = psrb*t2s;
   R t1lb = Qb*Xr, t1rb = -Qb*Xl;
   const R Xrb = Qb*t1l, Xlb = -Qb*t1r;
   prb += Xrb;  t1rb += Xrb*ur;
   R urb = Xrb*t1r;
   plb += Xlb;  t1lb += Xlb*ul;
   R ulb = Xlb*t1l;
   // vs = t2s*S
   t2sb += vsb*S;
   const R Sb = vsb*t2s;
   plb += Sb;  prb -= Sb;  t1lb += Sb*ul;  ulb += Sb*t1l;  t1rb -= Sb*ur;  urb -= Sb*t1r;
   // t2s = 1/(t1l - t1r)
   const R Db = -t2sb*t2s*t2s;
   t1lb += Db;  t1rb -= Db;
   // t1l = L0*Al, t1r = -R0*Ar
   lr[0] += t1lb*Al;
   rr[0] -= t1rb*Ar;
   const R Alb = t1lb*L[0], Arb = -t1rb*Rt[0];
   R cslb = R(0), csrb = R(0);
   if ( sl ) cslb += Alb; else { ulb += Alb;  urb -= Alb;  csrb += Alb; }
   if ( sr ) csrb += Arb; else { ulb += Arb;  urb -= Arb;  cslb += Arb; }
   // wl = min(wl1, wl2), wr = max(wr1, wr2)
   R wl1b = R(0), wl2b = R(0), wr1b = R(0), wr2b = R(0);
   if ( wl2 < wl1 ) wl2b = wlb; else wl1b = wlb;
   if ( wr2 > wr1 ) wr2b = wrb; else wr1b = wrb;
   ulb += wl1b + wr1b;  cslb += wr1b - wl1b;
   urb += wl2b + wr2b;  csrb += wr2b - wl2b;
   // cs = sqrt( gamma*p*ir )
   {
      const R c2b = cslb*( ( csl > R(0) ) ? R(0.5)/csl : R(0) );
      plb += c2b*ph.gamma*irl;  irlb += c2b*ph.gamma*pl;
   }
   {
      const R c2b = csrb*( ( csr > R(0) ) ? R(0.5)/csr : R(0) );
      prb += c2b*ph.gamma*irr;  irrb += c2b*ph.gamma*pr;
   }
   // p = floor( (E - 1/2 m^2 ir)*(gamma-1) )
   if ( !fll )
   {
      const R eb = plb*ph.gm1, m2b = -eb*R(0.5)*irl;
      lr[4] += eb;  irlb -= eb*R(0.5)*m2l;
      lr[n] += R(2)*m2b*L[n];  lr[t1] += R(2)*m2b*L[t1];  lr[t2] += R(2)*m2b*L[t2];
   }
   if ( !flr )
   {
      const R eb = prb*ph.gm1, m2b = -eb*R(0.5)*irr;
      rr[4] += eb;  irrb -= eb*R(0.5)*m2r;
      rr[n] += R(2)*m2b*Rt[n];  rr[t1] += R(2)*m2b*Rt[t1];  rr[t2] += R(2)*m2b*Rt[t2];
   }
   // u = ir*m_n, ir = 1/rho
   irlb += ulb*L[n];   lr[n] += ulb*irl;
   irrb += urb*Rt[n];  rr[n] += urb*irr;
   lr[0] -= irlb*irl*irl;
   rr[0] -= irrb*irr*irr;
#  pragma unroll
   for (int v=0; v<5; v++) { lb[v] = (double)lr[v];  rb[v] = (double)rr[v]; }
   return true;
}

// ---- A2: per face, Fbar and the Riemann Jacobian-transpose products ---------------------------
template <int RS, int D, typename R, int P>
GB_DEV void adj_face( const AdjArgs<R> &a, int pg, int ia, int ib, int ic )
{
   // (ia, ib, ic): face index along D and the two transverse indices, in the rotated frame
   // (NSkip_N = 0, NSkip_T = 1: left fc cell (ia, ib+1, ic+1), right = left + e_D)
   int L[3], Rr[3];
   L[D] = ia;  L[( D + 1 ) % 3] = ib + 1;  L[( D + 2 ) % 3] = ic + 1;
   Rr[0] = L[0];  Rr[1] = L[1];  Rr[2] = L[2];  Rr[D] += 1;
   const int fl = fc_index( L[0], L[1], L[2] ), fr = fc_index( Rr[0], Rr[1], Rr[2] );
   // adjacent output cells: fc - 1 in every direction
   const double *g = a.gout + (size_t)pg*ADJ_NC*OUT3;
   double fbar[ADJ_NC];
   const int ol[3] = { L[0] - 1, L[1] - 1, L[2] - 1 }, orr[3] = { Rr[0] - 1, Rr[1] - 1, Rr[2] - 1 };
   const bool lin = ( ol[D] >= 0 ), rin = ( orr[D] < PS2 );
   const double dtdh = (double)a.dt/(double)a.dh;
#  pragma unroll
   for (int v=0; v<ADJ_NC; v++)
   {
      const double gl = lin ? g[v*OUT3 + ( ol[2]*PS2 + ol[1] )*PS2 + ol[0]] : 0.0;
      const double gr = rin ? g[v*OUT3 + ( orr[2]*PS2 + orr[1] )*PS2 + orr[0]] : 0.0;
      fbar[v] = dtdh*( gr - gl );
   }
   const R *q = a.q + (size_t)pg*6*ADJ_NC*ADJ_F3;
   R ql[ADJ_NC], qr[ADJ_NC];
#  pragma unroll
   for (int v=0; v<ADJ_NC; v++) { ql[v] = q[( ( 2*D + 1 )*ADJ_NC + v )*ADJ_F3 + fl];  qr[v] = q[( 2*D*ADJ_NC + v )*ADJ_F3 + fr]; }
   double *qb = a.qbar + (size_t)pg*6*ADJ_NC*ADJ_F3;
   if constexpr ( RS == RS_HLLC && ADJ_NC == 5 )
   {
      double lbv[ADJ_NC], rbv[ADJ_NC];
      if ( hllc_vjp<D,R>( a.ph, ql, qr, fbar, lbv, rbv ) )
      {
#        pragma unroll
         for (int w=0; w<ADJ_NC; w++)
         {
            qb[( ( 2*D + 1 )*ADJ_NC + w )*ADJ_F3 + fl] = lbv[w];
            qb[( 2*D*ADJ_NC + w )*ADJ_F3 + fr] = rbv[w];
         }
         return;
      }
   }
   // forward-mode dual numbers (one evaluation per side, ADJ_NC tangents each): the HLLE and Roe
   // adjoints, and the HLLC faces whose flux needs the HLLE rescue
   typedef Dual<ADJ_NC,R> DR;
   const Phys<DR> dph = dual_phys<R,ADJ_NC>( a.ph );
   // Jacobian w.r.t. the left state
   {
      DR dl[ADJ_NC], dr[ADJ_NC], fo[ADJ_NC];
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++) { dl[v] = DR::var( ql[v], v );  dr[v] = DR( (double)qr[v] ); }
      riemann<RS,D,P,ADJ_NC>( dph, dl, dr, fo );
#     pragma unroll
      for (int w=0; w<ADJ_NC; w++)
      {
         double s = 0.0;
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++) s += fbar[v]*(double)fo[v].d[w];
         qb[( ( 2*D + 1 )*ADJ_NC + w )*ADJ_F3 + fl] = s;
      }
   }
   // Jacobian w.r.t. the right state
   {
      DR dl[ADJ_NC], dr[ADJ_NC], fo[ADJ_NC];
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++) { dl[v] = DR( (double)ql[v] );  dr[v] = DR::var( qr[v], v ); }
      riemann<RS,D,P,ADJ_NC>( dph, dl, dr, fo );
#     pragma unroll
      for (int w=0; w<ADJ_NC; w++)
      {
         double s = 0.0;
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++) s += fbar[v]*(double)fo[v].d[w];
         qb[( 2*D*ADJ_NC + w )*ADJ_F3 + fr] = s;
      }
   }
}

// face t of direction D, numbered with x fastest (so that neighbouring threads touch neighbouring
// face states for every D): (ia, ib, ic) in the rotated frame of adj_face
template <int RS, int D, typename R, int P>
GB_DEV void adj_face_item( const AdjArgs<R> &a, int pg, int t )
{
   constexpr int e0 = ( D == 0 ) ? NFLX : PS2, e1 = ( D == 1 ) ? NFLX : PS2;
   const int c[3] = { t % e0, ( t / e0 ) % e1, t / ( e0*e1 ) };
   adj_face<RS,D,R,P>( a, pg, c[D], c[( D + 1 ) % 3], c[( D + 2 ) % 3] );
}

template <typename R, int P, int RS>
__global__ void adj_face_kernel( const __grid_constant__ AdjArgs<R> a )
{
   constexpr int NFACE = NFLX*PS2*PS2;        // per direction
   ADJ_PG_LOOP( r, 3*NFACE )
   {
      const int d  = r / NFACE, t = r % NFACE;
      if      ( d == 0 ) adj_face_item<RS,0,R,P>( a, pg, t );
      else if ( d == 1 ) adj_face_item<RS,1,R,P>( a, pg, t );
      else               adj_face_item<RS,2,R,P>( a, pg, t );
   }
}

// float HLLC: the reverse sweep fits 3 CTAs of 256 threads per SM (80 registers); the dual-number
// fallback of its rare NaN-rescue faces spills instead
template <typename R, int P>
__global__ void __launch_bounds__( 256, 3 ) adj_face_kernel_hllc( const __grid_constant__ AdjArgs<R> a )
{
   constexpr int NFACE = NFLX*PS2*PS2;        // per direction
   ADJ_PG_LOOP( r, 3*NFACE )
   {
      const int d  = r / NFACE, t = r % NFACE;
      if      ( d == 0 ) adj_face_item<RS_HLLC,0,R,P>( a, pg, t );
      else if ( d == 1 ) adj_face_item<RS_HLLC,1,R,P>( a, pg, t );
      else               adj_face_item<RS_HLLC,2,R,P>( a, pg, t );
   }
}

// ---- A3: per face-state cell, Hancock + PLM adjoint, scattered to Wbar --------------------------
template <int D, typename R>
GB_DEV void adj_face_prim( const Phys<R> &ph, const R *w, const double *ubar, double accbar_sign_scale,
                           const double *accbar, double *wbar )
{
   // wbar = (du/dw)^T ubar + sign * (dF/dw)^T accbar, with u = Pri2Con(w) and F = pri_con2flux<D>(w, u),
   // by a reverse sweep in double over those two short routines
   constexpr int n = Dir<D>::n, t1 = Dir<D>::t1, t2 = Dir<D>::t2;
   const double wv[ADJ_NC] = { (double)w[0], (double)w[1], (double)w[2], (double)w[3], (double)w[4] };
   const double k2 = wv[1]*wv[1] + wv[2]*wv[2] + wv[3]*wv[3];
   double u[ADJ_NC];
   u[0] = wv[0];  u[1] = wv[0]*wv[1];  u[2] = wv[0]*wv[2];  u[3] = wv[0]*wv[3];
   u[4] = 0.5*wv[0]*k2 + wv[4]*(double)ph.inv_gm1;
   double ub[ADJ_NC], fb[ADJ_NC], wb[ADJ_NC];
#  pragma unroll
   for (int v=0; v<ADJ_NC; v++) { ub[v] = ubar[v];  fb[v] = accbar_sign_scale*accbar[v];  wb[v] = 0.0; }
   // F: f0 = u_n, f_n = vx u_n + P, f_t = vx u_t, f4 = vx (u4 + P), vx = w_n, P = w4
   const double vx = wv[n], pres = wv[4];
   ub[n]  += fb[0] + fb[n]*vx;
   ub[t1] += fb[t1]*vx;
   ub[t2] += fb[t2]*vx;
   ub[4]  += fb[4]*vx;
   wb[n]  += fb[n]*u[n] + fb[t1]*u[t1] + fb[t2]*u[t2] + fb[4]*( u[4] + pres );
   wb[4]  += fb[n] + fb[4]*vx;
   // u: u0 = w0, u_i = w0 w_i, u4 = 1/2 w0 |w_v|^2 + w4/(gamma-1)
   const double k2b = 0.5*ub[4]*wv[0];
   wb[0] += ub[0] + ub[1]*wv[1] + ub[2]*wv[2] + ub[3]*wv[3] + 0.5*ub[4]*k2;
   wb[1] += ub[1]*wv[0] + 2.0*wv[1]*k2b;
   wb[2] += ub[2]*wv[0] + 2.0*wv[2]*k2b;
   wb[3] += ub[3]*wv[0] + 2.0*wv[3]*k2b;
   wb[4] += ub[4]*(double)ph.inv_gm1;
#  pragma unroll
   for (int x=0; x<ADJ_NC; x++) wbar[x] = wb[x];
}

// the part of one direction of an fc cell: the Hancock adjoint needs the sum of all six face
// adjoints (accbar), the face part only the two faces of this direction; the neighbours' adjoints
// are added atomically, the cell's own is summed into cen
template <int D, typename R, int P>
GB_DEV void adj_cell_dir( const AdjArgs<R> &a, int pg, int f, int ci, int cj, int ck, const double *qb,
                          const double (&accbar)[ADJ_NC], const R (&wc)[ADJ_NC], double (&cen)[ADJ_NC] )
{
   const R *u = a.in + (size_t)pg*ADJ_NC*ADJ_N3;
   const uint8_t *tape = a.tape + (size_t)pg*3*ADJ_NC*ADJ_F3;
   double *wb = a.wbar + (size_t)pg*ADJ_NC*ADJ_N3;
   double ubl[ADJ_NC], ubr[ADJ_NC];
#  pragma unroll
   for (int v=0; v<ADJ_NC; v++) { ubl[v] = qb[( 2*D*ADJ_NC + v )*ADJ_F3 + f];  ubr[v] = qb[( ( 2*D + 1 )*ADJ_NC + v )*ADJ_F3 + f]; }
   R wm[ADJ_NC], wp[ADJ_NC], fl[ADJ_NC], fr[ADJ_NC];
   int br[ADJ_NC];
   const int im = ci - ( D == 0 ), jm = cj - ( D == 1 ), km = ck - ( D == 2 );
   const int ip = ci + ( D == 0 ), jp = cj + ( D == 1 ), kp = ck + ( D == 2 );
   load_pri<P>( a.ph, u, im, jm, km, wm );
   load_pri<P>( a.ph, u, ip, jp, kp, wp );
   adj_faces<D>( wm, wc, wp, a.coeff, fl, fr, br );
   // F_{2d} enters acc with -, F_{2d+1} with +
   double wbl[ADJ_NC], wbr[ADJ_NC];
   adj_face_prim<D>( a.ph, fl, ubl, -1.0, accbar, wbl );
   adj_face_prim<D>( a.ph, fr, ubr,  1.0, accbar, wbr );
#  pragma unroll
   for (int v=0; v<ADJ_NC; v++)
   {
      // the recorded branch must be the one the values give now (same arithmetic)
      const int code = tape[( D*ADJ_NC + v )*ADJ_F3 + f];
      R sl_, sc_, sr_;
      gminmod_partials( code, a.coeff, sl_, sc_, sr_ );
      // fl = C - S/2, fr = C + S/2
      const double dl = (double)sl_, dc = (double)sc_, dr = (double)sr_;
      const double bl = wbl[v], bri = wbr[v];
      atomicAdd( &wb[v*ADJ_N3 + cc_index( im, jm, km )], -0.5*dl*bl + 0.5*dl*bri );
      cen[v] += bl*( 1.0 - 0.5*dc ) + bri*( 1.0 + 0.5*dc );
      atomicAdd( &wb[v*ADJ_N3 + cc_index( ip, jp, kp )], -0.5*dr*bl + 0.5*dr*bri );
   }
}

// 3 CTAs of 256 threads per SM (80 registers; the few spills cost less than the lost occupancy:
// backward pass 33.3 -> 31.5 ms for K = 8 steps of 1024 patch groups)
template <typename R, int P>
__global__ void __launch_bounds__( 256, ( sizeof(R) == 8 ) ? 1 : 3 ) adj_cell_kernel( const __grid_constant__ AdjArgs<R> a )
{
   // one fc cell per item, its three directions in turn: the six face adjoints are summed once and
   // the cell's own adjoint is added once
   ADJ_PG_LOOP( f, ADJ_F3 )
   {
      const int i = f % ADJ_F, j = ( f / ADJ_F ) % ADJ_F, k = f / ( ADJ_F*ADJ_F );
      const double *qb = a.qbar + (size_t)pg*6*ADJ_NC*ADJ_F3;
      // sum over the six faces of each variable's adjoint (Hancock and reset both use it)
      double s[ADJ_NC];
      bool any = false;
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++)
      {
         double acc = 0.0;
#        pragma unroll
         for (int q=0; q<6; q++) { const double x = qb[( q*ADJ_NC + v )*ADJ_F3 + f];  acc += x;  any |= ( x != 0.0 ); }
         s[v] = acc;
      }
      if ( !any ) continue;
      const int ci = i + 1, cj = j + 1, ck = k + 1;
      const bool reset = a.tape[(size_t)a.npg*3*ADJ_NC*ADJ_F3 + (size_t)pg*ADJ_F3 + f] != 0;
      if ( reset )
      {
         // MHM_CHECK_PREDICT reset: every face state was the cell value
         double *ue = a.uext + (size_t)pg*ADJ_NC*ADJ_N3;
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++) atomicAdd( &ue[v*ADJ_N3 + cc_index( ci, cj, ck )], s[v] );
         continue;
      }
      // Hancock: q_f = u_f - k2 * acc  ->  ubar_f = qbar_f,  accbar = -k2 * sum_f qbar_f
      const double k2 = 0.5*(double)a.dt/(double)a.dh;
      double accbar[ADJ_NC], cen[ADJ_NC];
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++) { accbar[v] = -k2*s[v];  cen[v] = 0.0; }
      R wc[ADJ_NC];
      load_pri<P>( a.ph, a.in + (size_t)pg*ADJ_NC*ADJ_N3, ci, cj, ck, wc );
      adj_cell_dir<0,R,P>( a, pg, f, ci, cj, ck, qb, accbar, wc, cen );
      adj_cell_dir<1,R,P>( a, pg, f, ci, cj, ck, qb, accbar, wc, cen );
      adj_cell_dir<2,R,P>( a, pg, f, ci, cj, ck, qb, accbar, wc, cen );
      double *wb = a.wbar + (size_t)pg*ADJ_NC*ADJ_N3;
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++) atomicAdd( &wb[v*ADJ_N3 + cc_index( ci, cj, ck )], cen[v] );
   }
}

// ---- A4: per input cell, Ubar = J_Con2Pri^T Wbar + direct + reset -------------------------------
template <typename R, int P>
__global__ void adj_con2pri_kernel( const __grid_constant__ AdjArgs<R> a )
{
   typedef Dual<ADJ_NC,R> DR;
   ADJ_PG_LOOP( c, ADJ_N3 )
   {
      const int i = c % ADJ_N, j = ( c / ADJ_N ) % ADJ_N, k = c / ( ADJ_N*ADJ_N );
      const R *u = a.in + (size_t)pg*ADJ_NC*ADJ_N3;
      const double *wb = a.wbar + (size_t)pg*ADJ_NC*ADJ_N3;
      const double *ue = a.uext + (size_t)pg*ADJ_NC*ADJ_N3;
      double *gi = a.gin + (size_t)pg*ADJ_NC*ADJ_N3;
      double wbv[ADJ_NC];
      bool any = false;
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++) { wbv[v] = wb[v*ADJ_N3 + c];  any |= ( wbv[v] != 0.0 ); }
      double out[ADJ_NC];
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++) out[v] = ue[v*ADJ_N3 + c];
      if ( any )
      {
         const Phys<DR> dph = dual_phys<R,ADJ_NC>( a.ph );
         DR du[ADJ_NC], dw[ADJ_NC];
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++) du[v] = DR::var( u[v*ADJ_N3 + c], v );
         con2pri<P,ADJ_NC>( dph, du, dw );
#        pragma unroll
         for (int x=0; x<ADJ_NC; x++)
#           pragma unroll
            for (int v=0; v<ADJ_NC; v++) out[x] += wbv[v]*(double)dw[v].d[x];
      }
      // U_out = U_in - ...: the identity term of the output interior
      const int oi = i - 2, oj = j - 2, ok = k - 2;
      if ( oi >= 0 && oi < PS2 && oj >= 0 && oj < PS2 && ok >= 0 && ok < PS2 )
      {
         const double *g = a.gout + (size_t)pg*ADJ_NC*OUT3;
#        pragma unroll
         for (int v=0; v<ADJ_NC; v++) out[v] += g[v*OUT3 + ( ok*PS2 + oj )*PS2 + oi];
      }
#     pragma unroll
      for (int v=0; v<ADJ_NC; v++) gi[v*ADJ_N3 + c] = out[v];
   }
}

// ---- periodic box <-> patch-group windows ----------------------------------------------------
// box layout [ncomp][Z][Y][X] (x fastest), X = 16*npx ...; patch group p = (pz*npy + py)*npx + px;
// window [p][ncomp][nxt^3] with ghost width g = (nxt-16)/2 <= 16, wrapped periodically.
// Launch shapes: windows as grid (npg*ncomp), one window per CTA; box planes as grid
// (ceil(X*Y/B), npz, ncomp), each thread walking the 16 planes of one patch-group layer.  All index
// arithmetic is 32-bit within a window or a box plane.

// x - X if x >= X, x + X if x < 0 (|x| stays within one period for g <= 16)
GB_DEV int wrap1( int x, int X ) { return ( x < 0 ) ? x + X : ( x >= X ? x - X : x ); }

// one window per CTA (blockIdx.x = patch group x variable); with a compile-time width NXT the CTA
// has one thread per (i, j) column and walks the NXT planes, otherwise its threads stride over the
// nxt^3 cells; few, large CTAs: one CTA per plane or per 256 cells made CTA launch the bottleneck
template <typename R, int NXT>
__global__ void box_gather_kernel( const R *box, R *win, int npx, int npy, int npz, int nxt_rt, int nc )
{
   const int nxt = ( NXT > 0 ) ? NXT : nxt_rt;
   const int w = blockIdx.x, p = w / nc, v = w - p*nc;
   const int g = ( nxt - PS2 )/2, X = PS2*npx, Y = PS2*npy, Z = PS2*npz;
   const int px = p % npx, py = ( p / npx ) % npy, pz = p / ( npx*npy );
   const R *vol = box + (size_t)v*Z*( (size_t)Y*X );
   R *out = win + (size_t)w*( nxt*nxt*nxt );
   if ( NXT > 0 && (int)blockDim.x == NXT*NXT )
   {
      // one (i, j) column of the window per thread: x and y wrapped once, then the NXT planes
      const int i = threadIdx.x % NXT, j = threadIdx.x / NXT;
      const int x = wrap1( px*PS2 - g + i, X ), y = wrap1( py*PS2 - g + j, Y );
      const R *col = vol + (size_t)y*X + x;
#     pragma unroll 4
      for (int k = 0; k < NXT; k++)
      {
         const int z = wrap1( pz*PS2 - g + k, Z );
         out[( k*NXT + j )*NXT + i] = col[(size_t)z*Y*X];
      }
      return;
   }
   for (int t = threadIdx.x; t < nxt*nxt*nxt; t += blockDim.x)
   {
      const int k = t / ( nxt*nxt ), j = ( t / nxt ) % nxt, i = t % nxt;
      const int x = wrap1( px*PS2 - g + i, X ), y = wrap1( py*PS2 - g + j, Y ), z = wrap1( pz*PS2 - g + k, Z );
      out[t] = vol[( (size_t)z*Y + y )*X + x];
   }
}

template <typename R>
__global__ void box_scatter_kernel( const R *out, R *box, int npx, int npy, int npz, int nc )
{
   const int X = PS2*npx, Y = PS2*npy, Z = PS2*npz;
   const int t = blockIdx.x*blockDim.x + threadIdx.x;
   if ( t >= X*Y ) return;
   const int v = blockIdx.z;
   const int x = t % X, y = t / X;
   for (int z = blockIdx.y*PS2; z < blockIdx.y*PS2 + PS2; z++)
   {
      const int p = ( ( z/PS2 )*npy + y/PS2 )*npx + x/PS2;
      box[( (size_t)v*Z + z )*( (size_t)Y*X ) + t] = out[( (size_t)p*nc + v )*OUT3 + ( ( z%PS2 )*PS2 + y%PS2 )*PS2 + x%PS2];
   }
}

// adjoint of box_gather_kernel: every box cell sums the entries of all windows that contain it.
// Per axis, coordinate x (local offset r = x mod 16 in patch group q = x/16) appears in window q at
// i = r + g, in window q-1 at i = r + 16 + g when r < g, and in window q+1 at i = r - 16 + g when
// r >= 16 - g (neighbours taken periodically; with one or two groups per axis these are the same
// window at another index, which is also an image).  At most 3 images per axis.
GB_DEV int axis_images( int x, int np, int g, int *pp, int *ii )
{
   const int q = x / PS2, r = x - q*PS2;
   int n = 0;
   pp[n] = q;  ii[n] = r + g;  n++;
   if ( r < g )        { pp[n] = ( q == 0 ) ? np - 1 : q - 1;  ii[n] = r + PS2 + g;  n++; }
   if ( r >= PS2 - g ) { pp[n] = ( q == np - 1 ) ? 0 : q + 1;  ii[n] = r - PS2 + g;  n++; }
   return n;
}

__global__ void box_gather_adjoint_kernel( const double *wbar, double *boxbar, int npx, int npy, int npz, int nxt, int nc )
{
   const int X = PS2*npx, Y = PS2*npy, Z = PS2*npz;
   const int t = blockIdx.x*blockDim.x + threadIdx.x;
   if ( t >= X*Y ) return;
   const int v = blockIdx.z;
   const int x = t % X, y = t / X;
   const int g = ( nxt - PS2 )/2, n3 = nxt*nxt*nxt;
   int px[3], ix[3], py[3], iy[3], pz[3], iz[3];
   const int nx = axis_images( x, npx, g, px, ix );
   const int ny = axis_images( y, npy, g, py, iy );
   for (int z = blockIdx.y*PS2; z < blockIdx.y*PS2 + PS2; z++)
   {
      const int nz = axis_images( z, npz, g, pz, iz );
      double s = 0.0;
      for (int c=0; c<nz; c++)
      for (int b=0; b<ny; b++)
      for (int a=0; a<nx; a++)
      {
         const int p = ( pz[c]*npy + py[b] )*npx + px[a];
         s += wbar[( (size_t)p*nc + v )*n3 + ( iz[c]*nxt + iy[b] )*nxt + ix[a]];
      }
      boxbar[( (size_t)v*Z + z )*( (size_t)Y*X ) + t] = s;
   }
}

// adjoint of box_scatter_kernel (interiors): window outputs gather the box adjoint
__global__ void box_scatter_adjoint_kernel( const double *boxbar, double *outbar, int npx, int npy, int npz, int nc )
{
   const int X = PS2*npx, Y = PS2*npy, Z = PS2*npz;
   const int t = blockIdx.x*blockDim.x + threadIdx.x;
   if ( t >= X*Y ) return;
   const int v = blockIdx.z;
   const int x = t % X, y = t / X;
   for (int z = blockIdx.y*PS2; z < blockIdx.y*PS2 + PS2; z++)
   {
      const int p = ( ( z/PS2 )*npy + y/PS2 )*npx + x/PS2;
      outbar[( (size_t)p*nc + v )*OUT3 + ( ( z%PS2 )*PS2 + y%PS2 )*PS2 + x%PS2] = boxbar[( (size_t)v*Z + z )*( (size_t)Y*X ) + t];
   }
}

} // namespace gb

using namespace gb;

namespace {

// launch-shape limits of the box kernels: windows x ncomp in grid.x, one box plane (X*Y cells,
// 32-bit indices) per grid.x range, layers of 16 planes in grid.y, ncomp in grid.z
bool box_dims_ok( int npx, int npy, int npz, int nc, long long *nwin, long long *nplane )
{
   *nwin   = (long long)npx*npy*npz*nc;
   *nplane = (long long)PS2*npx*PS2*npy;
   return *nwin <= 0x7fffffffLL && *nplane <= 0x7fffffffLL - 256 && PS2*(long long)npz <= 65535 && nc <= 65535;
}

size_t adj_ws_bytes_pg( int rsize )
{
   return (size_t)6*ADJ_NC*ADJ_F3*rsize              // q
        + (size_t)( 3*ADJ_NC + 1 )*ADJ_F3            // tape + reset flags
        + (size_t)6*ADJ_NC*ADJ_F3*8                  // qbar
        + (size_t)2*ADJ_NC*ADJ_N3*8 + 256*6;         // wbar, uext, alignment slack
}

template <typename R, int P>
int adjoint_step_t( const gb_fluid_config &cfg, const void *flu_in, const double *gout, double *gin, int npg,
                    const gb_fluid_params *prm, void *ws, size_t ws_bytes, cudaStream_t st )
{
   // carve the workspace for as many patch groups as fit, then loop over chunks
   const size_t per = adj_ws_bytes_pg( sizeof(R) );
   const size_t fit = ws_bytes / per;
   if ( fit < 1 ) return GB_E_INVALID;
   const int chunk = ( fit > 65535 ) ? 65535 : (int)fit;     // patch groups of a chunk run along grid.y
   for (int p0 = 0; p0 < npg; p0 += chunk)
   {
      const int n = ( npg - p0 < chunk ) ? npg - p0 : chunk;
      char *w = (char*)ws;
      auto take = [&]( size_t bytes ) { char *r = w;  w += ( bytes + 255 ) & ~(size_t)255;  return r; };
      AdjArgs<R> a;
      memset( &a, 0, sizeof(a) );
      a.in   = (const R*)flu_in + (size_t)p0*ADJ_NC*ADJ_N3;
      a.gout = gout + (size_t)p0*ADJ_NC*OUT3;
      a.gin  = gin + (size_t)p0*ADJ_NC*ADJ_N3;
      a.q    = (R*)take( (size_t)n*6*ADJ_NC*ADJ_F3*sizeof(R) );
      a.tape = (uint8_t*)take( (size_t)n*( 3*ADJ_NC + 1 )*ADJ_F3 );
      a.qbar = (double*)take( (size_t)n*6*ADJ_NC*ADJ_F3*8 );
      a.wbar = (double*)take( (size_t)n*ADJ_NC*ADJ_N3*8 );
      a.uext = (double*)take( (size_t)n*ADJ_NC*ADJ_N3*8 );
      a.npg = n;
      a.coeff = (R)prm->minmod_coeff;
      a.ph.gamma = (R)cfg.gamma;  a.ph.gm1 = (R)( cfg.gamma - 1.0 );  a.ph.inv_gm1 = (R)( 1.0/( cfg.gamma - 1.0 ) );
      a.ph.min_dens = (R)prm->min_dens;  a.ph.min_pres = (R)prm->min_pres;  a.ph.min_eint = (R)prm->min_eint;
      a.ph.de_switch = (R)prm->dual_energy_switch;
      a.dt = (R)prm->dt;  a.dh = (R)prm->dh;
      if ( cudaMemsetAsync( a.qbar, 0, (size_t)n*6*ADJ_NC*ADJ_F3*8, st ) != cudaSuccess ) return GB_E_CUDA;
      if ( cudaMemsetAsync( a.wbar, 0, (size_t)n*ADJ_NC*ADJ_N3*8, st ) != cudaSuccess ) return GB_E_CUDA;
      if ( cudaMemsetAsync( a.uext, 0, (size_t)n*ADJ_NC*ADJ_N3*8, st ) != cudaSuccess ) return GB_E_CUDA;
      const int B = 256;
      const dim3 gf( ( ADJ_F3 + B - 1 )/B, n ), gr( ( 3*NFLX*PS2*PS2 + B - 1 )/B, n ), gc( ( ADJ_N3 + B - 1 )/B, n );
      adj_forward_kernel<R,P><<< gf, B, 0, st >>>( a );
      if ( cfg.rsolver == GB_RSOLVER_HLLC )
      {
         if constexpr ( sizeof(R) == 4 ) adj_face_kernel_hllc<R,P><<< gr, B, 0, st >>>( a );
         else                            adj_face_kernel<R,P,RS_HLLC><<< gr, B, 0, st >>>( a );
      }
      else if ( cfg.rsolver == GB_RSOLVER_HLLE )
         adj_face_kernel<R,P,RS_HLLE><<< gr, B, 0, st >>>( a );
      else if ( cfg.rsolver == GB_RSOLVER_EXACT )
         adj_face_kernel<R,P,RS_EXACT><<< gr, B, 0, st >>>( a );
      else
         adj_face_kernel<R,P,RS_ROE><<< gr, B, 0, st >>>( a );
      adj_cell_kernel<R,P><<< dim3( ( ADJ_F3 + B - 1 )/B, n ), B, 0, st >>>( a );
      adj_con2pri_kernel<R,P><<< gc, B, 0, st >>>( a );
      if ( cudaGetLastError() != cudaSuccess ) return GB_E_CUDA;
   }
   return GB_OK;
}

bool adjoint_supported( const gb_fluid_config &c, const gb_fluid_params *p )
{
   return c.scheme == GB_SCHEME_MHM && c.lr_scheme == GB_LR_PLM && c.dual_energy == GB_DE_NONE &&
          c.npassive_user == 0 && !p->jeans_min_pres && !c.char_reconstruction && c.flu_nxt == 20 && c.precision != GB_PREC_MIXED &&
          p->lr_limiter == GB_LIM_GMINMOD && p->minmod_coeff < 2.0 && p->minmod_maxiter == 0;
}

} // namespace

// the solver handle's configuration is needed here: read it through the public creation record
struct gb_fluid_solver;
extern "C" int gb_fluid_get_config( const gb_fluid_solver *s, gb_fluid_config *cfg );

extern "C" {

int gb_fluid_adjoint_workspace_bytes( const gb_fluid_solver *s, int npg, unsigned long long *bytes )
{
   gb_fluid_config c;
   if ( s == nullptr || bytes == nullptr || npg < 0 || gb_fluid_get_config( s, &c ) != GB_OK ) return GB_E_INVALID;
   *bytes = (unsigned long long)adj_ws_bytes_pg( ( c.precision == GB_PREC_FP64 ) ? 8 : 4 )*(unsigned long long)npg;
   return GB_OK;
}

int gb_fluid_adjoint_step_device( gb_fluid_solver *s, const void *flu_in, const double *gout, double *gin, int npg,
                                  const gb_fluid_params *prm, void *workspace, unsigned long long ws_bytes,
                                  void *stream )
{
   gb_fluid_config c;
   if ( s == nullptr || prm == nullptr || npg < 0 || gb_fluid_get_config( s, &c ) != GB_OK ) return GB_E_INVALID;
   if ( npg == 0 ) return GB_OK;
   if ( flu_in == nullptr || gout == nullptr || gin == nullptr || workspace == nullptr ) return GB_E_INVALID;
   if ( !( prm->dh > 0.0 ) || !( prm->dt >= 0.0 ) ) return GB_E_INVALID;
   if ( !adjoint_supported( c, prm ) ) return GB_E_UNSUPPORTED;
   if ( c.precision == GB_PREC_FP64 )
      return adjoint_step_t<double,P_FP64>( c, flu_in, gout, gin, npg, prm, workspace, ws_bytes, (cudaStream_t)stream );
   return adjoint_step_t<float,P_FP32>( c, flu_in, gout, gin, npg, prm, workspace, ws_bytes, (cudaStream_t)stream );
}

int gb_box_gather_device( const void *box, void *windows, int npx, int npy, int npz, int nxt, int ncomp,
                          int precision, void *stream )
{
   if ( box == nullptr || windows == nullptr || npx < 1 || npy < 1 || npz < 1 || ncomp < 1 ) return GB_E_INVALID;
   if ( nxt < PS2 || ( nxt - PS2 ) % 2 != 0 || ( nxt - PS2 )/2 > PS2 ) return GB_E_INVALID;
   long long nwin = 0, nplane = 0;
   if ( !box_dims_ok( npx, npy, npz, ncomp, &nwin, &nplane ) ) return GB_E_INVALID;
   cudaStream_t st = (cudaStream_t)stream;
   const dim3 grid( (unsigned)nwin );
   // compile-time widths: one thread per (i, j) column of a window; otherwise 256 threads over its cells
#  define GB_GATHER( R, N ) box_gather_kernel<R,N><<< grid, ( N > 0 ) ? N*N : 256, 0, st >>>( (const R*)box, (R*)windows, npx, npy, npz, nxt, ncomp )
   if ( precision == GB_PREC_FP64 )
   {
      if      ( nxt == 20 ) GB_GATHER( double, 20 );
      else if ( nxt == 22 ) GB_GATHER( double, 22 );
      else                  GB_GATHER( double, 0 );
   }
   else
   {
      if      ( nxt == 20 ) GB_GATHER( float, 20 );
      else if ( nxt == 22 ) GB_GATHER( float, 22 );
      else                  GB_GATHER( float, 0 );
   }
#  undef GB_GATHER
   return ( cudaGetLastError() == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

int gb_box_scatter_device( const void *pg_out, void *box, int npx, int npy, int npz, int ncomp, int precision,
                           void *stream )
{
   if ( box == nullptr || pg_out == nullptr || npx < 1 || npy < 1 || npz < 1 || ncomp < 1 ) return GB_E_INVALID;
   long long nwin = 0, nplane = 0;
   if ( !box_dims_ok( npx, npy, npz, ncomp, &nwin, &nplane ) ) return GB_E_INVALID;
   cudaStream_t st = (cudaStream_t)stream;
   const dim3 grid( (unsigned)( ( nplane + 255 )/256 ), npz, ncomp );
   if ( precision == GB_PREC_FP64 )
      box_scatter_kernel<double><<< grid, 256, 0, st >>>( (const double*)pg_out, (double*)box, npx, npy, npz, ncomp );
   else
      box_scatter_kernel<float><<< grid, 256, 0, st >>>( (const float*)pg_out, (float*)box, npx, npy, npz, ncomp );
   return ( cudaGetLastError() == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

int gb_box_gather_adjoint_device( const double *wbar, double *boxbar, int npx, int npy, int npz, int nxt, int ncomp,
                                  void *stream )
{
   if ( wbar == nullptr || boxbar == nullptr || npx < 1 || npy < 1 || npz < 1 || ncomp < 1 ) return GB_E_INVALID;
   if ( nxt < PS2 || ( nxt - PS2 ) % 2 != 0 || ( nxt - PS2 )/2 > PS2 ) return GB_E_INVALID;
   long long nwin = 0, nplane = 0;
   if ( !box_dims_ok( npx, npy, npz, ncomp, &nwin, &nplane ) ) return GB_E_INVALID;
   const dim3 grid( (unsigned)( ( nplane + 255 )/256 ), npz, ncomp );
   box_gather_adjoint_kernel<<< grid, 256, 0, (cudaStream_t)stream >>>( wbar, boxbar, npx, npy, npz, nxt, ncomp );
   return ( cudaGetLastError() == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

int gb_box_scatter_adjoint_device( const double *boxbar, double *outbar, int npx, int npy, int npz, int ncomp,
                                   void *stream )
{
   if ( boxbar == nullptr || outbar == nullptr || npx < 1 || npy < 1 || npz < 1 || ncomp < 1 ) return GB_E_INVALID;
   long long nwin = 0, nplane = 0;
   if ( !box_dims_ok( npx, npy, npz, ncomp, &nwin, &nplane ) ) return GB_E_INVALID;
   const dim3 grid( (unsigned)( ( nplane + 255 )/256 ), npz, ncomp );
   box_scatter_adjoint_kernel<<< grid, 256, 0, (cudaStream_t)stream >>>( boxbar, outbar, npx, npy, npz, ncomp );
   return ( cudaGetLastError() == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

} // extern "C"
