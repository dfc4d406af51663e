// Hand-written adjoint of one MHM + PLM step of a batch of patch groups (hydro, no dual energy).
//
// Forward map of one patch group (the reference: CPU_FluidSolver_MHM.cpp:265-589):
//   W = Con2Pri(U)                                   per input cell
//   w_f = PLM face values of W (per variable, limiter branch b)      per face-state cell, 6 faces
//   u_f = Pri2Con(w_f);  F_f = flux of (w_f, u_f)                     per face
//   q_f = u_f - dt/(2dh) * sum_d ( F_{2d+1} - F_{2d} )                 Hancock half step
//   Fhat = Riemann(q_{+d} of the left cell, q_{-d} of the right cell)  per cell face
//   U_out = U_in - dt/dh * sum_d ( Fhat_{+d} - Fhat_{-d} )
// Adjoint, given Ubar_out (d loss / d U_out):
//   A1 (forward recompute, tape): q_f of every face-state cell, and the limiter branch b of every
//      (cell, direction, variable) and the Hancock-reset flag, recorded for A3;
//   A2 (faces): Fbar = dt/dh (Ubar_out[right] - Ubar_out[left]); the Riemann Jacobians w.r.t. the
//      left and the right state are recomputed per face with forward-mode duals through the same
//      templated solver the forward kernel runs, giving qbar of the two face states;
//   A3 (cells): Hancock adjoint (accbar = -dt/(2dh) sum_f qbar_f), the Jacobians of Pri2Con and of
//      the face flux w.r.t. w_f (duals), and the PLM derivative of branch b (piecewise linear),
//      scattered to the 7-cell stencil of Wbar (double atomics);
//   A4 (cells): Ubar_in = J_Con2Pri^T Wbar + Ubar_out (interior) + reset contributions.
// Accumulations (qbar, Wbar, Ubar) are in double.  Floors are treated as inactive (smooth data),
// the limiter must be generalized MinMod with theta < 2 (no clamp acts), MinMod retries are off.
#pragma once
#include "hydro_physics.cuh"
#include "dual.cuh"

namespace gb {

// PLM-specific sizes (FLU_NXT = 20)
constexpr int ADJ_N   = 20;
constexpr int ADJ_N3  = ADJ_N*ADJ_N*ADJ_N;
constexpr int ADJ_F   = NFC;                 // 18 face-state cells per direction
constexpr int ADJ_F3  = ADJ_F*ADJ_F*ADJ_F;
constexpr int ADJ_NC  = 5;

// limiter branch codes of the generalized MinMod slope
enum { BR_ZERO = 0, BR_LEFT = 1, BR_RIGHT = 2, BR_CENTRAL = 3 };

// generalized MinMod slope and the branch that produced it (Hydro_LimitSlope, GMINMOD case)
template <typename R>
GB_DEV R gminmod_branch( R cl, R cc, R cr, R coeff, int &br )
{
   R sl = cc - cl, sr = cr - cc;
   const R sc = R(0.5)*( sl + sr );
   if ( !( sl*sr > R(0) ) ) { br = BR_ZERO; return R(0); }
   sl *= coeff;  sr *= coeff;
   R s = gabs( sl );  br = BR_LEFT;
   if ( gabs( sr ) < s ) { s = gabs( sr ); br = BR_RIGHT; }
   if ( gabs( sc ) < s ) { s = gabs( sc ); br = BR_CENTRAL; }
   return s*gsign( sc );
}

// dS/d(L,C,R) of branch br
template <typename R>
GB_DEV void gminmod_partials( int br, R coeff, R &dl, R &dc, R &dr )
{
   switch ( br )
   {
      case BR_LEFT:    dl = -coeff;  dc = coeff;   dr = R(0);    break;   // S = theta*(C-L)
      case BR_RIGHT:   dl = R(0);    dc = -coeff;  dr = coeff;   break;   // S = theta*(R-C)
      case BR_CENTRAL: dl = R(-0.5); dc = R(0);    dr = R(0.5);  break;   // S = (R-L)/2
      default:         dl = R(0);    dc = R(0);    dr = R(0);    break;
   }
}

template <typename R>
struct AdjArgs {
   const R *in;        // [npg][5][20^3] input windows
   const double *gout; // [npg][5][16^3] d loss / d U_out
   double *gin;        // [npg][5][20^3] d loss / d U_in (output)
   R       *q;         // [npg][6][5][18^3] forward face states (workspace)
   uint8_t *tape;      // [npg][3][5][18^3] limiter branches + [npg][18^3] reset flags (workspace)
   double  *qbar;      // [npg][6][5][18^3] (workspace)
   double  *wbar;      // [npg][5][20^3]    (workspace)
   double  *uext;      // [npg][5][20^3]    reset contributions (workspace)
   int      npg;
   R        coeff;
   Phys<R>  ph;
   R        dt, dh;
};

template <typename T, int M>
GB_DEV Phys< Dual<M,T> > dual_phys( const Phys<T> &p )
{
   Phys< Dual<M,T> > q;
   q.gamma = Dual<M,T>( (double)p.gamma );  q.gm1 = Dual<M,T>( (double)p.gm1 );
   q.inv_gm1 = Dual<M,T>( (double)p.inv_gm1 );
   q.min_dens = Dual<M,T>( (double)p.min_dens );  q.min_pres = Dual<M,T>( (double)p.min_pres );
   q.min_eint = Dual<M,T>( (double)p.min_eint );  q.de_switch = Dual<M,T>( (double)p.de_switch );
   return q;
}

} // namespace gb
