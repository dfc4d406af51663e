// Coarse-to-fine spatial interpolation of GAMER's AMR ghost-zone fill and refinement
// (Interpolate(), src/Interpolation/Interpolate.cpp:90-206, and its schemes Int_*.cpp), for a batch
// of independent interpolation regions of one shape, and the window assembly of the ghost-zone fill.
//
// The reference interpolates a region dimension by dimension: the x pass turns every coarse line of
// the region (plus CGhost layers in y and z) into pairs of fine values, the y pass does the same on
// the x-pass result, the z pass on the y-pass result, each pass into a temporary array.  A fine cell
// of coarse parent (i,j,k) therefore depends only on the (2*CGhost+1)^3 coarse cells around it, so here
// one thread owns one coarse cell and produces its 2x2x2 fine children directly: the x operator on
// the (2G+1)^2 lines through the neighbourhood, the y operator on their results, the z operator last
// -- the same operands and the same operations as the reference's passes, with no temporary arrays.
// INT_MINMOD1D (unsplit) takes the three limited slopes of the parent directly.
//
// Interpolate_Iterate (:208-560), the path GAMER's hydro ghost-zone fill takes for the conserved
// variables (src/Main/InterpolateGhostZone.cpp:1805), is built too: a parent whose eight children
// include an unphysical state (Hydro_IsUnphysical) is interpolated again, first in primitive variables
// (OPT__INT_PRIM), then with the monotonicity coefficient reduced MONO_MAX_ITER times; with the
// reference's INTERP_MASK (include/Macro.h:947) every parent iterates on its own, so this is again one
// thread per parent.  A parent still failing after the last iteration sets GB_INTERP_FAILED (the
// reference aborts the run there).
//
// Every multiplication, addition and division is written with explicitly rounded intrinsics, so the
// compiler contracts nothing into FMA and divides are IEEE: the results equal the reference CPU build
// bit for bit (in FP64 always; in FP32 as long as no intermediate is subnormal -- the device flushes
// those to zero).
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "gb_common.cuh"

namespace gb {
namespace {

// IntScheme_t (include/Typedef.h:171-180)
constexpr int INT_MINMOD3D = 1, INT_MINMOD1D = 2, INT_VANLEER = 3, INT_CQUAD = 4, INT_QUAD = 5, INT_CQUAR = 6,
              INT_QUAR = 7;

__host__ __device__ constexpr int int_ghost( int sch ) { return ( sch == INT_CQUAR || sch == INT_QUAR ) ? 2 : 1; }

// explicitly rounded arithmetic (never contracted into FMA)
GB_DEV float  radd( float a, float b )   { return __fadd_rn( a, b ); }
GB_DEV double radd( double a, double b ) { return __dadd_rn( a, b ); }
GB_DEV float  rsub( float a, float b )   { return __fsub_rn( a, b ); }
GB_DEV double rsub( double a, double b ) { return __dsub_rn( a, b ); }
GB_DEV float  rmul( float a, float b )   { return __fmul_rn( a, b ); }
GB_DEV double rmul( double a, double b ) { return __dmul_rn( a, b ); }
GB_DEV float  rdiv( float a, float b )   { return __fdiv_rn( a, b ); }
GB_DEV double rdiv( double a, double b ) { return __ddiv_rn( a, b ); }
GB_DEV float  rmin( float a, float b )   { return fminf( a, b ); }
GB_DEV double rmin( double a, double b ) { return fmin( a, b ); }
GB_DEV float  rmax( float a, float b )   { return fmaxf( a, b ); }
GB_DEV double rmax( double a, double b ) { return fmax( a, b ); }
GB_DEV float  rabs( float a )            { return fabsf( a ); }
GB_DEV double rabs( double a )           { return fabs( a ); }

template <typename R> GB_DEV R sign_of( R a ) { return ( a < R(0) ) ? R(-1) : R(+1); }   // SIGN (include/Macro.h:1178)

// the limited-slope fallback shared by the quadratic and quartic schemes: the centred slope
// 0.125*(R1 - L1) bounded by MonoCoeff/4 of each one-sided slope (Int_Quadratic.cpp, Int_Quartic.cpp)
template <typename R>
GB_DEV R mono_fallback( R L1, R R1, R ls, R rs, R mc4 )
{
   R s = rmul( R(0.125), rsub( R1, L1 ) );
   ls = rmul( ls, mc4 );
   rs = rmul( rs, mc4 );
   const R sg = sign_of( ls );
   s = rmul( s, sg );
   s = rmin( rmul( sg, ls ), s );
   s = rmin( rmul( sg, rs ), s );
   return rmul( s, sg );
}

// the conservative schemes' limiter on the half slope s (Int_CQuadratic.cpp, Int_CQuartic.cpp)
template <typename R>
GB_DEV R mono_conservative( R s, R ls, R rs, R coeff )
{
   const R sg = sign_of( ls );
   s  = rmul( s, sg );
   ls = rmul( ls, sg );
   rs = rmul( rs, sg );
   if ( ls < rs ) ls = rmul( ls, coeff );
   else           rs = rmul( rs, coeff );
   s = rmin( ls, s );
   s = rmin( rs, s );
   return rmul( s, sg );
}

// One dimension of a split scheme: the two fine children (lo, hi) of the centre c[G] of a line of
// 2G+1 coarse values.  coeff = the monotonicity coefficient of this iteration.
template <int SCH, typename R>
GB_DEV void op1d( const R *c, bool mono, R coeff, bool opp, R &lo, R &hi )
{
   constexpr int G = int_ghost( SCH );
   const R C = c[G], L1 = c[G-1], R1 = c[G+1];
   const bool flat = opp && rmul( L1, R1 ) < R(0);     // OppSign0thOrder
   if constexpr ( SCH == INT_MINMOD3D || SCH == INT_VANLEER )
   {
      const R ls = rsub( C, L1 ), rs = rsub( R1, C );
      R s;
      if ( rmul( rs, ls ) <= R(0) ) s = R(0);
      else if constexpr ( SCH == INT_MINMOD3D ) s = rmul( R(0.25), ( rabs( rs ) < rabs( ls ) ) ? rs : ls );
      else                                      s = rdiv( rmul( rmul( R(0.5), ls ), rs ), radd( ls, rs ) );
      if ( flat ) s = R(0);
      lo = rsub( C, s );  hi = radd( C, s );
   }
   else if constexpr ( SCH == INT_CQUAD || SCH == INT_CQUAR )
   {
      R s;
      if constexpr ( SCH == INT_CQUAD ) s = rmul( R(0.125), rsub( R1, L1 ) );
      else
      {
         const R L2 = c[0], R2 = c[4];
         s = radd( radd( radd( rmul( R(+3.0/128.0), L2 ), rmul( R(-22.0/128.0), L1 ) ), rmul( R(+22.0/128.0), R1 ) ),
                   rmul( R(-3.0/128.0), R2 ) );
      }
      if ( mono )
      {
         const R ls = rmul( R(0.25), rsub( C, L1 ) ), rs = rmul( R(0.25), rsub( R1, C ) );
         if ( rmul( ls, rs ) > R(0) )
         {
            if constexpr ( SCH == INT_CQUAR ) if ( rmul( s, ls ) < R(0) ) s = rmul( R(0.125), rsub( R1, L1 ) );
            s = mono_conservative( s, ls, rs, coeff );
         }
         else s = R(0);
      }
      if ( flat ) s = R(0);
      lo = rsub( C, s );  hi = radd( C, s );
   }
   else   // INT_QUAD / INT_QUAR: fixed-weight interpolation, limited where it over- or undershoots
   {
      if constexpr ( SCH == INT_QUAD )
      {
         lo = radd( radd( rmul( R(+5.0/32.0), L1 ), rmul( R(+30.0/32.0), C ) ), rmul( R(-3.0/32.0), R1 ) );
         hi = radd( radd( rmul( R(-3.0/32.0), L1 ), rmul( R(+30.0/32.0), C ) ), rmul( R(+5.0/32.0), R1 ) );
      }
      else
      {
         const R L2 = c[0], R2 = c[4];
         lo = radd( radd( radd( radd( rmul( R(-45.0/2048.0), L2 ), rmul( R(+420.0/2048.0), L1 ) ),
                                rmul( R(+1890.0/2048.0), C ) ), rmul( R(-252.0/2048.0), R1 ) ), rmul( R(+35.0/2048.0), R2 ) );
         hi = radd( radd( radd( radd( rmul( R(+35.0/2048.0), L2 ), rmul( R(-252.0/2048.0), L1 ) ),
                                rmul( R(+1890.0/2048.0), C ) ), rmul( R(+420.0/2048.0), R1 ) ), rmul( R(-45.0/2048.0), R2 ) );
      }
      if ( mono )
      {
         const R ls = rsub( C, L1 ), rs = rsub( R1, C );
         if ( rmul( ls, rs ) > R(0) )
         {
            const R cmax = ( ls > R(0) ) ? R1 : L1, cmin = ( ls > R(0) ) ? L1 : R1;
            bool over = rmax( lo, hi ) > cmax || rmin( lo, hi ) < cmin;
            if constexpr ( SCH == INT_QUAR ) over = over || rmul( rsub( hi, lo ), ls ) < R(0);
            if ( over )
            {
               const R s = mono_fallback( L1, R1, ls, rs, rmul( R(0.25), coeff ) );
               lo = rsub( C, s );  hi = radd( C, s );
            }
         }
         else { lo = C;  hi = C; }
      }
      if ( flat ) { lo = C;  hi = C; }
   }
}

// MinMod-1D limited slope of one direction (Int_MinMod1D.cpp)
template <typename R>
GB_DEV R minmod_slope( R L1, R C, R R1, bool opp )
{
   const R ls = rsub( C, L1 ), rs = rsub( R1, C );
   R s = ( rmul( rs, ls ) <= R(0) ) ? R(0) : rmul( R(0.25), ( rabs( rs ) < rabs( ls ) ) ? rs : ls );
   if ( opp && rmul( L1, R1 ) < R(0) ) s = R(0);
   return s;
}

template <typename R>
struct IntArgs {
   const R *cdata;            // [nbatch][ncomp][cz][cy][cx]
   R       *fdata;            // [nbatch][ncomp][fz][fy][fx]
   int      csize[3], cstart[3], crange[3], fsize[3], fstart[3];
   int      ncomp, nbatch;
   unsigned mono;             // bit v: Monotonic[v]
   R        mono_coeff;       // INT_MONO_COEFF
   int      opp;              // OppSign0thOrder
   // Interpolate_Iterate (hydro conserved variables, ncomp = 5)
   int      int_prim;         // OPT__INT_PRIM: second attempt in primitive variables
   int      mono_max_iter;    // MONO_MAX_ITER of ReduceMonoCoeff (0 = fixed coefficient)
   R        gm1, inv_gm1, min_pres;
   int     *status;           // GB_INTERP_FAILED is OR-ed in where a parent still fails
};

// value of variable v of coarse cell q, conserved or (prim) primitive as Hydro_Con2Pri computes it
// for Interpolate_Iterate (src/Interpolation/Interpolate.cpp:250-262; CPU_Shared_FluUtility.cpp:209-296)
template <typename R>
GB_DEV R coarse_value( const IntArgs<R> &a, const R *cb, size_t c3, int v, int q, bool prim )
{
   if ( !prim || v == 0 ) return cb[(size_t)v*c3 + q];
   const R d = cb[q];
   const R ird = rdiv( R(1), d );
   if ( v < 4 ) return rmul( cb[(size_t)v*c3 + q], ird );
   const R mx = cb[c3 + q], my = cb[2*c3 + q], mz = cb[3*c3 + q], e = cb[4*c3 + q];
   // Hydro_Con2Eint, EoS_DensEint2Pres_Gamma, Hydro_CheckMinPres
   const R eint = rsub( e, rdiv( rmul( R(0.5), radd( radd( rmul( mx, mx ), rmul( my, my ) ), rmul( mz, mz ) ) ), d ) );
   const R p = rmul( eint, a.gm1 );
   return ( p == p ) ? rmax( p, a.min_pres ) : p;
}

// the eight children f[fz][fy][fx] of coarse cell (i, j, k) of batch item cb, variable v
template <int SCH, typename R>
GB_DEV void children( const IntArgs<R> &a, const R *cb, size_t c3, int v, int i, int j, int k, bool prim, R coeff,
                      R (&f)[2][2][2] )
{
   const int cx = a.csize[0], cxy = a.csize[0]*a.csize[1];
   const bool mono = ( a.mono >> v ) & 1u, opp = a.opp != 0;
   if constexpr ( SCH == INT_MINMOD1D )
   {
      const int q = k*cxy + j*cx + i;
      const R C = coarse_value( a, cb, c3, v, q, prim );
      const R sx = minmod_slope( coarse_value( a, cb, c3, v, q - 1,   prim ), C, coarse_value( a, cb, c3, v, q + 1,   prim ), opp );
      const R sy = minmod_slope( coarse_value( a, cb, c3, v, q - cx,  prim ), C, coarse_value( a, cb, c3, v, q + cx,  prim ), opp );
      const R sz = minmod_slope( coarse_value( a, cb, c3, v, q - cxy, prim ), C, coarse_value( a, cb, c3, v, q + cxy, prim ), opp );
#     pragma unroll
      for (int fz=0; fz<2; fz++)
#     pragma unroll
      for (int fy=0; fy<2; fy++)
#     pragma unroll
      for (int fx=0; fx<2; fx++)
      {
         R t = fz ? radd( C, sz ) : rsub( C, sz );
         t = fy ? radd( t, sy ) : rsub( t, sy );
         f[fz][fy][fx] = fx ? radd( t, sx ) : rsub( t, sx );
      }
   }
   else
   {
      constexpr int G = int_ghost( SCH ), W = 2*G + 1;
      R tx[W][W][2];         // x pass: [z][y][fine x]
#     pragma unroll
      for (int zz=0; zz<W; zz++)
#     pragma unroll
      for (int yy=0; yy<W; yy++)
      {
         R line[W];
         const int q = ( k + zz - G )*cxy + ( j + yy - G )*cx + i;
#        pragma unroll
         for (int xx=0; xx<W; xx++) line[xx] = coarse_value( a, cb, c3, v, q + xx - G, prim );
         op1d<SCH>( line, mono, coeff, opp, tx[zz][yy][0], tx[zz][yy][1] );
      }
      R ty[W][2][2];         // y pass: [z][fine y][fine x]
#     pragma unroll
      for (int zz=0; zz<W; zz++)
#     pragma unroll
      for (int fx=0; fx<2; fx++)
      {
         R line[W];
#        pragma unroll
         for (int yy=0; yy<W; yy++) line[yy] = tx[zz][yy][fx];
         op1d<SCH>( line, mono, coeff, opp, ty[zz][0][fx], ty[zz][1][fx] );
      }
#     pragma unroll
      for (int fy=0; fy<2; fy++)
#     pragma unroll
      for (int fx=0; fx<2; fx++)
      {
         R line[W];
#        pragma unroll
         for (int zz=0; zz<W; zz++) line[zz] = ty[zz][fy][fx];
         op1d<SCH>( line, mono, coeff, opp, f[0][fy][fx], f[1][fy][fx] );
      }
   }
}

// Interpolate(): every variable of every parent of the range, the fixed coefficient
template <int SCH, typename R>
__global__ void interp_kernel( const __grid_constant__ IntArgs<R> a )
{
   const int nx = a.crange[0], nxy = a.crange[0]*a.crange[1], ncell = nxy*a.crange[2];
   const size_t c3 = (size_t)a.csize[0]*a.csize[1]*a.csize[2], f3 = (size_t)a.fsize[0]*a.fsize[1]*a.fsize[2];
   for (long long t = blockIdx.x*(long long)blockDim.x + threadIdx.x; t < (long long)ncell*a.nbatch*a.ncomp;
        t += (long long)gridDim.x*blockDim.x)
   {
      const int c = (int)( t % ncell );
      const long long bv = t / ncell;
      const int v = (int)( bv % a.ncomp ), b = (int)( bv / a.ncomp );
      const int ii = c % nx, jj = ( c / nx ) % a.crange[1], kk = c / nxy;
      const R *cb = a.cdata + (size_t)b*a.ncomp*c3;
      R f[2][2][2];
      children<SCH>( a, cb, c3, v, a.cstart[0] + ii, a.cstart[1] + jj, a.cstart[2] + kk, false, a.mono_coeff, f );
      R *fb = a.fdata + ( (size_t)b*a.ncomp + v )*f3;
#     pragma unroll
      for (int fz=0; fz<2; fz++)
#     pragma unroll
      for (int fy=0; fy<2; fy++)
#     pragma unroll
      for (int fx=0; fx<2; fx++)
         fb[(size_t)( a.fstart[2] + 2*kk + fz )*a.fsize[0]*a.fsize[1] + ( a.fstart[1] + 2*jj + fy )*a.fsize[0] +
            ( a.fstart[0] + 2*ii + fx )] = f[fz][fy][fx];
   }
}

// Hydro_IsUnphysical of an interpolated child (src/Model_Hydro/CPU_Hydro/CPU_Shared_FluUtility.cpp:843-1010):
// conserved (with the internal-energy test) or primitive (then with the internal energy P/(gamma-1)
// of Interpolate_Iterate :399-430)
template <typename R>
GB_DEV bool child_fails( const IntArgs<R> &a, const R (&u)[5], bool prim )
{
   bool bad = false;
#  pragma unroll
   for (int v=0; v<5; v++)
   {
      bad |= ( u[v] != u[v] );
      if ( v >= 1 && v <= 3 ) bad |= ( u[v] < -Lim<R>::huge() || u[v] > Lim<R>::huge() );
      else if ( prim && v == 4 ) bad |= ( u[v] < R(0) || u[v] > Lim<R>::huge() );
      else                       bad |= ( u[v] <= R(0) || u[v] > Lim<R>::huge() );
   }
   if ( prim )
   {
      const R eint = rmul( u[4], a.inv_gm1 );
      bad |= ( eint < R(0) || eint > Lim<R>::huge() || eint != eint );
   }
   else
   {
      const R eint = rsub( u[4], rdiv( rmul( R(0.5), radd( radd( rmul( u[1], u[1] ), rmul( u[2], u[2] ) ), rmul( u[3], u[3] ) ) ), u[0] ) );
      bad |= ( eint < rmul( rmul( R(-3.0), u[4] ), Lim<R>::eps() ) || eint > Lim<R>::huge() || eint != eint );
   }
   return bad;
}

// Interpolate_Iterate for the five conserved hydro variables (INTERP_MASK: each parent on its own)
template <int SCH, typename R>
__global__ void interp_iterate_kernel( const __grid_constant__ IntArgs<R> a )
{
   const int nx = a.crange[0], nxy = a.crange[0]*a.crange[1], ncell = nxy*a.crange[2];
   const size_t c3 = (size_t)a.csize[0]*a.csize[1]*a.csize[2], f3 = (size_t)a.fsize[0]*a.fsize[1]*a.fsize[2];
   const int mono_iter = a.mono_max_iter;
   const int max_iter = a.int_prim ? mono_iter + 1 : mono_iter;
   for (long long t = blockIdx.x*(long long)blockDim.x + threadIdx.x; t < (long long)ncell*a.nbatch;
        t += (long long)gridDim.x*blockDim.x)
   {
      const int c = (int)( t % ncell ), b = (int)( t / ncell );
      const int ii = c % nx, jj = ( c / nx ) % a.crange[1], kk = c / nxy;
      const int i = a.cstart[0] + ii, j = a.cstart[1] + jj, k = a.cstart[2] + kk;
      const R *cb = a.cdata + (size_t)b*5*c3;
      R f[5][2][2][2];
      bool prim = false, ok = false;
      R coeff = a.mono_coeff;
      for (int it = 0; it <= max_iter && !ok; it++)
      {
         if ( it == 1 && a.int_prim ) prim = true;
         else if ( it >= 1 ) coeff = rmax( rsub( coeff, rdiv( a.mono_coeff, (R)mono_iter ) ), R(0) );
         // one variable at a time (the children of all five are kept for the checks)
#        pragma unroll 1
         for (int v=0; v<5; v++) children<SCH>( a, cb, c3, v, i, j, k, prim, coeff, f[v] );
         ok = true;
#        pragma unroll
         for (int q=0; q<8; q++)
         {
            R u[5];
#           pragma unroll
            for (int v=0; v<5; v++) u[v] = f[v][q >> 2][( q >> 1 ) & 1][q & 1];
            ok &= !child_fails( a, u, prim );
         }
      }
      if ( !ok ) atomicOr( a.status, GB_INTERP_FAILED );
      R *fb = a.fdata + (size_t)b*5*f3;
#     pragma unroll
      for (int q=0; q<8; q++)
      {
         const int fz = q >> 2, fy = ( q >> 1 ) & 1, fx = q & 1;
         R u[5];
#        pragma unroll
         for (int v=0; v<5; v++) u[v] = f[v][fz][fy][fx];
         if ( prim )
         {
            // Hydro_Pri2Con: momenta rho*v, E = 1/2 |m|^2/rho + P/(gamma-1) (Hydro_ConEint2Etot)
            const R d = u[0];
            u[1] = rmul( d, u[1] );  u[2] = rmul( d, u[2] );  u[3] = rmul( d, u[3] );
            const R eint = rmul( u[4], a.inv_gm1 );
            u[4] = radd( rdiv( rmul( R(0.5), radd( radd( rmul( u[1], u[1] ), rmul( u[2], u[2] ) ), rmul( u[3], u[3] ) ) ), d ), eint );
         }
         const size_t o = (size_t)( a.fstart[2] + 2*kk + fz )*a.fsize[0]*a.fsize[1] + ( a.fstart[1] + 2*jj + fy )*a.fsize[0] +
                          ( a.fstart[0] + 2*ii + fx );
#        pragma unroll
         for (int v=0; v<5; v++) fb[(size_t)v*f3 + o] = u[v];
      }
   }
}

template <typename R>
cudaError_t interp_launch( int scheme, bool iterate, const IntArgs<R> &a, cudaStream_t st )
{
   const long long ncell = (long long)a.crange[0]*a.crange[1]*a.crange[2];
   const long long items = ncell*a.nbatch*( iterate ? 1 : a.ncomp );
   constexpr int B = 128;
   long long g = ( items + B - 1 )/B;
   int dev = 0, nsm = 148;
   cudaGetDevice( &dev );
   cudaDeviceGetAttribute( &nsm, cudaDevAttrMultiProcessorCount, dev );
   if ( g > 32LL*nsm ) g = 32LL*nsm;
   if ( g < 1 ) return cudaSuccess;
#  define GB_INT_CASE( S ) \
   case S: if ( iterate ) interp_iterate_kernel<S,R><<< (unsigned)g, B, 0, st >>>( a ); \
           else           interp_kernel<S,R><<< (unsigned)g, B, 0, st >>>( a ); break;
   switch ( scheme )
   {
      GB_INT_CASE( INT_MINMOD3D )
      GB_INT_CASE( INT_MINMOD1D )
      GB_INT_CASE( INT_VANLEER )
      GB_INT_CASE( INT_CQUAD )
      GB_INT_CASE( INT_QUAD )
      GB_INT_CASE( INT_CQUAR )
      GB_INT_CASE( INT_QUAR )
      default: return cudaErrorInvalidValue;
   }
#  undef GB_INT_CASE
   return cudaGetLastError();
}

template <typename R>
int interp_run( const gb_interp_params *p, const void *cdata, void *fdata, int nbatch, cudaStream_t st )
{
   IntArgs<R> a;
   a.cdata = (const R*)cdata;  a.fdata = (R*)fdata;
   for (int d=0; d<3; d++)
   {
      a.csize[d] = p->csize[d];  a.cstart[d] = p->cstart[d];  a.crange[d] = p->crange[d];
      a.fsize[d] = p->fsize[d];  a.fstart[d] = p->fstart[d];
   }
   a.ncomp = p->ncomp;  a.nbatch = nbatch;
   a.mono = p->monotonic;  a.mono_coeff = (R)p->mono_coeff;  a.opp = p->opp_sign_0th_order;
   a.int_prim = p->int_prim;  a.mono_max_iter = p->mono_max_iter;
   // EoS_SetAuxArray_Gamma: constants formed in double, then cast
   a.gm1 = (R)( p->gamma - 1.0 );  a.inv_gm1 = (R)( 1.0/( p->gamma - 1.0 ) );  a.min_pres = (R)p->min_pres;
   a.status = p->status;
   // Interpolate() takes the iterative path only with IntPrim or ReduceMonoCoeff (Interpolate.cpp:152-156)
   const bool iterate = ( p->mode == GB_INTERP_ITERATE ) && ( p->int_prim || p->mono_max_iter > 0 );
   const cudaError_t e = interp_launch<R>( p->scheme, iterate, a, st );
   return ( e == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

// ---- window assembly of the ghost-zone fill ------------------------------------------------------
// Prepare_PatchData (src/Main/Prepare_PatchData.cpp) fills each side of a patch group's window from
// the patch groups of the same level where they exist and by interpolation from the coarser level
// where they do not (InterpolateGhostZone).  Here: one thread per window cell and variable; the side
// of the cell picks its source -- the patch group's own interior, the interior of the same-level patch
// group nbr[p][s], or the coarse-interpolated window cint[p] (gb_interpolate_device over the window).
template <typename R>
__global__ void assemble_windows_kernel( const R *fine, const int *nbr, const R *cint, R *win, int npg, int ncomp,
                                         int nxt )
{
   const int g = ( nxt - PS2 )/2, n3 = nxt*nxt*nxt;
   const long long total = (long long)npg*ncomp*n3;
   for (long long t = blockIdx.x*(long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x*blockDim.x)
   {
      const int c = (int)( t % n3 );
      const long long pv = t / n3;
      const int v = (int)( pv % ncomp ), p = (int)( pv / ncomp );
      const int i = c % nxt, j = ( c / nxt ) % nxt, k = c / ( nxt*nxt );
      int x = i - g, y = j - g, z = k - g;
      const int dx = ( x < 0 ) ? -1 : ( x >= PS2 ), dy = ( y < 0 ) ? -1 : ( y >= PS2 ), dz = ( z < 0 ) ? -1 : ( z >= PS2 );
      int src = p;
      if ( dx | dy | dz )
      {
         src = nbr[p*27 + ( dz + 1 )*9 + ( dy + 1 )*3 + ( dx + 1 )];
         x -= PS2*dx;  y -= PS2*dy;  z -= PS2*dz;
      }
      R val;
      if ( src >= npg ) val = R(NAN);    // not a patch group of the batch
      else if ( src >= 0 ) val = fine[( (size_t)src*ncomp + v )*PS2*PS2*PS2 + ( z*PS2 + y )*PS2 + x];
      else if ( cint )     val = cint[( (size_t)p*ncomp + v )*n3 + c];
      else                 val = R(NAN);  // a coarse side without an interpolated window
      win[( (size_t)p*ncomp + v )*n3 + c] = val;
   }
}

} // namespace
} // namespace gb

extern "C"
int gb_interpolate_device( const gb_interp_params *p, const void *cdata, void *fdata, int nbatch, void *stream )
{
   using namespace gb;
   if ( p == nullptr || nbatch < 0 ) return GB_E_INVALID;
   if ( nbatch == 0 ) return GB_OK;
   if ( cdata == nullptr || fdata == nullptr ) return GB_E_INVALID;
   if ( p->scheme < INT_MINMOD3D || p->scheme > INT_QUAR ) return ( p->scheme == 8 ) ? GB_E_UNSUPPORTED : GB_E_INVALID;
   if ( p->precision != GB_PREC_FP32 && p->precision != GB_PREC_FP64 ) return GB_E_INVALID;
   if ( p->ncomp < 1 || p->ncomp > 32 ) return GB_E_INVALID;
   if ( p->mode != GB_INTERP_PLAIN && p->mode != GB_INTERP_ITERATE ) return GB_E_INVALID;
   // the region the reference's Interpolate() accepts (Interpolate.cpp:104-117): CGhost coarse cells
   // around the range inside CData, the 2x finer range inside FData
   const int G = int_ghost( p->scheme );
   long long c3 = 1, f3 = 1;
   for (int d=0; d<3; d++)
   {
      if ( p->csize[d] < 1 || p->fsize[d] < 1 || p->crange[d] < 1 ) return GB_E_INVALID;
      if ( p->cstart[d] < G || p->cstart[d] + p->crange[d] > p->csize[d] - G ) return GB_E_INVALID;
      if ( p->fstart[d] < 0 || p->fstart[d] + 2*p->crange[d] > p->fsize[d] ) return GB_E_INVALID;
      c3 *= p->csize[d];  f3 *= p->fsize[d];
   }
   if ( c3*p->ncomp*nbatch > 0x7fffffffLL*8 || f3*p->ncomp*nbatch > 0x7fffffffLL*8 ) return GB_E_INVALID;
   if ( p->mode == GB_INTERP_ITERATE )
   {
      // Interpolate_Iterate: all five conserved hydro variables, the fine region from the origin
      // (Interpolate.cpp:218-220), a positive gamma - 1, the failure flag; the reference refuses to
      // reduce the coefficient of MinMod-3D/1D and vanLeer (:273-276)
      if ( p->ncomp != 5 || p->status == nullptr || !( p->gamma > 1.0 ) || p->mono_max_iter < 0 ) return GB_E_INVALID;
      if ( p->fstart[0] || p->fstart[1] || p->fstart[2] ) return GB_E_INVALID;
      if ( p->mono_max_iter > 0 && ( p->scheme == INT_MINMOD3D || p->scheme == INT_MINMOD1D || p->scheme == INT_VANLEER ) )
         return GB_E_INVALID;
   }
   if ( p->precision == GB_PREC_FP64 ) return interp_run<double>( p, cdata, fdata, nbatch, (cudaStream_t)stream );
   return interp_run<float>( p, cdata, fdata, nbatch, (cudaStream_t)stream );
}

extern "C"
int gb_assemble_windows_device( const void *fine, const int *nbr, const void *cint, void *windows, int npg, int ncomp,
                                int nxt, int precision, void *stream )
{
   using namespace gb;
   if ( npg < 0 || ncomp < 1 || nxt < PS2 + 2 || nxt > PS2 + 2*PS2 || ( nxt - PS2 ) % 2 != 0 ) return GB_E_INVALID;
   if ( precision != GB_PREC_FP32 && precision != GB_PREC_FP64 ) return GB_E_INVALID;
   if ( npg == 0 ) return GB_OK;
   if ( fine == nullptr || nbr == nullptr || windows == nullptr ) return GB_E_INVALID;
   const long long total = (long long)npg*ncomp*nxt*nxt*nxt;
   constexpr int B = 256;
   int dev = 0, nsm = 148;
   cudaGetDevice( &dev );
   cudaDeviceGetAttribute( &nsm, cudaDevAttrMultiProcessorCount, dev );
   long long g = ( total + B - 1 )/B;
   if ( g > 16LL*nsm ) g = 16LL*nsm;
   cudaStream_t st = (cudaStream_t)stream;
   if ( precision == GB_PREC_FP64 )
      assemble_windows_kernel<double><<< (unsigned)g, B, 0, st >>>( (const double*)fine, nbr, (const double*)cint,
                                                                    (double*)windows, npg, ncomp, nxt );
   else
      assemble_windows_kernel<float><<< (unsigned)g, B, 0, st >>>( (const float*)fine, nbr, (const float*)cint,
                                                                   (float*)windows, npg, ncomp, nxt );
   return ( cudaGetLastError() == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}
