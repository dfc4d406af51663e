// Forward-mode dual numbers: a value and M tangents.  Instantiating the templated device routines
// of hydro_physics.cuh with Dual<M,T> gives their Jacobian columns in one evaluation, with every
// branch decided by the value part exactly as in the plain evaluation.
#pragma once
#include "gb_common.cuh"
#include "hydro_physics.cuh"

namespace gb {

template <int M, typename T>
struct Dual {
   T v;
   T d[M];

   __device__ __forceinline__ Dual() {}
   __device__ __forceinline__ Dual( double x ) : v( (T)x ) {
#     pragma unroll
      for (int k=0; k<M; k++) d[k] = T(0);
   }
   __device__ __forceinline__ explicit operator T() const { return v; }
   static __device__ __forceinline__ Dual var( T x, int k ) {
      Dual r( 0.0 );  r.v = x;
#     pragma unroll
      for (int q=0; q<M; q++) r.d[q] = ( q == k ) ? T(1) : T(0);
      return r;
   }
};

#define GB_DUAL_TPL template <int M, typename T>
#define GB_D Dual<M,T>

GB_DUAL_TPL GB_DEV GB_D operator+( const GB_D &a, const GB_D &b ) {
   GB_D r;  r.v = a.v + b.v;
#  pragma unroll
   for (int k=0; k<M; k++) r.d[k] = a.d[k] + b.d[k];
   return r;
}
GB_DUAL_TPL GB_DEV GB_D operator-( const GB_D &a, const GB_D &b ) {
   GB_D r;  r.v = a.v - b.v;
#  pragma unroll
   for (int k=0; k<M; k++) r.d[k] = a.d[k] - b.d[k];
   return r;
}
GB_DUAL_TPL GB_DEV GB_D operator+( const GB_D &a ) { return a; }
GB_DUAL_TPL GB_DEV GB_D operator-( const GB_D &a ) {
   GB_D r;  r.v = -a.v;
#  pragma unroll
   for (int k=0; k<M; k++) r.d[k] = -a.d[k];
   return r;
}
GB_DUAL_TPL GB_DEV GB_D operator*( const GB_D &a, const GB_D &b ) {
   GB_D r;  r.v = a.v*b.v;
#  pragma unroll
   for (int k=0; k<M; k++) r.d[k] = a.d[k]*b.v + a.v*b.d[k];
   return r;
}
GB_DUAL_TPL GB_DEV GB_D operator/( const GB_D &a, const GB_D &b ) {
   GB_D r;  const T ib = T(1)/b.v;  r.v = a.v*ib;
#  pragma unroll
   for (int k=0; k<M; k++) r.d[k] = ( a.d[k] - r.v*b.d[k] )*ib;
   return r;
}
GB_DUAL_TPL GB_DEV GB_D &operator+=( GB_D &a, const GB_D &b ) { a = a + b; return a; }
GB_DUAL_TPL GB_DEV GB_D &operator-=( GB_D &a, const GB_D &b ) { a = a - b; return a; }
GB_DUAL_TPL GB_DEV GB_D &operator*=( GB_D &a, const GB_D &b ) { a = a * b; return a; }

GB_DUAL_TPL GB_DEV bool operator< ( const GB_D &a, const GB_D &b ) { return a.v <  b.v; }
GB_DUAL_TPL GB_DEV bool operator> ( const GB_D &a, const GB_D &b ) { return a.v >  b.v; }
GB_DUAL_TPL GB_DEV bool operator<=( const GB_D &a, const GB_D &b ) { return a.v <= b.v; }
GB_DUAL_TPL GB_DEV bool operator>=( const GB_D &a, const GB_D &b ) { return a.v >= b.v; }
GB_DUAL_TPL GB_DEV bool operator==( const GB_D &a, const GB_D &b ) { return a.v == b.v; }
GB_DUAL_TPL GB_DEV bool operator!=( const GB_D &a, const GB_D &b ) { return a.v != b.v; }

GB_DUAL_TPL GB_DEV GB_D gsqrt( const GB_D &a ) {
   GB_D r;  r.v = gsqrt( a.v );
   const T h = ( r.v > T(0) ) ? T(0.5)/r.v : T(0);
#  pragma unroll
   for (int k=0; k<M; k++) r.d[k] = a.d[k]*h;
   return r;
}
GB_DUAL_TPL GB_DEV GB_D gabs( const GB_D &a ) { return ( a.v < T(0) ) ? -a : a; }
GB_DUAL_TPL GB_DEV GB_D gmin( const GB_D &a, const GB_D &b ) { return ( b.v < a.v ) ? b : a; }
GB_DUAL_TPL GB_DEV GB_D gmax( const GB_D &a, const GB_D &b ) { return ( b.v > a.v ) ? b : a; }
GB_DUAL_TPL GB_DEV GB_D gpow( const GB_D &a, const GB_D &b ) {
   // exponent is a constant in every use (gamma - 1)
   GB_D r;  r.v = gpow( a.v, b.v );
   const T dv = ( a.v != T(0) ) ? b.v*r.v/a.v : T(0);
#  pragma unroll
   for (int k=0; k<M; k++) r.d[k] = a.d[k]*dv;
   return r;
}

template <int M, typename T> struct ScalarOf< Dual<M,T> > { typedef T type;  static constexpr bool dual = true;  static constexpr int ntan = M; };

// the value parts of the EoS and floor parameters
template <int M, typename T>
GB_DEV Phys<T> value_phys( const Phys< Dual<M,T> > &p )
{
   Phys<T> q;
   q.gamma = p.gamma.v;  q.gm1 = p.gm1.v;  q.inv_gm1 = p.inv_gm1.v;
   q.min_dens = p.min_dens.v;  q.min_pres = p.min_pres.v;  q.min_eint = p.min_eint.v;
   q.de_switch = p.de_switch.v;  q.jeans_coeff = p.jeans_coeff.v;  q.jeans = p.jeans;
   q.frac_mask = p.frac_mask;  q.pfloor = p.pfloor;
   return q;
}

template <int M, typename T> struct Lim< Dual<M,T> > {
   static GB_DEV Dual<M,T> tiny() { return Dual<M,T>( (double)Lim<T>::tiny() ); }
   static GB_DEV Dual<M,T> huge() { return Dual<M,T>( (double)Lim<T>::huge() ); }
   static GB_DEV Dual<M,T> eps()  { return Dual<M,T>( (double)Lim<T>::eps() ); }
};

#undef GB_DUAL_TPL
#undef GB_D

} // namespace gb
