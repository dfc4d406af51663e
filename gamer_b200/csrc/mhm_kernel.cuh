// Fused MHM patch-group kernel (hydro, PLM or PPM, HLLC / HLLE / Roe), one CTA per patch group.
//
// Reference path replaced: CUFLU_FluidSolver_MHM (src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_MHM.cpp:265-589),
// which runs Con2Pri -> data reconstruction -> Riemann fluxes -> full-step update as separate passes
// over a whole patch group with ~2 MB of global-memory scratch per group.
//
// Here a CTA sweeps its patch group plane by plane along z and keeps every intermediate on chip.
// Two CTA-wide phases per plane, each ended by one barrier:
//   (A) face states of fc plane kf (PLM/PPM + Hancock half step) for the 16x16 interior cells and
//       the 4x16 halo cells of the x/y faces; x/y face states go to shared memory.  The thread of
//       interior column (i,j) keeps its cell's z face states in registers, so it also solves the
//       z Riemann problem between planes kf-1 and kf from registers, and finishes output cell
//       (i,j) of plane o = kf-2 as soon as that z flux exists:
//          U_out = U_in - dt/dh * ( (dFx + dFy) + dFz ),
//       the summation order of Hydro_FullStepUpdate (CPU_Shared_FullStepUpdate.cpp:105-117), with
//       the x/y fluxes of plane kf-1 from phase (B) of the previous step;
//   (B) the x (17x16) and y (16x17) Riemann problems of plane kf into a double-buffered flux plane,
//       and the conversion of the next input plane to primitive variables.
// Input planes arrive by 1-D bulk copies (cp.async.bulk, TMA) into a ring of plane slots, two planes
// ahead of use (one for PPM, which forms its limited slopes where it uses them).
// Global traffic per patch group: the input once, the output once, the 9 flux planes once.
//
// Index conventions (scheme-minimal input width N = 16 + 2*(NG+1), NG = LR ghost width):
//   cc  : input cell index in [0, N)          (an input wider than N is offset by s = (nin-N)/2)
//   fc  : face-state cell index in [0, 18),   fc = cc - NG
//   out : output cell index in [0, 16),       out = fc - 1
//   flux: x-flux i in [0,17) is the +x face of fc cell (i, j+1, k+1)  (NSkip_N = 0, NSkip_T = 1,
//         CPU_Shared_ComputeFlux.cpp:203-220)
#pragma once
#include <type_traits>
#include "hydro_physics.cuh"
#include "hydro_pair.cuh"
#include "tma.cuh"

namespace gb {

constexpr int GB_MAX_LEVEL = 16;

template <typename R>
struct MhmArgs {
   const R *in;          // [npg][NC][nin^3]  (MHM_RP: the half-step primitive state [npg][NC][20^3])
   const R *uin;         // MHM_RP only: the conserved input [npg][NC][22^3] of the full-step update
   R       *out;         // [npg][NC][16^3]
   R       *flux;        // [npg][9][NC][16^2]  (nullptr: do not store)
   char    *de;          // [npg][16^3]         (dual energy only; nullptr: do not store)
   int     *pg_fail;     // [npg]               (nullptr: do not store) 1 = unphysical after all retries
   int     *status;      // one status word, GB_ST_* bits OR-ed in
   int      npg, nin;
   int      limiter, minmod_maxiter;
   R        minmod_coeff;
   Phys<R>  ph;
   int      nlevel;
   int      level_start[GB_MAX_LEVEL + 1];   // patch-group ranges of each level (batched launches)
   R        dt[GB_MAX_LEVEL], dh[GB_MAX_LEVEL];
   int      nnorm;                           // NormPassive: number of listed passive scalars (0 = off)
   int      norm_idx[4];                     // NormIdx (passive indices, no repeats)
};

// shared-memory carve-up (byte offsets), identical on host and device
struct MhmLayout {
   int bar, pri, fcx, fcy, flx, fly, car, flag, total;
};

__host__ __device__ inline int gb_align16( int x ) { return ( x + 15 ) & ~15; }

// The float policies' PLM with 5 or 6 variables (the headline family) convert the next plane to
// primitive variables in phase A, on the threads that own no interior column (the 64 ring cells of
// a 320-thread CTA leave those with time to spare), instead of in phase B after the x/y Riemann
// problems, where it made the slowest threads do both; the plane then has to arrive one phase
// earlier, so the ring fetches three planes ahead (one more slot, two CTAs per SM still fit).
__host__ __device__ constexpr bool mhm_conv_in_a( int p, int lr, int nc, int sch )
{
   return ( p == P_FP32 || p == P_MIXED ) && lr == LR_PLM && nc <= 6 && sch == 0;
}

// plane ring depth: PLM keeps 3 live primitive planes, PPM 4, plus the planes in flight (one, or two
// when the next plane is converted in phase A)
__host__ __device__ constexpr int mhm_nslot( int lr, bool conv_a = false ) { return ( lr == LR_PPM ) ? 5 : ( conv_a ? 5 : 4 ); }

// PPM ("lean"): every limited slope is formed where it is used from the primitive planes instead
// of from slope planes; the ring then holds 5 live planes (centre +-2 for the z slopes) and the
// next plane is fetched one step ahead instead of two.  In FP64 the slope planes would not fit one
// SM's shared memory; in float, without them (and with float flux planes) two CTAs of 320 threads
// share an SM: PPM+Roe mixed 3.41 -> 2.40 ms, PPM+HLLC FP32 2.87 -> 2.06 ms at 4096 patch groups.
__host__ __device__ constexpr bool mhm_lean( int rsz, int lr ) { return lr == LR_PPM; }

// rsz / asz / fsz: bytes of the storage type, of the accumulation type and of the x/y flux planes
// (the mixed policy keeps them in double, so that each flux is converted once, where two CTAs
// still fit an SM: PLM without passive scalars).
// carry_smem: the per-column z state (upper z face of the previous fc plane, z flux below it) is
// kept in shared memory instead of registers (the mixed policy, whose double accumulation leaves
// no registers for it at two CTAs per SM)
__host__ __device__ inline MhmLayout mhm_layout( int rsz, int asz, int fsz, int nc, int nin, int lr, bool carry_smem,
                                                 bool conv_a = false )
{
   MhmLayout L;
   int o = 0;
   L.bar  = o;  o += 64;
   L.pri  = o;  o = gb_align16( o + mhm_nslot( lr, conv_a )*nc*nin*nin*rsz );
   L.fcx  = o;  o = gb_align16( o + 2*nc*PS2*NFC*rsz );
   L.fcy  = o;  o = gb_align16( o + 2*nc*NFC*PS2*rsz );
   L.flx  = o;  o = gb_align16( o + nc*PS2*NFLX*fsz );
   L.fly  = o;  o = gb_align16( o + nc*NFLX*PS2*fsz );
   L.car  = o;  o = gb_align16( o + ( carry_smem ? nc*PS2*PS2*( rsz + asz ) : 0 ) );
   L.flag = o;  o += 16;
   L.total = o;
   return L;
}

// smallest CTA of the kernel: the thread of interior column e is thread e
constexpr int MHM_MIN_BLOCK = PS2*PS2;

// variable sets the MHM kernel is built for (NC = NCOMP_TOTAL): the 5 fluid variables (5), with the
// dual-energy field (6), with GB_NPASSIVE_USER = 2 user passive scalars (7), with both (8).  The
// dual-energy field is the last variable, as in the reference (DUAL = NCOMP_TOTAL-1,
// include/Macro.h:290-305).
__host__ __device__ constexpr bool mhm_has_dual( int nc ) { return nc == 6 || nc == 8; }

// the per-column z state (2*NC values) is kept in shared memory instead of registers by the mixed
// policy (its double accumulation leaves no registers for it) and by the float kernels with user
// passive scalars (96 registers); the FP64 kernels (255 registers) keep it in registers, which
// leaves the shared memory to the planes (FP64 with 7 variables: 215 KB)
__host__ __device__ constexpr bool mhm_carry_smem( int p, int nc ) { return p == P_MIXED || ( nc > 6 && p == P_FP32 ); }

// ---------------------------------------------------------------------------------------------
// face states of one fc cell: reconstruction along x, y, z + Hancock half step + MHM_CHECK_PREDICT
// (Hydro_DataReconstruction PLM :189-689 / PPM :704-1395 and Hydro_HancockPredict :2064-2160)
// ---------------------------------------------------------------------------------------------
template <int D, typename R, int P, int LR, int NC, bool CHARR, bool HANC = true>
GB_DEV void recon_dir( const Phys<R> &ph, const R *cc, const R *pl, const R *pr,
                       const R *sl, const R *sc, const R *sr,
                       int lim, R coeff, bool clamp, R (&fcon)[6][NC], R (&fpres)[6], R (&acc)[NC] )
{
   R wl[NC], wr[NC];
   // (PPM with CHAR_RECONSTRUCTION: sl / sc / sr are already limited in characteristic variables)
   if constexpr ( CHARR && LR == LR_PLM ) plm_faces_char<D,NC>( ph, pl, cc, pr, lim, coeff, wl, wr );
   else
   {
#     pragma unroll
      for (int v=0; v<NC; v++)
      {
         if constexpr ( LR == LR_PLM ) plm_faces( pl[v], cc[v], pr[v], lim, coeff, clamp, wl[v], wr[v] );
         else                          ppm_faces( pl[v], cc[v], pr[v], sl[v], sc[v], sr[v], lim, wl[v], wr[v] );
      }
   }
   fpres[2*D] = wl[4];  fpres[2*D+1] = wr[4];
   pri2con<NC>( ph, wl, fcon[2*D] );
   pri2con<NC>( ph, wr, fcon[2*D+1] );
   if constexpr ( !HANC ) return;    // MHM_RP: no Hancock half step
   // Hancock flux difference, accumulated in the reference's order F1-F0+F3-F2+F5-F4
   R fL[NC], fR[NC];
   pri_con2flux<D,NC>( wl, fcon[2*D],   fL );
   pri_con2flux<D,NC>( wr, fcon[2*D+1], fR );
#  pragma unroll
   for (int v=0; v<NC; v++)
   {
      if constexpr ( D == 0 ) acc[v] = fR[v] - fL[v];
      else                    acc[v] = ( acc[v] + fR[v] ) - fL[v];
   }
}

template <typename R, int P, int NC>
GB_DEV void hancock_finish( const Phys<R> &ph, R dt_dh2, R (&fcon)[6][NC], const R (&fpres)[6],
                            const R (&acc)[NC], const R *g_cc, size_t g_stride, bool &reset )
{
#  pragma unroll
   for (int v=0; v<NC; v++)
   {
      const R df = dt_dh2*acc[v];
#     pragma unroll
      for (int f=0; f<6; f++) fcon[f][v] -= df;
   }
   bool bad = false;
#  pragma unroll
   for (int f=0; f<6; f++)
   {
      const R d = fcon[f][0], e = fcon[f][4], p = fpres[f];
      bad |= ( d < Lim<R>::tiny() || d > Lim<R>::huge() || d != d );
      bad |= ( e < Lim<R>::tiny() || e > Lim<R>::huge() || e != e );
      bad |= ( p < R(0)           || p > Lim<R>::huge() || p != p );
   }
   reset = bad;
   if ( bad )
   {
      // back to the cell-centred input values (read from global memory: rare path)
#     pragma unroll
      for (int v=0; v<NC; v++)
      {
         const R c = g_cc[v*g_stride];
#        pragma unroll
         for (int f=0; f<6; f++) fcon[f][v] = c;
      }
   }
   else
   {
#     pragma unroll
      for (int f=0; f<6; f++)
      {
         fcon[f][0] = gmax( fcon[f][0], ph.min_dens );
         fcon[f][4] = floor_eint_in_engy<P>( ph, fcon[f][0], fcon[f][1], fcon[f][2], fcon[f][3], fcon[f][4] );
#        pragma unroll
         for (int v=5; v<NC; v++) if ( ph.pfloor & ( 1u << v ) ) fcon[f][v] = gmax( fcon[f][v], Lim<R>::tiny() );
      }
   }
}

// ---------------------------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------------------------
// LIMK: LIMK_GMINMOD builds the generalized-MinMod limiter with theta < 2 in (the default, and the
// only limiter code in that instantiation, without the PLM clamps, which never act there);
// LIMK_ANY selects the limiter at run time from MhmArgs::limiter; LIMK_CHAR limits in
// characteristic variables (CHAR_RECONSTRUCTION), the limiter chosen at run time
constexpr int LIMK_ANY = 0, LIMK_GMINMOD = 1, LIMK_CHAR = 2;

// SCH: SCH_MHM, or SCH_MHM_RP, the full step of MHM_RP (CPU_FluidSolver_MHM.cpp:402-520): PLM over the
// half-step primitive state that mhm_rp_half_kernel wrote (20^3 per patch group, no conversion),
// face states without the Hancock predictor, and the update of the conserved 22^3 input
// (FLU_GHOST_SIZE = 3, include/Macro.h:656)
constexpr int SCH_MHM = 0, SCH_MHM_RP = 1;
constexpr int RP_NX = 22, RP_NV = 20;

// Registers: the float kernels are held to 96 per thread, so that two CTAs of 320 threads (the
// default launch) share an SM; FP64 (one CTA of 256 per SM) may use all 255.  REG != 0 caps them at
// REG instead (the autotuner's register variants: 64 / 72 / 80 let two CTAs of 512 / 448 / 384
// threads share an SM, 128 two CTAs of 256).
constexpr int mhm_maxnreg( int rsize, int reg ) { return reg ? reg : ( rsize == 8 ? 255 : 96 ); }

template <typename R, int P, int LR, int RS, int NC, int NIN, int LIMK, int SCH = SCH_MHM, int REG = 0>
__global__ void __maxnreg__( mhm_maxnreg( (int)sizeof(R), REG ) )
mhm_kernel( const __grid_constant__ MhmArgs<R> a )
{
   typedef typename std::conditional<P == P_MIXED, double, R>::type A;   // accumulation type
   typedef typename std::conditional<P == P_MIXED && NC == 5 && LR == LR_PLM, double, R>::type FP;   // x/y flux planes
   constexpr int NG    = ( LR == LR_PPM ) ? 2 : 1;    // LR_GHOST_SIZE
   constexpr int G     = NG + 1;                      // FLU_GHOST_SIZE of the scheme
   constexpr int N     = PS2 + 2*G;                   // scheme input width (20 PLM, 22 PPM)
   constexpr bool CONV_A = mhm_conv_in_a( P, LR, NC, SCH );   // next plane converted in phase A
   constexpr int NSLOT = mhm_nslot( LR, CONV_A );     // plane ring: live planes + those in flight
   constexpr bool LEAN = mhm_lean( sizeof(R), LR );   // PPM: slopes formed in place
   constexpr int AHEAD = LEAN ? 1 : ( CONV_A ? 3 : 2 );   // prefetch distance of the plane ring
   constexpr int LAG   = ( LR == LR_PPM ) ? 2 : 1;    // fc plane kf = t - NG - LAG at step t
   // float PLM: the two faces of each direction are evaluated as one float2 (hydro_pair.cuh)
   constexpr bool PAIR = std::is_same<R, float>::value && LR == LR_PLM;
   constexpr bool CARRY_SMEM = mhm_carry_smem( P, NC );   // per-column z state in shared memory
   // float PLM HLLC without passive scalars: an x face and a y face per thread as float2 lanes
   constexpr bool X2 = PAIR && RS == RS_HLLC && NC == 5;
   constexpr bool CHARR = ( LIMK == LIMK_CHAR );
   constexpr bool DUAL  = mhm_has_dual( NC );         // the last variable is the dual-energy field
   constexpr int  NPU   = NC - 5 - ( DUAL ? 1 : 0 );  // user passive scalars
   constexpr bool RP    = ( SCH == SCH_MHM_RP );
   // MHM_RP: the full step over the half-step state, PLM 20^3 (input 22^3) or PPM 22^3 (input 24^3)
   constexpr int RPX = ( LR == LR_PPM ) ? RP_NX + 2 : RP_NX, RPG = ( RPX - PS2 )/2;   // input width, ghost
   static_assert( !RP || NIN == RPX - 2, "MHM_RP: the full step over the half-step state" );

   extern __shared__ __align__(128) unsigned char smem[];
   constexpr int nin = NIN, nin2 = NIN*NIN;           // input width: a compile-time constant, so the
                                                      // shared-memory addressing folds to offsets
   constexpr int sh  = ( nin - N )/2;                 // offset of the scheme window in the input
   static_assert( NIN >= N && ( NIN - N ) % 2 == 0, "input narrower than the scheme needs" );
   const MhmLayout lay = mhm_layout( sizeof(R), sizeof(A), sizeof(FP), NC, nin, LR, CARRY_SMEM, CONV_A );
   uint64_t *bar  = (uint64_t*)( smem + lay.bar );    // one mbarrier per ring slot
   R *s_pln  = (R*)( smem + lay.pri );     // [NSLOT][NC][nin2]  conserved on arrival, primitive after conversion
   R *s_fcx  = (R*)( smem + lay.fcx );     // [2][NC][16][18]   [side][v][j-1][i]
   R *s_fcy  = (R*)( smem + lay.fcy );     // [2][NC][18][16]   [side][v][j][i-1]
   // one x and one y flux plane: phase B of step t writes those of fc plane kf, phase A of step t+1
   // reads them (the update of output plane kf-1), and the barrier between the phases separates
   // the reads from the next plane's writes
   FP *s_flx = (FP*)( smem + lay.flx );    // [NC][16][17]   [v][j][i]
   FP *s_fly = (FP*)( smem + lay.fly );    // [NC][17][16]   [v][j][i]
   R *s_czu  = (R*)( smem + lay.car );     // [NC][16][16]      upper z face of plane kf-1 (CARRY_SMEM)
   A *s_cfz  = (A*)( smem + lay.car + NC*PS2*PS2*sizeof(R) );   // [NC][16][16] z flux below it
   int *s_flag = (int*)( smem + lay.flag );   // [0] unphysical output, [1] abort

   const int tid = threadIdx.x, nth = blockDim.x;
   const int lim = ( LIMK == LIMK_GMINMOD ) ? LIM_GMINMOD : a.limiter;
   const Phys<R> ph = a.ph;
   const uint32_t plane_bytes = NC*nin2*sizeof(R);

   if ( nth < MHM_MIN_BLOCK ) return;      // rejected by the host; nothing is touched

   if ( tid == 0 )
   {
      for (int q=0; q<NSLOT; q++) mbar_init( &bar[q], 1 );
      mbar_init_fence();
      s_flag[1] = 0;
   }
   __syncthreads();

   // ring slot, and mbarrier phase parity, of cc plane c during sweep number `pass` of this CTA
   // (every sweep loads planes 0..N-1 in order, so slot q is used cnt(q) times per sweep)
   uint32_t pass = 0;
   auto slot_of   = [&]( int c ) { return c % NSLOT; };
   auto parity_of = [&]( int c ) {
      const int q = c % NSLOT;
      const uint32_t cnt = ( N - q + NSLOT - 1 )/NSLOT;
      return ( pass*cnt + (uint32_t)( c/NSLOT ) ) & 1u;
   };
   // primitive plane c, shifted to the scheme window: element (ci, cj) of variable v is
   // plane(c)[v*nin2 + cj*nin + ci]
   auto plane = [&]( int c ) { return s_pln + slot_of( c )*NC*nin2 + sh*nin + sh; };

   for (int pg = blockIdx.x; pg < a.npg; pg += gridDim.x)
   {
      int lv = 0;
      while ( lv + 1 < a.nlevel && pg >= a.level_start[lv + 1] ) lv++;
      const R dt = a.dt[lv], dh = a.dh[lv];
      const R dt_dh2 = R(0.5)*dt/dh;
      const A dt_dh  = (A)dt/(A)dh;
      const R *g_in = a.in + (size_t)pg*NC*nin*nin2;
      R *g_out = a.out + (size_t)pg*NC*PS2*PS2*PS2;
      R *g_flux = ( a.flux != nullptr ) ? a.flux + (size_t)pg*9*NC*PS2*PS2 : nullptr;
      char *g_de = ( a.de != nullptr ) ? a.de + (size_t)pg*PS2*PS2*PS2 : nullptr;

      // one thread issues the bulk copies of cc plane c (all NC variables) into its ring slot
      auto issue = [&]( int c ) {
         const int q = slot_of( c );
         fence_proxy_async();
         mbar_expect_tx( &bar[q], plane_bytes );
         for (int v=0; v<NC; v++)
            bulk_g2s( s_pln + ( q*NC + v )*nin2, g_in + (size_t)v*nin*nin2 + (size_t)( c + sh )*nin2,
                      nin2*sizeof(R), &bar[q] );
      };

      // wait for cc plane c and convert it to primitive variables in place: the calling thread is
      // number vt of the nconv threads the cells are dealt out to
      auto convert = [&]( int c, int vt, int nconv ) {
         if ( !mbar_wait_bounded( &bar[slot_of( c )], parity_of( c ) ) )
         {
            atomicOr( a.status, GB_ST_TMA_TIMEOUT );
            s_flag[1] = 1;
         }
         if constexpr ( RP ) return;      // the half-step state arrives as primitive variables
         R *pt = plane( c );
         if constexpr ( PAIR )
         {
            // two cells per thread, (e, e + N*N/2), as the two lanes of float2
            static_assert( ( N*N ) % 2 == 0, "odd plane size" );
            for (int e = vt; e < N*N/2; e += nconv)
            {
               const int e1 = e + N*N/2;
               const int si0 = ( e / N )*nin + e % N, si1 = ( e1 / N )*nin + e1 % N;
               float2 u[NC], w[NC];
#              pragma unroll
               for (int v=0; v<NC; v++) u[v] = make_float2( pt[v*nin2 + si0], pt[v*nin2 + si1] );
               con2pri_cc_pair<P,NC>( ph, u, w );
#              pragma unroll
               for (int v=0; v<NC; v++) { pt[v*nin2 + si0] = w[v].x;  pt[v*nin2 + si1] = w[v].y; }
            }
         }
         else
         {
            for (int e = vt; e < N*N; e += nconv)
            {
               const int si = ( e / N )*nin + e % N;
               R u[NC], w[NC];
#              pragma unroll
               for (int v=0; v<NC; v++) u[v] = pt[v*nin2 + si];
               con2pri_cc<P,NC>( ph, u, w );
#              pragma unroll
               for (int v=0; v<NC; v++) pt[v*nin2 + si] = w[v];
            }
         }
      };

      // a bulk copy never arrived: wait once more (bounded) for the copies that may still be in
      // flight (planes c to c + AHEAD - 1), then this CTA gives up
      auto bail = [&]( int c ) {
         if ( tid == 0 )
            for (int q = c; q < c + AHEAD && q < N; q++) mbar_wait_bounded( &bar[slot_of( q )], parity_of( q ) );
         __syncthreads();
      };
      // phase-A conversion: the threads from conv0 on (those without an interior column when the
      // CTA has at least one spare warp, all threads otherwise)
      const int conv0 = ( nth >= PS2*PS2 + 32 ) ? PS2*PS2 : 0;

      int iter = 0;
      bool again;
      do {
         R coeff = ( a.minmod_maxiter == 0 ) ? a.minmod_coeff
                 : a.minmod_coeff - (R)iter*a.minmod_coeff/(R)a.minmod_maxiter;
         coeff = gmax( coeff, R(0) );
         // the GMinMod instantiation is only chosen with theta < 2, where the clamps never act
         const bool clamp = ( LIMK == LIMK_GMINMOD ) ? false : plm_clamp_needed( lim, (double)coeff );
         if ( tid == 0 ) { s_flag[0] = 0;  for (int q=0; q<AHEAD; q++) issue( q ); }
         convert( 0, tid, nth );
         __syncthreads();
         if ( s_flag[1] ) { bail( 0 );  return; }

         // carried by the thread of each interior column from one fc plane to the next: the upper z
         // face state of plane kf-1 and the z flux below it (in registers, or in the column's own
         // slots of s_czu / s_cfz)
         R zup[CARRY_SMEM ? 1 : NC];
         A fzp[CARRY_SMEM ? 1 : NC];

         for (int t = 0; t < N; t++)
         {
            const int kf = t - NG - LAG;
            const int cz = kf + NG;                                  // centre cc plane

            // (A) face states of fc plane kf; z Riemann problem below it and output plane kf-2
            if ( kf >= 0 )
            {
               const R *pc = plane( cz ), *pm = plane( cz - 1 ), *pp = plane( cz + 1 );
               const bool edge = ( kf == 0 || kf == NFC - 1 );
               const int ncell = edge ? PS2*PS2 : PS2*PS2 + 4*PS2;
               for (int e = tid; e < ncell; e += nth)
               {
                  int i, j;
                  if ( e < PS2*PS2 ) { i = 1 + e % PS2;  j = 1 + e / PS2; }
                  else {
                     const int h = e - PS2*PS2, q = h / PS2, r = h % PS2;
                     if      ( q == 0 ) { i = 0;       j = 1 + r; }
                     else if ( q == 1 ) { i = NFC - 1; j = 1 + r; }
                     else if ( q == 2 ) { i = 1 + r;   j = 0;     }
                     else               { i = 1 + r;   j = NFC - 1; }
                  }
                  const int ce = ( j + NG )*nin + ( i + NG );
                  const size_t gidx = (size_t)( cz + sh )*nin2 + ( j + NG + sh )*nin + ( i + NG + sh );
                  R cc[NC], nl[NC], nr[NC];
                  R fcon[6][NC], fpres[6], acc[NC];
                  bool reset;
#                 pragma unroll
                  for (int v=0; v<NC; v++) cc[v] = pc[v*nin2 + ce];
                  if constexpr ( PAIR )
                  {
                     float2 fc2[3][NC];
#                    pragma unroll
                     for (int v=0; v<NC; v++) { nl[v] = pc[v*nin2 + ce - 1];  nr[v] = pc[v*nin2 + ce + 1]; }
                     recon_dir_pair<0,P,NC,CHARR,!RP>( ph, cc, nl, nr, lim, coeff, clamp, fc2, fpres, acc );
#                    pragma unroll
                     for (int v=0; v<NC; v++) { nl[v] = pc[v*nin2 + ce - nin];  nr[v] = pc[v*nin2 + ce + nin]; }
                     recon_dir_pair<1,P,NC,CHARR,!RP>( ph, cc, nl, nr, lim, coeff, clamp, fc2, fpres, acc );
#                    pragma unroll
                     for (int v=0; v<NC; v++) { nl[v] = pm[v*nin2 + ce];  nr[v] = pp[v*nin2 + ce]; }
                     recon_dir_pair<2,P,NC,CHARR,!RP>( ph, cc, nl, nr, lim, coeff, clamp, fc2, fpres, acc );
                     if constexpr ( !RP ) hancock_finish_pair<P,NC>( ph, dt_dh2, fc2, fpres, acc, g_in + gidx, (size_t)nin*nin2, reset );
#                    pragma unroll
                     for (int d=0; d<3; d++)
#                       pragma unroll
                        for (int v=0; v<NC; v++) { fcon[2*d][v] = fc2[d][v].x;  fcon[2*d+1][v] = fc2[d][v].y; }
                  }
                  else
                  {
                     R sl[NC], sc[NC], sr[NC];
                     // x
#                    pragma unroll
                     for (int v=0; v<NC; v++) { nl[v] = pc[v*nin2 + ce - 1];  nr[v] = pc[v*nin2 + ce + 1]; }
                     if constexpr ( LEAN && CHARR ) {
                        R ll[NC], rr[NC];
#                       pragma unroll
                        for (int v=0; v<NC; v++) { ll[v] = pc[v*nin2 + ce - 2];  rr[v] = pc[v*nin2 + ce + 2]; }
                        ppm_char_slopes<0,NC>( ph, ll, nl, cc, nr, rr, lim, coeff, sl, sc, sr );
                     }
                     else if constexpr ( LEAN ) {
#                       pragma unroll
                        for (int v=0; v<NC; v++) {
                           const R *q = pc + v*nin2 + ce;
                           sl[v] = limit_slope( q[-2], q[-1], q[0], lim, coeff );
                           sc[v] = limit_slope( q[-1], q[0],  q[1], lim, coeff );
                           sr[v] = limit_slope( q[0],  q[1],  q[2], lim, coeff );
                        }
                     }
                     recon_dir<0,R,P,LR,NC,CHARR,!RP>( ph, cc, nl, nr, sl, sc, sr, lim, coeff, clamp, fcon, fpres, acc );
                     // y
#                    pragma unroll
                     for (int v=0; v<NC; v++) { nl[v] = pc[v*nin2 + ce - nin];  nr[v] = pc[v*nin2 + ce + nin]; }
                     if constexpr ( LEAN && CHARR ) {
                        R ll[NC], rr[NC];
#                       pragma unroll
                        for (int v=0; v<NC; v++) { ll[v] = pc[v*nin2 + ce - 2*nin];  rr[v] = pc[v*nin2 + ce + 2*nin]; }
                        ppm_char_slopes<1,NC>( ph, ll, nl, cc, nr, rr, lim, coeff, sl, sc, sr );
                     }
                     else if constexpr ( LEAN ) {
#                       pragma unroll
                        for (int v=0; v<NC; v++) {
                           const R *q = pc + v*nin2 + ce;
                           sl[v] = limit_slope( q[-2*nin], q[-nin], q[0],   lim, coeff );
                           sc[v] = limit_slope( q[-nin],   q[0],    q[nin], lim, coeff );
                           sr[v] = limit_slope( q[0],      q[nin],  q[2*nin], lim, coeff );
                        }
                     }
                     recon_dir<1,R,P,LR,NC,CHARR,!RP>( ph, cc, nl, nr, sl, sc, sr, lim, coeff, clamp, fcon, fpres, acc );
                     // z
#                    pragma unroll
                     for (int v=0; v<NC; v++) { nl[v] = pm[v*nin2 + ce];  nr[v] = pp[v*nin2 + ce]; }
                     if constexpr ( LEAN && CHARR ) {
                        const R *pmm = plane( cz - 2 ), *ppp = plane( cz + 2 );
                        R ll[NC], rr[NC];
#                       pragma unroll
                        for (int v=0; v<NC; v++) { ll[v] = pmm[v*nin2 + ce];  rr[v] = ppp[v*nin2 + ce]; }
                        ppm_char_slopes<2,NC>( ph, ll, nl, cc, nr, rr, lim, coeff, sl, sc, sr );
                     }
                     else if constexpr ( LEAN ) {
                        const R *pmm = plane( cz - 2 ), *ppp = plane( cz + 2 );
#                       pragma unroll
                        for (int v=0; v<NC; v++) {
                           const int q = v*nin2 + ce;
                           sl[v] = limit_slope( pmm[q], pm[q], pc[q], lim, coeff );
                           sc[v] = limit_slope( pm[q],  pc[q], pp[q], lim, coeff );
                           sr[v] = limit_slope( pc[q],  pp[q], ppp[q], lim, coeff );
                        }
                     }
                     recon_dir<2,R,P,LR,NC,CHARR,!RP>( ph, cc, nl, nr, sl, sc, sr, lim, coeff, clamp, fcon, fpres, acc );
                     if constexpr ( !RP ) hancock_finish<R,P,NC>( ph, dt_dh2, fcon, fpres, acc, g_in + gidx, (size_t)nin*nin2, reset );
                  }

                  const bool inner = ( e < PS2*PS2 );
                  if ( !edge )
                  {
                     if ( inner || i == 0 || i == NFC - 1 )
                     {
                        const int o = ( j - 1 )*NFC + i;
#                       pragma unroll
                        for (int v=0; v<NC; v++) { s_fcx[v*PS2*NFC + o] = fcon[0][v];  s_fcx[( NC + v )*PS2*NFC + o] = fcon[1][v]; }
                     }
                     if ( inner || j == 0 || j == NFC - 1 )
                     {
                        const int o = j*PS2 + ( i - 1 );
#                       pragma unroll
                        for (int v=0; v<NC; v++) { s_fcy[v*NFC*PS2 + o] = fcon[2][v];  s_fcy[( NC + v )*NFC*PS2 + o] = fcon[3][v]; }
                     }
                  }
                  if ( inner )
                  {
                     // interior column e = (i-1, j-1) is always thread e (blockDim >= 256)
                     const int col = e;
                     if ( kf >= 1 )
                     {
                        // z flux between fc planes kf-1 and kf, below output plane ko = kf-1
                        R zl[NC], F[NC];
#                       pragma unroll
                        for (int v=0; v<NC; v++) zl[v] = CARRY_SMEM ? s_czu[v*PS2*PS2 + col] : zup[CARRY_SMEM ? 0 : v];
                        riemann<RS,2,P,NC>( ph, zl, fcon[4], F );
                        const int ko = kf - 1;
                        if ( g_flux != nullptr && ( ko & 7 ) == 0 )
                        {
                           R *dst = g_flux + (size_t)( ( 6 + ( ko >> 3 ) )*NC )*PS2*PS2 + col;
#                          pragma unroll
                           for (int v=0; v<NC; v++) dst[v*PS2*PS2] = F[v];
                        }
                        if ( kf >= 2 )
                        {
                           // output plane o = kf-2: its x/y fluxes are those of fc plane kf-1
                           const int o = kf - 2, oi0 = i - 1, oj0 = j - 1;
                           const FP *fx = s_flx, *fy = s_fly;
                           // U_in of the output cell: the input at offset FLU_GHOST_SIZE (MHM_RP: the
                           // conserved 22^3 input, FLU_GHOST_SIZE = 3)
                           constexpr size_t ustride = RP ? (size_t)RPX*RPX*RPX : (size_t)nin*nin2;
                           const R *uin = RP ? a.uin + (size_t)pg*NC*ustride + (size_t)( o + RPG )*RPX*RPX + ( oj0 + RPG )*RPX + ( oi0 + RPG )
                                             : g_in + (size_t)( o + G + sh )*nin2 + ( oj0 + G + sh )*nin + ( oi0 + G + sh );
                           R u[NC];
#                          pragma unroll
                           for (int v=0; v<NC; v++)
                           {
                              const A dfx = (A)fx[v*PS2*NFLX + oj0*NFLX + oi0 + 1] - (A)fx[v*PS2*NFLX + oj0*NFLX + oi0];
                              const A dfy = (A)fy[v*NFLX*PS2 + ( oj0 + 1 )*PS2 + oi0] - (A)fy[v*NFLX*PS2 + oj0*PS2 + oi0];
                              const A fzl = CARRY_SMEM ? s_cfz[v*PS2*PS2 + col] : fzp[CARRY_SMEM ? 0 : v];
                              const A dfz = (A)F[v] - fzl;
                              u[v] = (R)( (A)uin[(size_t)v*ustride] - dt_dh*( ( dfx + dfy ) + dfz ) );
                           }
                           const int oi = ( o*PS2 + oj0 )*PS2 + oi0;
                           if constexpr ( NC > 5 )
                           {
                              // floors and normalisation of the passive scalars, then the dual-energy
                              // fix (FullStepUpdate.cpp:144-201)
#                             pragma unroll
                              for (int v=5; v<NC; v++) if ( ph.pfloor & ( 1u << v ) ) u[v] = gmax( u[v], Lim<R>::tiny() );
                              if constexpr ( NPU > 0 ) if ( a.nnorm > 0 ) normalize_passive<NC>( u[0], u, a.nnorm, a.norm_idx );
                              if constexpr ( DUAL )
                              {
                                 const R ekin = R(0.5)*( u[1]*u[1] + u[2]*u[2] + u[3]*u[3] )/u[0];
                                 if ( u[0] > R(0) && u[4]*R(2) > ekin )
                                 {
                                    char st;
                                    dual_energy_fix<P>( ph, u[0], u[1], u[2], u[3], u[4], u[NC-1], st );
                                    if ( g_de != nullptr ) g_de[oi] = st;
                                 }
                              }
                           }
#                          pragma unroll
                           for (int v=0; v<NC; v++) g_out[v*PS2*PS2*PS2 + oi] = u[v];
                           if ( is_unphysical<P,NC>( u, ph.pfloor ) ) s_flag[0] = 1;
                        }
#                       pragma unroll
                        for (int v=0; v<NC; v++)
                        {
                           if constexpr ( CARRY_SMEM ) s_cfz[v*PS2*PS2 + col] = (A)F[v];
                           else                        fzp[v] = (A)F[v];
                        }
                     }
#                    pragma unroll
                     for (int v=0; v<NC; v++)
                     {
                        if constexpr ( CARRY_SMEM ) s_czu[v*PS2*PS2 + col] = fcon[5][v];
                        else                        zup[v] = fcon[5][v];
                     }
                  }
               }
            }
            if constexpr ( CONV_A )
               if ( t + 1 < N && tid >= conv0 ) convert( t + 1, tid - conv0, nth - conv0 );
            __syncthreads();
            // the slot of the oldest live plane is free now: prefetch cc plane t+AHEAD into it
            if ( tid == 0 && t + AHEAD < N ) issue( t + AHEAD );

            // (B) x (17x16) and y (16x17) Riemann problems of plane kf for kf in [1,17); conversion
            // of cc plane t+1
            int nrm = 0;
            if ( kf >= 1 && kf <= NFC - 2 )
            {
               const int nx = PS2*NFLX;
               const int ko = kf - 1;          // k index of the x/y fluxes
               FP *flx = s_flx, *fly = s_fly;
               if constexpr ( X2 )
               {
                  // x face e and y face e of the plane as the two lanes of one HLLC, rotated frame
                  // (x: rho, m_x, m_y, m_z, E; y: rho, m_y, m_z, m_x, E)
                  constexpr int ry[5] = { 0, 2, 3, 1, 4 };
                  nrm = nx;
                  for (int e = tid; e < nx; e += nth)
                  {
                     const int ix = e % NFLX, jx = e / NFLX, ox = jx*NFC + ix;
                     const int iy = e % PS2,  jy = e / PS2,  oy = jy*PS2 + iy;
                     float2 L[5], Rr[5], F[5];
#                    pragma unroll
                     for (int q=0; q<5; q++)
                     {
                        L[q]  = make_float2( s_fcx[( NC + q )*PS2*NFC + ox],  s_fcy[( NC + ry[q] )*NFC*PS2 + oy] );
                        Rr[q] = make_float2( s_fcx[q*PS2*NFC + ox + 1],      s_fcy[ry[q]*NFC*PS2 + oy + PS2] );
                     }
                     bool nan_x, nan_y;
                     riemann_hllc_x2<P>( ph, L, Rr, F, nan_x, nan_y );
                     float Fx[5], Fy[5];
#                    pragma unroll
                     for (int q=0; q<5; q++) { Fx[q] = F[q].x;  Fy[ry[q]] = F[q].y; }
                     if ( nan_x || nan_y )
                     {
                        // HLLE rescue of a NaN flux (CPU_Shared_ComputeFlux.cpp:313-362), per face
                        float l[5], r[5];
                        if ( nan_x )
                        {
#                          pragma unroll
                           for (int q=0; q<5; q++) { l[q] = L[q].x;  r[q] = Rr[q].x; }
                           riemann_hlle_outlined<0,P,5>( ph, l, r, Fx );
                        }
                        if ( nan_y )
                        {
#                          pragma unroll
                           for (int q=0; q<5; q++) { l[ry[q]] = L[q].y;  r[ry[q]] = Rr[q].y; }
                           riemann_hlle_outlined<1,P,5>( ph, l, r, Fy );
                        }
                     }
#                    pragma unroll
                     for (int v=0; v<NC; v++) { flx[v*PS2*NFLX + jx*NFLX + ix] = (FP)Fx[v];  fly[v*NFLX*PS2 + oy] = (FP)Fy[v]; }
                     if ( g_flux != nullptr )
                     {
                        if ( ( ix & 7 ) == 0 )
                        {
                           R *dst = g_flux + (size_t)( ( ix >> 3 )*NC )*PS2*PS2 + ko*PS2 + jx;
#                          pragma unroll
                           for (int v=0; v<NC; v++) dst[v*PS2*PS2] = Fx[v];
                        }
                        if ( ( jy & 7 ) == 0 )
                        {
                           R *dst = g_flux + (size_t)( ( 3 + ( jy >> 3 ) )*NC )*PS2*PS2 + ko*PS2 + iy;
#                          pragma unroll
                           for (int v=0; v<NC; v++) dst[v*PS2*PS2] = Fy[v];
                        }
                     }
                  }
               }
               else
               {
               nrm = 2*nx;
               for (int e = tid; e < 2*nx; e += nth)
               {
                  R L[NC], Rr[NC], F[NC];
                  if ( e < nx )
                  {
                     const int i = e % NFLX, j = e / NFLX, o = j*NFC + i;
#                    pragma unroll
                     for (int v=0; v<NC; v++) { L[v] = s_fcx[( NC + v )*PS2*NFC + o];  Rr[v] = s_fcx[v*PS2*NFC + o + 1]; }
                     riemann<RS,0,P,NC>( ph, L, Rr, F );
#                    pragma unroll
                     for (int v=0; v<NC; v++) flx[v*PS2*NFLX + j*NFLX + i] = (FP)F[v];
                     if ( g_flux != nullptr && ( i & 7 ) == 0 )
                     {
                        R *dst = g_flux + (size_t)( ( i >> 3 )*NC )*PS2*PS2 + ko*PS2 + j;
#                       pragma unroll
                        for (int v=0; v<NC; v++) dst[v*PS2*PS2] = F[v];
                     }
                  }
                  else
                  {
                     const int e2 = e - nx, i = e2 % PS2, j = e2 / PS2, o = j*PS2 + i;
#                    pragma unroll
                     for (int v=0; v<NC; v++) { L[v] = s_fcy[( NC + v )*NFC*PS2 + o];  Rr[v] = s_fcy[v*NFC*PS2 + o + PS2]; }
                     riemann<RS,1,P,NC>( ph, L, Rr, F );
#                    pragma unroll
                     for (int v=0; v<NC; v++) fly[v*NFLX*PS2 + o] = (FP)F[v];
                     if ( g_flux != nullptr && ( j & 7 ) == 0 )
                     {
                        R *dst = g_flux + (size_t)( ( 3 + ( j >> 3 ) )*NC )*PS2*PS2 + ko*PS2 + i;
#                       pragma unroll
                        for (int v=0; v<NC; v++) dst[v*PS2*PS2] = F[v];
                     }
                  }
               }
               }
            }
            // the cells are dealt out starting at the first thread with one Riemann problem fewer
            if constexpr ( !CONV_A )
               if ( t + 1 < N ) convert( t + 1, ( tid + nth - nrm % nth ) % nth, nth );
            __syncthreads();
            if ( s_flag[1] ) { bail( t + 1 );  return; }
         } // for t

         pass++;
         const bool fail = ( s_flag[0] != 0 );
         iter++;
         again = fail && iter <= a.minmod_maxiter;
         if ( fail && !again )
         {
            if ( tid == 0 )
            {
               if ( a.pg_fail != nullptr ) a.pg_fail[pg] = 1;
               atomicOr( a.status, GB_ST_UNPHYSICAL );
            }
         }
         else if ( !fail && tid == 0 && a.pg_fail != nullptr ) a.pg_fail[pg] = 0;
         __syncthreads();
      } while ( again );
   } // for pg
}

} // namespace gb
