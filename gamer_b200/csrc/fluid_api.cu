// C ABI of the B200 patch-group fluid solver (declared in include/gamer_b200_fluid.h).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"
#include "mhm_launch.cuh"

using namespace gb;

struct gb_fluid_graph;

struct gb_fluid_solver {
   gb_fluid_config cfg;
   int  ncomp;
   int  block;              // threads per CTA
   int  ctas_per_sm;        // cap on the MHM kernel's CTAs per SM (0: as many as fit)
   int  max_reg;            // register cap of the MHM kernel variant (0: the default instantiation)
   int  device;
   int *d_status;           // device status word (GB_STATUS_* bits)
   cudaStream_t last;       // stream of the last launch (for gb_fluid_get_status)
   // staging for the host-array entry point
   static constexpr int NSTREAM = 3;
   cudaStream_t streams[NSTREAM];
   cudaEvent_t  ev_start;            // the caller's stream, before an asynchronous host-array call
   cudaEvent_t  ev_done[NSTREAM];    // each stream, after it
   void  *d_in[NSTREAM], *d_out[NSTREAM], *d_flux[NSTREAM];
   char  *d_de[NSTREAM];
   size_t stage_npg;        // patch groups each staging slot holds
   // CTU + MHD: magnetic staging and per-stream scratch of the multi-kernel pipeline
   void  *d_bin[NSTREAM], *d_bout[NSTREAM], *d_ele[NSTREAM];
   void  *d_scratch[NSTREAM];
   size_t scratch_bytes;    // bytes of each scratch slot
   int    mhd_chunk;        // patch groups per CTU chunk (0: default)
};

namespace gb {
size_t ctu_scratch_bytes_per_pg( int precision );
size_t mhmrp_mhd_scratch_bytes_per_pg( int precision );
size_t mhmrp_ppm_mhd_scratch_bytes_per_pg( int precision );
size_t mhm_mhd_scratch_bytes_per_pg( int precision );
size_t ctu_ppm_mhd_scratch_bytes_per_pg( int precision );
size_t mhm_ppm_mhd_scratch_bytes_per_pg( int precision );
size_t ctu_hydro_scratch_bytes_per_pg( int precision, int ncomp, int lr_scheme );
int ctu_hydro_solve( const gb_fluid_config &cfg, const void *flu_in, void *flu_out, void *flux, char *de, int npg,
                     const gb_fluid_params *prm, void *scratch, size_t scratch_bytes, cudaStream_t st );
int ctu_solve( const gb_fluid_config &cfg, const void *flu_in, const void *mag_in, void *flu_out, void *mag_out,
               void *flux, void *ele, int npg, const gb_fluid_params *prm, void *scratch, size_t scratch_bytes,
               cudaStream_t st );
int mhm_rp_half( int precision, int rsolver, int nc, int nxi, const void *in, void *half, int npg, double dt, double dh,
                 const Phys<double> &phd, cudaStream_t st );
}

namespace {

// tuned launch shapes on B200 (gamer_b200/autotune.py, gamer_b200/tuned.json): the float kernels keep
// 2 CTAs of 320 threads per SM (one face-state cell per thread per plane), with dual energy too
// (mixed, 1000 patch groups: 320 -> 0.443 ms, 448 -> 0.588 ms) and for PPM; FP64 is bounded to 256
int default_block( const gb_fluid_config &c )
{
   if ( c.precision == GB_PREC_FP64 ) return 256;
   return 320;
}
constexpr int GB_HOST_CHUNK    = 256;     // patch groups per pipelined chunk of gb_fluid_solve_host

bool aligned16( const void *p ) { return ( reinterpret_cast<uintptr_t>( p ) & 15u ) == 0; }

size_t real_size( const gb_fluid_config &c ) { return ( c.precision == GB_PREC_FP64 ) ? 8 : 4; }

// FLU_NXT of the scheme (include/Macro.h:653-665): MHM 1 + LR ghost, CTU hydro 1 + LR ghost,
// CTU MHD 2 + LR ghost, on each side of PS2
int scheme_min_nxt( const gb_fluid_config &c )
{
   if ( c.scheme == GB_SCHEME_MHM_RP ) return PS2 + 2*( ( c.lr_scheme == GB_LR_PPM ) ? 4 : 3 );
   const int lrg = ( c.lr_scheme == GB_LR_PPM ) ? 2 : 1;
   const bool mhd = ( c.scheme == GB_SCHEME_CTU && gb::cfg_mhd( c ) );
   return PS2 + 2*( ( mhd ? 2 : 1 ) + lrg );
}

size_t in_bytes_pg ( const gb_fluid_solver *s ) { return real_size( s->cfg )*s->ncomp*(size_t)s->cfg.flu_nxt*s->cfg.flu_nxt*s->cfg.flu_nxt; }
size_t out_bytes_pg( const gb_fluid_solver *s ) { return real_size( s->cfg )*s->ncomp*(size_t)PS2*PS2*PS2; }
size_t flx_bytes_pg( const gb_fluid_solver *s ) { return real_size( s->cfg )*9*s->ncomp*(size_t)PS2*PS2; }
bool   is_ctu      ( const gb_fluid_solver *s ) { return s->cfg.scheme == GB_SCHEME_CTU; }
bool   is_rp       ( const gb_fluid_solver *s ) { return s->cfg.scheme == GB_SCHEME_MHM_RP; }
bool   is_mhd      ( const gb_fluid_solver *s ) { return gb::cfg_mhd( s->cfg ); }
size_t bin_bytes_pg( const gb_fluid_solver *s ) { const size_t n = s->cfg.flu_nxt; return is_mhd( s ) ? real_size( s->cfg )*3*( n + 1 )*n*n : 0; }
size_t bout_bytes_pg( const gb_fluid_solver *s ) { return is_mhd( s ) ? real_size( s->cfg )*3*( PS2 + 1 )*(size_t)PS2*PS2 : 0; }
size_t ele_bytes_pg( const gb_fluid_solver *s ) { return is_mhd( s ) ? real_size( s->cfg )*9*2*( PS2 + 1 )*(size_t)PS2 : 0; }

// patch groups per CTU chunk of the device entry point (scratch ~2.8 MB per PG for MHD in FP32,
// 1.2 MB for hydro, twice that in FP64).  Measured on B200 (MHD, 2048 PGs, FP32), with the
// directions of each face / edge kernel along grid.y and the patch groups along grid.z: 128 ->
// 7.58, 256 -> 6.92, 512 -> 6.58, 1024 -> 6.41, 2048 -> 6.32 ms: fewer, wider launches beat
// keeping the scratch in L2.  The default takes 2048 (5.7 GB of scratch at most, FP32 MHD; a call
// of fewer patch groups allocates only for those) and 1024 in FP64.
int mhd_chunk( const gb_fluid_solver *s )
{
   if ( s->mhd_chunk > 0 ) return s->mhd_chunk;
   return ( s->cfg.precision == GB_PREC_FP64 ) ? 1024 : 2048;
}

// the host entry point pipelines its chunks over the streams, so it keeps them small
constexpr int GB_HOST_CTU_CHUNK = 512;

// device scratch per patch group: the MHD pipelines' (CTU, MHM_RP) or hydro CTU's intermediate
// arrays, or the hydro MHM_RP half-step state [NC][20^3]
size_t ctu_per_pg( const gb_fluid_solver *s )
{
   if ( is_mhd( s ) ) return is_rp( s )  ? ( ( s->cfg.lr_scheme == GB_LR_PPM ) ? gb::mhmrp_ppm_mhd_scratch_bytes_per_pg( s->cfg.precision )
                                                                               : gb::mhmrp_mhd_scratch_bytes_per_pg( s->cfg.precision ) )
                           : is_ctu( s ) ? ( ( s->cfg.lr_scheme == GB_LR_PPM ) ? gb::ctu_ppm_mhd_scratch_bytes_per_pg( s->cfg.precision )
                                                                               : gb::ctu_scratch_bytes_per_pg( s->cfg.precision ) )
                                         : ( ( s->cfg.lr_scheme == GB_LR_PPM ) ? gb::mhm_ppm_mhd_scratch_bytes_per_pg( s->cfg.precision )
                                                                               : gb::mhm_mhd_scratch_bytes_per_pg( s->cfg.precision ) );
   if ( is_rp( s ) ) { const size_t nv = s->cfg.flu_nxt - 2;  return real_size( s->cfg )*s->ncomp*nv*nv*nv; }
   return gb::ctu_hydro_scratch_bytes_per_pg( s->cfg.precision, s->ncomp, s->cfg.lr_scheme );
}

// device scratch of stream slot `slot` for chunks of npg patch groups; the slots grow together and
// never shrink
int ensure_scratch( gb_fluid_solver *s, int slot, int npg )
{
   const size_t need = ctu_per_pg( s )*(size_t)npg;
   if ( need > s->scratch_bytes )
   {
      cudaDeviceSynchronize();
      for (int i=0; i<gb_fluid_solver::NSTREAM; i++) { cudaFree( s->d_scratch[i] );  s->d_scratch[i] = nullptr; }
      s->scratch_bytes = need;
   }
   if ( s->d_scratch[slot] == nullptr &&
        cudaMalloc( &s->d_scratch[slot], s->scratch_bytes ) != cudaSuccess ) { s->d_scratch[slot] = nullptr;  cudaGetLastError();  return GB_E_NOMEM; }
   return GB_OK;
}

template <typename R>
void fill_phys( Phys<R> &ph, const gb_fluid_config &c, const gb_fluid_params &p, int ncomp )
{
   // EoS_SetAuxArray_Gamma (src/EoS/Gamma/CPU_EoS_Gamma.cpp): constants formed in double, then cast
   ph.gamma     = (R)c.gamma;
   ph.gm1       = (R)( c.gamma - 1.0 );
   ph.inv_gm1   = (R)( 1.0/( c.gamma - 1.0 ) );
   ph.min_dens  = (R)p.min_dens;
   ph.min_pres  = (R)p.min_pres;
   ph.min_eint  = (R)p.min_eint;
   ph.de_switch = (R)p.dual_energy_switch;
   // run-time options of the data reconstruction and the passive scalars
   ph.jeans       = p.jeans_min_pres ? 1 : 0;
   ph.jeans_coeff = (R)p.jeans_min_pres_coeff;
   ph.pfloor      = 0u;
   for (int v=5; v<ncomp; v++) if ( p.passive_floor & ( 1LL << v ) ) ph.pfloor |= 1u << v;
   ph.frac_mask   = 0u;
   if ( p.frac_passive ) for (int k=0; k<p.nfrac; k++) ph.frac_mask |= 1u << p.frac_idx[k];
}

// a list of passive-scalar indices (NormIdx / FracIdx): 1..npassive distinct entries in [0, npassive)
bool passive_list_ok( int n, const int *idx, int npassive )
{
   if ( n < 1 || n > npassive || n > GB_MAX_PASSIVE ) return false;
   for (int k=0; k<n; k++)
   {
      if ( idx[k] < 0 || idx[k] >= npassive ) return false;
      for (int q=0; q<k; q++) if ( idx[q] == idx[k] ) return false;
   }
   return true;
}

// the passive-scalar and Jeans options of a call against the solver's variables: NormPassive and
// FracPassive need passive scalars (the reference's NCOMP_PASSIVE = user scalars + the dual-energy
// field), JeansMinPres a non-negative coefficient
int check_passive_params( const gb_fluid_solver *s, const gb_fluid_params *p )
{
   const int npassive = s->ncomp - 5;
   if ( p->norm_passive && !passive_list_ok( p->nnorm, p->norm_idx, npassive ) ) return GB_E_INVALID;
   if ( p->frac_passive && !passive_list_ok( p->nfrac, p->frac_idx, npassive ) ) return GB_E_INVALID;
   if ( p->jeans_min_pres && !( p->jeans_min_pres_coeff >= 0.0 ) ) return GB_E_INVALID;
   return GB_OK;
}

int check_params( const gb_fluid_params *p )
{
   if ( p == nullptr ) return GB_E_INVALID;
   if ( !( p->dh > 0.0 ) || !( p->dt >= 0.0 ) ) return GB_E_INVALID;
   switch ( p->lr_limiter ) {
      case GB_LIM_VANLEER: case GB_LIM_GMINMOD: case GB_LIM_ALBADA: case GB_LIM_VL_GMINMOD: case GB_LIM_CENTRAL: break;
      default: return GB_E_INVALID;
   }
   if ( p->minmod_maxiter < 0 || p->minmod_coeff < 0.0 ) return GB_E_INVALID;
   return GB_OK;
}

// rp_in: NULL for MHM; for the MHM_RP full step, the conserved input, while `in` is the half-step
// state (nin = 20)
template <typename R>
int launch_mhm( gb_fluid_solver *s, const void *in, void *out, char *de, void *flux, int *pg_fail,
                int nlevel, const int *level_npg, const double *level_dt, const double *level_dh,
                const gb_fluid_params *p, cudaStream_t st, const void *rp_in = nullptr )
{
   MhmArgs<R> a;
   memset( &a, 0, sizeof(a) );
   a.in = (const R*)in;  a.out = (R*)out;  a.flux = (R*)flux;  a.de = de;  a.pg_fail = pg_fail;
   a.uin = (const R*)rp_in;
   a.status = s->d_status;
   const int sch = ( rp_in != nullptr ) ? SCH_MHM_RP : SCH_MHM;
   a.nin = ( sch == SCH_MHM_RP ) ? s->cfg.flu_nxt - 2 : s->cfg.flu_nxt;     // MHM_RP: the half-step state
   a.limiter = p->lr_limiter;  a.minmod_maxiter = p->minmod_maxiter;  a.minmod_coeff = (R)p->minmod_coeff;
   fill_phys( a.ph, s->cfg, *p, s->ncomp );
   if ( p->norm_passive )
   {
      a.nnorm = p->nnorm;
      for (int k=0; k<p->nnorm; k++) a.norm_idx[k] = p->norm_idx[k];
   }
   a.nlevel = nlevel;
   int npg = 0;
   for (int l=0; l<nlevel; l++)
   {
      a.level_start[l] = npg;
      npg += level_npg[l];
      a.dt[l] = (R)level_dt[l];
      a.dh[l] = (R)level_dh[l];
   }
   a.level_start[nlevel] = npg;
   a.npg = npg;
   if ( npg == 0 ) return GB_OK;

   MhmLaunchFn<R> fn = nullptr;
   int limk = s->cfg.char_reconstruction ? LIMK_CHAR :
                    ( s->cfg.rsolver == GB_RSOLVER_EXACT ) ? LIMK_ANY :
                    ( p->lr_limiter == GB_LIM_GMINMOD && p->minmod_coeff < 2.0 ) ? LIMK_GMINMOD : LIMK_ANY;
   // the register-capped variant where it is built, the default instantiation otherwise
   auto lookup = [&]( int reg ) {
      if constexpr ( sizeof(R) == 8 ) return mhm_lookup_fp64( sch, s->cfg.lr_scheme, s->cfg.rsolver, s->ncomp, a.nin, limk, reg, &fn );
      else if ( s->cfg.precision == GB_PREC_MIXED )
         return mhm_lookup_mixed( sch, s->cfg.lr_scheme, s->cfg.rsolver, s->ncomp, a.nin, limk, reg, &fn );
      else return mhm_lookup_fp32( sch, s->cfg.lr_scheme, s->cfg.rsolver, s->ncomp, a.nin, limk, reg, &fn );
   };
   bool ok = ( s->max_reg != 0 && lookup( s->max_reg ) ) || lookup( 0 );
   // configurations built with the run-time limiter only (MHM_RP with passive scalars)
   if ( !ok && limk == LIMK_GMINMOD ) { limk = LIMK_ANY;  ok = lookup( 0 ); }
   if ( !ok ) return GB_E_UNSUPPORTED;
   int grid = 0;
   const cudaError_t err = fn( a, s->block, s->ctas_per_sm, st, &grid );
   s->last = st;
   if ( err == cudaErrorNotSupported ) return GB_E_UNSUPPORTED;
   return ( err == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

int solve_levels( gb_fluid_solver *s, const void *in, void *out, char *de, void *flux, int *pg_fail,
                  int nlevel, const int *level_npg, const double *level_dt, const double *level_dh,
                  const gb_fluid_params *p, cudaStream_t st )
{
   if ( s->cfg.scheme != GB_SCHEME_MHM || gb::cfg_mhd( s->cfg ) ) return GB_E_UNSUPPORTED;
   if ( s->cfg.precision == GB_PREC_FP64 )
      return launch_mhm<double>( s, in, out, de, flux, pg_fail, nlevel, level_npg, level_dt, level_dh, p, st );
   return launch_mhm<float>( s, in, out, de, flux, pg_fail, nlevel, level_npg, level_dt, level_dh, p, st );
}

// MHM_RP (CPU_FluidSolver_MHM.cpp:402-520): the half step of a chunk into the scratch of stream slot
// `slot` (mhm_rp_half), then the full step over it (the MHM kernel's SCH_MHM_RP instantiation), in
// chunks of at most chunk_max patch groups
int solve_rp( gb_fluid_solver *s, const void *in, void *out, char *de, void *flux, int *pg_fail, int npg,
              const gb_fluid_params *p, cudaStream_t st, int slot, int chunk_max )
{
   const int chunk = ( npg < chunk_max ) ? npg : chunk_max;
   int rc = ensure_scratch( s, slot, chunk );
   if ( rc != GB_OK ) return rc;
   Phys<double> phd;
   fill_phys( phd, s->cfg, *p, s->ncomp );
   const size_t bi = in_bytes_pg( s ), bo = out_bytes_pg( s ), bf = flx_bytes_pg( s ), bd = PS2*PS2*PS2;
   const double dt = p->dt, dh = p->dh;
   for (int p0 = 0; p0 < npg; p0 += chunk)
   {
      const int n = ( npg - p0 < chunk ) ? npg - p0 : chunk;
      const char *cin = (const char*)in + p0*bi;
      rc = gb::mhm_rp_half( s->cfg.precision, s->cfg.rsolver, s->ncomp, s->cfg.flu_nxt, cin, s->d_scratch[slot], n, dt, dh,
                            phd, st );
      if ( rc != GB_OK ) return rc;
      char *cout = (char*)out + p0*bo, *cde = de ? de + p0*bd : nullptr;
      void *cflux = flux ? (char*)flux + p0*bf : nullptr;
      int *cfail = pg_fail ? pg_fail + p0 : nullptr;
      rc = ( s->cfg.precision == GB_PREC_FP64 )
         ? launch_mhm<double>( s, s->d_scratch[slot], cout, cde, cflux, cfail, 1, &n, &dt, &dh, p, st, cin )
         : launch_mhm<float> ( s, s->d_scratch[slot], cout, cde, cflux, cfail, 1, &n, &dt, &dh, p, st, cin );
      if ( rc != GB_OK ) return rc;
   }
   return GB_OK;
}

int check_arrays( const gb_fluid_solver *s, const void *in, const void *out, const char *de, const void *flux,
                  int npg, const gb_fluid_params *p )
{
   if ( npg < 0 ) return GB_E_INVALID;
   if ( npg == 0 ) return GB_OK;
   if ( in == nullptr || out == nullptr ) return GB_E_INVALID;
   if ( p->store_flux && flux == nullptr ) return GB_E_INVALID;
   if ( !aligned16( in ) || !aligned16( out ) ) return GB_E_ALIGN;
   (void)de;
   return GB_OK;
}

void free_staging( gb_fluid_solver *s )
{
   for (int i=0; i<gb_fluid_solver::NSTREAM; i++)
   {
      cudaFree( s->d_in[i] );   s->d_in[i] = nullptr;
      cudaFree( s->d_out[i] );  s->d_out[i] = nullptr;
      cudaFree( s->d_flux[i] ); s->d_flux[i] = nullptr;
      cudaFree( s->d_de[i] );   s->d_de[i] = nullptr;
      cudaFree( s->d_bin[i] );  s->d_bin[i] = nullptr;
      cudaFree( s->d_bout[i] ); s->d_bout[i] = nullptr;
      cudaFree( s->d_ele[i] );  s->d_ele[i] = nullptr;
   }
   s->stage_npg = 0;
}

int ensure_staging( gb_fluid_solver *s, size_t npg )
{
   if ( npg <= s->stage_npg ) return GB_OK;
   free_staging( s );
   for (int i=0; i<gb_fluid_solver::NSTREAM; i++)
   {
      if ( cudaMalloc( &s->d_in[i],   npg*in_bytes_pg( s ) ) != cudaSuccess ||
           cudaMalloc( &s->d_out[i],  npg*out_bytes_pg( s ) ) != cudaSuccess ||
           cudaMalloc( &s->d_flux[i], npg*flx_bytes_pg( s ) ) != cudaSuccess ||
           cudaMalloc( (void**)&s->d_de[i], npg*PS2*PS2*PS2 ) != cudaSuccess ||
           ( is_mhd( s ) && ( cudaMalloc( &s->d_bin[i],  npg*bin_bytes_pg( s ) ) != cudaSuccess ||
                              cudaMalloc( &s->d_bout[i], npg*bout_bytes_pg( s ) ) != cudaSuccess ||
                              cudaMalloc( &s->d_ele[i],  npg*ele_bytes_pg( s ) ) != cudaSuccess ) ) )
      {
         free_staging( s );
         cudaGetLastError();
         return GB_E_NOMEM;
      }
   }
   s->stage_npg = npg;
   return GB_OK;
}

// host-array CTU solve (MHD or hydro): chunks round-robin over the streams, each with its own
// staging and scratch; enqueued only
int solve_host_ctu( gb_fluid_solver *s, const void *flu_in, void *flu_out, const void *mag_in, void *mag_out,
                    void *flux, void *ele, char *de_out, int npg, const gb_fluid_params *prm )
{
   int chunk = ( mhd_chunk( s ) < GB_HOST_CTU_CHUNK ) ? mhd_chunk( s ) : GB_HOST_CTU_CHUNK;
   if ( npg < chunk ) chunk = npg;
   const bool dual = ( s->cfg.dual_energy == GB_DE_ENPY );
   const size_t bd = (size_t)PS2*PS2*PS2;
   int rc = ensure_staging( s, chunk );
   if ( rc != GB_OK ) return rc;
   for (int q=0; q<gb_fluid_solver::NSTREAM; q++)
      if ( ( rc = ensure_scratch( s, q, chunk ) ) != GB_OK ) return rc;
   const size_t scratch_chunk = ctu_per_pg( s )*(size_t)chunk;
   const size_t bi = in_bytes_pg( s ), bo = out_bytes_pg( s ), bf = flx_bytes_pg( s );
   const size_t bbi = bin_bytes_pg( s ), bbo = bout_bytes_pg( s ), be = ele_bytes_pg( s );
   int k = 0;
   for (int p0 = 0; p0 < npg; p0 += chunk, k++)
   {
      const int n = ( npg - p0 < chunk ) ? npg - p0 : chunk;
      const int q = k % gb_fluid_solver::NSTREAM;
      cudaStream_t st = s->streams[q];
      const bool mhd = is_mhd( s );
      if ( cudaMemcpyAsync( s->d_in[q],  (const char*)flu_in + p0*bi,  n*bi,  cudaMemcpyHostToDevice, st ) != cudaSuccess ||
           ( mhd && cudaMemcpyAsync( s->d_bin[q], (const char*)mag_in + p0*bbi, n*bbi, cudaMemcpyHostToDevice, st ) != cudaSuccess ) )
         return GB_E_CUDA;
      if ( mhd )
         rc = gb::ctu_solve( s->cfg, s->d_in[q], s->d_bin[q], s->d_out[q], s->d_bout[q],
                             prm->store_flux ? s->d_flux[q] : nullptr, prm->store_electric ? s->d_ele[q] : nullptr,
                             n, prm, s->d_scratch[q], scratch_chunk, st );
      else
      {
         // the dual-energy status is written only where the fix runs: the caller's values elsewhere
         if ( dual && de_out &&
              cudaMemcpyAsync( s->d_de[q], de_out + p0*bd, n*bd, cudaMemcpyHostToDevice, st ) != cudaSuccess )
            return GB_E_CUDA;
         rc = gb::ctu_hydro_solve( s->cfg, s->d_in[q], s->d_out[q], prm->store_flux ? s->d_flux[q] : nullptr,
                                   ( dual && de_out ) ? s->d_de[q] : nullptr, n, prm, s->d_scratch[q], scratch_chunk, st );
      }
      if ( rc != GB_OK ) return rc;
      if ( dual && de_out && !mhd &&
           cudaMemcpyAsync( de_out + p0*bd, s->d_de[q], n*bd, cudaMemcpyDeviceToHost, st ) != cudaSuccess )
         return GB_E_CUDA;
      if ( cudaMemcpyAsync( (char*)flu_out + p0*bo,  s->d_out[q],  n*bo,  cudaMemcpyDeviceToHost, st ) != cudaSuccess ||
           ( mhd && cudaMemcpyAsync( (char*)mag_out + p0*bbo, s->d_bout[q], n*bbo, cudaMemcpyDeviceToHost, st ) != cudaSuccess ) )
         return GB_E_CUDA;
      if ( prm->store_flux &&
           cudaMemcpyAsync( (char*)flux + p0*bf, s->d_flux[q], n*bf, cudaMemcpyDeviceToHost, st ) != cudaSuccess )
         return GB_E_CUDA;
      if ( mhd && prm->store_electric &&
           cudaMemcpyAsync( (char*)ele + p0*be, s->d_ele[q], n*be, cudaMemcpyDeviceToHost, st ) != cudaSuccess )
         return GB_E_CUDA;
   }
   s->last = s->streams[0];
   return GB_OK;
}

// host-array MHM solve: chunks round-robin over the streams, the H2D of chunk k+1 overlapping the
// solve of chunk k and the D2H of chunk k-1 (the reference's GPU_NSTREAM split,
// CUAPI_Asyn_FluidSolver.cu:432-445); enqueued only
int enqueue_host_mhm( gb_fluid_solver *s, const void *flu_in, void *flu_out, char *de_out, void *flux, int npg,
                      const gb_fluid_params *prm )
{
   const bool dual = ( s->cfg.dual_energy == GB_DE_ENPY );
   const int chunk = ( npg < GB_HOST_CHUNK ) ? npg : GB_HOST_CHUNK;
   int rc = ensure_staging( s, chunk );
   if ( rc != GB_OK ) return rc;
   const size_t bi = in_bytes_pg( s ), bo = out_bytes_pg( s ), bf = flx_bytes_pg( s ), bd = PS2*PS2*PS2;
   int k = 0;
   for (int p0 = 0; p0 < npg; p0 += chunk, k++)
   {
      const int n = ( npg - p0 < chunk ) ? npg - p0 : chunk;
      const int q = k % gb_fluid_solver::NSTREAM;
      cudaStream_t st = s->streams[q];
      if ( cudaMemcpyAsync( s->d_in[q], (const char*)flu_in + p0*bi, n*bi, cudaMemcpyHostToDevice, st ) != cudaSuccess )
         return GB_E_CUDA;
      if ( dual && de_out != nullptr )
         if ( cudaMemcpyAsync( s->d_de[q], de_out + p0*bd, n*bd, cudaMemcpyHostToDevice, st ) != cudaSuccess )
            return GB_E_CUDA;
      const double dt = prm->dt, dh = prm->dh;
      if ( is_rp( s ) )
         rc = solve_rp( s, s->d_in[q], s->d_out[q], ( dual && de_out ) ? s->d_de[q] : nullptr,
                        prm->store_flux ? s->d_flux[q] : nullptr, nullptr, n, prm, st, q, chunk );
      else
         rc = solve_levels( s, s->d_in[q], s->d_out[q], ( dual && de_out ) ? s->d_de[q] : nullptr,
                            prm->store_flux ? s->d_flux[q] : nullptr, nullptr, 1, &n, &dt, &dh, prm, st );
      if ( rc != GB_OK ) return rc;
      if ( cudaMemcpyAsync( (char*)flu_out + p0*bo, s->d_out[q], n*bo, cudaMemcpyDeviceToHost, st ) != cudaSuccess )
         return GB_E_CUDA;
      if ( prm->store_flux )
         if ( cudaMemcpyAsync( (char*)flux + p0*bf, s->d_flux[q], n*bf, cudaMemcpyDeviceToHost, st ) != cudaSuccess )
            return GB_E_CUDA;
      if ( dual && de_out != nullptr )
         if ( cudaMemcpyAsync( de_out + p0*bd, s->d_de[q], n*bd, cudaMemcpyDeviceToHost, st ) != cudaSuccess )
            return GB_E_CUDA;
   }
   s->last = s->streams[0];
   return GB_OK;
}

// the run-time parameters of a solver call
int check_call( const gb_fluid_solver *s, const gb_fluid_params *p )
{
   const int rc = check_params( p );
   if ( rc != GB_OK ) return rc;
   return check_passive_params( s, p );
}

// argument checks shared by the host-array entry points
int check_host_call( const gb_fluid_solver *s, const void *flu_in, const void *flu_out, const void *mag_in,
                     const void *mag_out, const void *flux, const void *ele, int npg, const gb_fluid_params *prm )
{
   const int rc = check_call( s, prm );
   if ( rc != GB_OK ) return rc;
   if ( npg < 0 || ( npg > 0 && ( flu_in == nullptr || flu_out == nullptr ) ) ) return GB_E_INVALID;
   if ( npg > 0 && prm->store_flux && flux == nullptr ) return GB_E_INVALID;
   if ( npg > 0 && is_mhd( s ) &&
        ( mag_in == nullptr || mag_out == nullptr || ( prm->store_electric && ele == nullptr ) ) ) return GB_E_INVALID;
   return GB_OK;
}

// enqueue a host-array call on the solver's streams (no synchronisation)
int enqueue_host( gb_fluid_solver *s, const void *flu_in, void *flu_out, const void *mag_in, void *mag_out,
                  char *de_out, void *flux, void *ele, int npg, const gb_fluid_params *prm )
{
   if ( is_mhd( s ) ) return solve_host_ctu( s, flu_in, flu_out, mag_in, mag_out, flux, ele, nullptr, npg, prm );
   if ( is_ctu( s ) ) return solve_host_ctu( s, flu_in, flu_out, nullptr, nullptr, flux, nullptr, de_out, npg, prm );
   return enqueue_host_mhm( s, flu_in, flu_out, de_out, flux, npg, prm );
}

} // namespace

// a captured multi-level launch (gb_fluid_graph_*)
struct gb_fluid_graph {
   gb_fluid_solver *s;
   const void *in;  void *out;  char *de;  void *flux;  int *pg_fail;
   int    nlevel;
   int    npg[GB_MAX_LEVEL];
   double dt[GB_MAX_LEVEL], dh[GB_MAX_LEVEL];
   gb_fluid_params prm;
   cudaStream_t    cap;
   cudaGraphExec_t exec;
};

namespace {

// record the multi-level launch of g into a new graph
int capture_levels( gb_fluid_graph *g, cudaGraph_t *graph )
{
   if ( cudaStreamBeginCapture( g->cap, cudaStreamCaptureModeRelaxed ) != cudaSuccess ) return GB_E_CUDA;
   const int rc = solve_levels( g->s, g->in, g->out, g->de, g->prm.store_flux ? g->flux : nullptr, g->pg_fail,
                                g->nlevel, g->npg, g->dt, g->dh, &g->prm, g->cap );
   const cudaError_t e = cudaStreamEndCapture( g->cap, graph );
   if ( rc != GB_OK ) { if ( e == cudaSuccess ) cudaGraphDestroy( *graph ); return rc; }
   return ( e == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

} // namespace

extern "C" {

int gb_fluid_graph_create_levels( gb_fluid_solver *s, const void *flu_in, void *flu_out, char *de_out,
                                  void *flux, int *pg_fail, int nlevel, const int *level_npg,
                                  const double *level_dt, const double *level_dh,
                                  const gb_fluid_params *prm, gb_fluid_graph **out )
{
   if ( out == nullptr ) return GB_E_INVALID;
   *out = nullptr;
   if ( s == nullptr || level_npg == nullptr || level_dt == nullptr || level_dh == nullptr ) return GB_E_INVALID;
   if ( nlevel < 1 || nlevel > GB_MAX_LEVEL ) return GB_E_INVALID;
   int rc = check_call( s, prm );
   if ( rc != GB_OK ) return rc;
   long long total = 0;
   for (int l=0; l<nlevel; l++)
   {
      if ( level_npg[l] < 0 || !( level_dh[l] > 0.0 ) || !( level_dt[l] >= 0.0 ) ) return GB_E_INVALID;
      total += level_npg[l];
   }
   if ( total <= 0 || total > 0x7fffffff ) return GB_E_INVALID;
   rc = check_arrays( s, flu_in, flu_out, de_out, flux, (int)total, prm );
   if ( rc != GB_OK ) return rc;

   gb_fluid_graph *g = new (std::nothrow) gb_fluid_graph;
   if ( g == nullptr ) return GB_E_NOMEM;
   memset( (void*)g, 0, sizeof(*g) );
   g->s = s;  g->in = flu_in;  g->out = flu_out;  g->de = de_out;  g->flux = flux;  g->pg_fail = pg_fail;
   g->nlevel = nlevel;  g->prm = *prm;
   for (int l=0; l<nlevel; l++) { g->npg[l] = level_npg[l];  g->dt[l] = level_dt[l];  g->dh[l] = level_dh[l]; }
   if ( cudaStreamCreateWithFlags( &g->cap, cudaStreamNonBlocking ) != cudaSuccess ) { delete g; return GB_E_CUDA; }
   cudaGraph_t graph;
   rc = capture_levels( g, &graph );
   if ( rc != GB_OK ) { cudaStreamDestroy( g->cap ); delete g; return rc; }
   const cudaError_t e = cudaGraphInstantiate( &g->exec, graph, 0 );
   cudaGraphDestroy( graph );
   if ( e != cudaSuccess ) { cudaStreamDestroy( g->cap ); delete g; cudaGetLastError(); return GB_E_CUDA; }
   *out = g;
   return GB_OK;
}

int gb_fluid_graph_set_dt( gb_fluid_graph *g, const double *level_dt )
{
   if ( g == nullptr || level_dt == nullptr ) return GB_E_INVALID;
   for (int l=0; l<g->nlevel; l++) if ( !( level_dt[l] >= 0.0 ) ) return GB_E_INVALID;
   for (int l=0; l<g->nlevel; l++) g->dt[l] = level_dt[l];
   cudaGraph_t graph;
   int rc = capture_levels( g, &graph );
   if ( rc != GB_OK ) return rc;
   cudaGraphExecUpdateResultInfo info;
   cudaError_t e = cudaGraphExecUpdate( g->exec, graph, &info );
   if ( e != cudaSuccess )
   {
      // topology changed (it cannot here, but stay correct): instantiate afresh
      cudaGetLastError();
      cudaGraphExecDestroy( g->exec );
      e = cudaGraphInstantiate( &g->exec, graph, 0 );
   }
   cudaGraphDestroy( graph );
   return ( e == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

int gb_fluid_graph_launch( gb_fluid_graph *g, void *stream )
{
   if ( g == nullptr ) return GB_E_INVALID;
   g->s->last = (cudaStream_t)stream;
   return ( cudaGraphLaunch( g->exec, (cudaStream_t)stream ) == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

int gb_fluid_graph_destroy( gb_fluid_graph *g )
{
   if ( g == nullptr ) return GB_E_INVALID;
   cudaStreamSynchronize( g->cap );
   cudaGraphExecDestroy( g->exec );
   cudaStreamDestroy( g->cap );
   delete g;
   return GB_OK;
}


int gb_fluid_version( void ) { return 100; }

int gb_fluid_get_config( const gb_fluid_solver *s, gb_fluid_config *cfg )
{
   if ( s == nullptr || cfg == nullptr ) return GB_E_INVALID;
   *cfg = s->cfg;
   return GB_OK;
}

const char *gb_fluid_strerror( int code )
{
   switch ( code ) {
      case GB_OK:            return "success";
      case GB_E_INVALID:     return "invalid argument";
      case GB_E_ALIGN:       return "array not 16-byte aligned";
      case GB_E_CUDA:        return "CUDA runtime error";
      case GB_E_NOMEM:       return "out of memory";
      case GB_E_UNSUPPORTED: return "configuration not supported";
      default:               return "unknown error";
   }
}

int gb_fluid_create( const gb_fluid_config *cfg, gb_fluid_solver **out )
{
   if ( cfg == nullptr || out == nullptr ) return GB_E_INVALID;
   *out = nullptr;
   const gb_fluid_config c = *cfg;
   if ( c.precision < GB_PREC_FP32 || c.precision > GB_PREC_FP64 ) return GB_E_INVALID;
   if ( c.dual_energy != GB_DE_NONE && c.dual_energy != GB_DE_ENPY ) return GB_E_INVALID;
   if ( !( c.gamma > 1.0 ) ) return GB_E_INVALID;
   if ( c.char_reconstruction != 0 && c.char_reconstruction != 1 ) return GB_E_INVALID;
   // user passive scalars: built for NCOMP_PASSIVE_USER = GB_NPASSIVE_USER in hydro MHM, MHM_RP and
   // CTU, with the scheme's own FLU_NXT
   if ( c.npassive_user != 0 && c.npassive_user != GB_NPASSIVE_USER ) return ( c.npassive_user < 0 ) ? GB_E_INVALID : GB_E_UNSUPPORTED;
   if ( c.npassive_user != 0 && ( gb::cfg_mhd( c ) || c.flu_nxt != scheme_min_nxt( c ) ) ) return GB_E_UNSUPPORTED;
   // characteristic limiting is built for every scheme: MHM and MHM_RP (PLM and PPM) and CTU (hydro
   // and MHD)
   // MHM and MHM_RP in FP64 with PPM, two passive scalars and dual energy (8 variables): the five
   // primitive planes of 8 x 22^2 doubles and the face-state and flux planes take 257 KB of shared
   // memory (and the MHM_RP half step 237 KB), above the 227 KB of a CTA
   if ( c.precision == GB_PREC_FP64 && c.lr_scheme == GB_LR_PPM && c.npassive_user && c.dual_energy != GB_DE_NONE &&
        c.scheme != GB_SCHEME_CTU )
      return GB_E_UNSUPPORTED;
   // the exact solver with PPM and characteristic limiting: MHM on its own FLU_NXT, 5 or 6 variables
   if ( c.char_reconstruction && c.lr_scheme == GB_LR_PPM && c.rsolver == GB_RSOLVER_EXACT && c.scheme == GB_SCHEME_MHM &&
        ( c.flu_nxt != 22 || c.npassive_user != 0 ) )
      return GB_E_UNSUPPORTED;
   if ( c.scheme == GB_SCHEME_MHM_RP )
   {
      // MHM_RP is built on the scheme's own FLU_NXT: hydro with PLM (22) or PPM (24) and HLLC / HLLE
      // / ROE (and their HLLE rescue), with or without two passive scalars, with or without
      // characteristic limiting; MHD with PLM (22) or PPM (24) and HLLD (HLLE rescue), without dual energy,
      // with or without characteristic limiting
      if ( c.lr_scheme != GB_LR_PLM && c.lr_scheme != GB_LR_PPM ) return GB_E_INVALID;
      if ( c.rsolver < GB_RSOLVER_EXACT || c.rsolver > GB_RSOLVER_HLLD ) return GB_E_INVALID;
      if ( c.rsolver == GB_RSOLVER_HLLD )
      {
         if ( c.dual_energy != GB_DE_NONE || c.npassive_user ) return GB_E_UNSUPPORTED;
      }
      else if ( c.rsolver == GB_RSOLVER_EXACT ) return GB_E_UNSUPPORTED;
      if ( c.flu_nxt != scheme_min_nxt( c ) ) return ( c.flu_nxt < scheme_min_nxt( c ) ) ? GB_E_INVALID : GB_E_UNSUPPORTED;
   }
   else if ( c.scheme == GB_SCHEME_MHM )
   {
      if ( c.lr_scheme != GB_LR_PLM && c.lr_scheme != GB_LR_PPM ) return GB_E_INVALID;
      // MHD (HLLD): PLM or PPM, without dual energy, with or without characteristic limiting
      if ( c.rsolver == GB_RSOLVER_HLLD && c.dual_energy != GB_DE_NONE ) return GB_E_UNSUPPORTED;
      if ( c.rsolver == GB_RSOLVER_HLLD && c.flu_nxt != scheme_min_nxt( c ) )
         return ( c.flu_nxt < scheme_min_nxt( c ) ) ? GB_E_INVALID : GB_E_UNSUPPORTED;
      if ( c.rsolver != GB_RSOLVER_HLLC && c.rsolver != GB_RSOLVER_HLLE && c.rsolver != GB_RSOLVER_ROE &&
           c.rsolver != GB_RSOLVER_EXACT && c.rsolver != GB_RSOLVER_HLLD ) return GB_E_INVALID;
   }
   else if ( c.scheme == GB_SCHEME_CTU )
   {
      // CTU is built for MHD with HLLD (HLLE rescue), PLM (FLU_NXT = 22) or PPM (24), no dual energy, and for
      // hydro with PLM (FLU_NXT = 20) or PPM (22) and HLLC / exact (HLLE rescue), HLLE or Roe, with or
      // without dual energy and user passive scalars, each with or without characteristic limiting
      if ( c.lr_scheme != GB_LR_PLM && c.lr_scheme != GB_LR_PPM ) return GB_E_INVALID;
      if ( c.rsolver < GB_RSOLVER_EXACT || c.rsolver > GB_RSOLVER_HLLD ) return GB_E_INVALID;
      if ( c.rsolver == GB_RSOLVER_HLLD && c.dual_energy != GB_DE_NONE ) return GB_E_UNSUPPORTED;
      if ( c.flu_nxt != scheme_min_nxt( c ) ) return ( c.flu_nxt < scheme_min_nxt( c ) ) ? GB_E_INVALID : GB_E_UNSUPPORTED;
   }
   else return GB_E_INVALID;
   if ( c.flu_nxt < scheme_min_nxt( c ) || ( c.flu_nxt - scheme_min_nxt( c ) ) % 2 != 0 ) return GB_E_INVALID;
   // kernels are built for the scheme's own FLU_NXT and for FLU_NXT + 2
   if ( c.flu_nxt > scheme_min_nxt( c ) + 2 ) return GB_E_UNSUPPORTED;

   gb_fluid_solver *s = new (std::nothrow) gb_fluid_solver;
   if ( s == nullptr ) return GB_E_NOMEM;
   memset( (void*)s, 0, sizeof(*s) );
   s->cfg   = c;
   s->ncomp = 5 + c.npassive_user + ( ( c.dual_energy == GB_DE_ENPY ) ? 1 : 0 );
   s->block = default_block( c );
   s->ctas_per_sm = 0;
   s->max_reg = 0;
   if ( cudaGetDevice( &s->device ) != cudaSuccess ) { delete s; cudaGetLastError(); return GB_E_CUDA; }
   if ( cudaMalloc( &s->d_status, sizeof(int) ) != cudaSuccess ) { delete s; cudaGetLastError(); return GB_E_NOMEM; }
   if ( cudaMemset( s->d_status, 0, sizeof(int) ) != cudaSuccess ) { cudaFree( s->d_status ); delete s; return GB_E_CUDA; }
   for (int i=0; i<gb_fluid_solver::NSTREAM; i++)
      if ( cudaStreamCreateWithFlags( &s->streams[i], cudaStreamNonBlocking ) != cudaSuccess ||
           cudaEventCreateWithFlags( &s->ev_done[i], cudaEventDisableTiming ) != cudaSuccess )
      {
         for (int k=0; k<=i; k++) { if ( s->streams[k] ) cudaStreamDestroy( s->streams[k] );  if ( s->ev_done[k] ) cudaEventDestroy( s->ev_done[k] ); }
         cudaFree( s->d_status );  delete s;  cudaGetLastError();  return GB_E_CUDA;
      }
   if ( cudaEventCreateWithFlags( &s->ev_start, cudaEventDisableTiming ) != cudaSuccess )
   {
      for (int k=0; k<gb_fluid_solver::NSTREAM; k++) { cudaStreamDestroy( s->streams[k] );  cudaEventDestroy( s->ev_done[k] ); }
      cudaFree( s->d_status );  delete s;  cudaGetLastError();  return GB_E_CUDA;
   }
   *out = s;
   return GB_OK;
}

int gb_fluid_destroy( gb_fluid_solver *s )
{
   if ( s == nullptr ) return GB_E_INVALID;
   cudaDeviceSynchronize();
   free_staging( s );
   for (int i=0; i<gb_fluid_solver::NSTREAM; i++)
   {
      cudaFree( s->d_scratch[i] );  cudaStreamDestroy( s->streams[i] );  cudaEventDestroy( s->ev_done[i] );
   }
   cudaEventDestroy( s->ev_start );
   cudaFree( s->d_status );
   delete s;
   return GB_OK;
}

int gb_fluid_set_block_size( gb_fluid_solver *s, int threads )
{
   if ( s == nullptr ) return GB_E_INVALID;
   if ( threads == 0 ) { s->block = default_block( s->cfg ); return GB_OK; }
   // the MHM kernel gives each of the 16x16 interior columns its own thread
   if ( threads < 256 || threads > 512 || threads % 32 != 0 ) return GB_E_INVALID;
   s->block = threads;
   return GB_OK;
}

int gb_fluid_set_launch( gb_fluid_solver *s, int threads, int ctas_per_sm, int max_registers )
{
   if ( s == nullptr ) return GB_E_INVALID;
   if ( threads != 0 && ( threads < 256 || threads > 512 || threads % 32 != 0 ) ) return GB_E_INVALID;
   if ( ctas_per_sm < 0 || ctas_per_sm > 8 ) return GB_E_INVALID;
   if ( max_registers != 0 && max_registers != 64 && max_registers != 72 && max_registers != 80 &&
        max_registers != 128 ) return GB_E_INVALID;
   s->block = threads ? threads : default_block( s->cfg );
   s->ctas_per_sm = ctas_per_sm;
   s->max_reg = max_registers;
   return GB_OK;
}

int gb_fluid_get_launch( gb_fluid_solver *s, int *threads, int *ctas_per_sm, int *max_registers )
{
   if ( s == nullptr ) return GB_E_INVALID;
   if ( threads != nullptr ) *threads = s->block;
   if ( ctas_per_sm != nullptr ) *ctas_per_sm = s->ctas_per_sm;
   if ( max_registers != nullptr ) *max_registers = s->max_reg;
   return GB_OK;
}

int gb_fluid_set_mhd_chunk( gb_fluid_solver *s, int npg )
{
   if ( s == nullptr || npg < 0 || npg > 4096 ) return GB_E_INVALID;
   s->mhd_chunk = npg;
   return GB_OK;
}

int gb_fluid_get_block_size( gb_fluid_solver *s, int *threads )
{
   if ( s == nullptr || threads == nullptr ) return GB_E_INVALID;
   *threads = s->block;
   return GB_OK;
}

int gb_fluid_array_bytes( const gb_fluid_solver *s, unsigned long long *in_bytes, unsigned long long *out_bytes,
                          unsigned long long *flux_bytes )
{
   if ( s == nullptr ) return GB_E_INVALID;
   if ( in_bytes )   *in_bytes   = in_bytes_pg( s );
   if ( out_bytes )  *out_bytes  = out_bytes_pg( s );
   if ( flux_bytes ) *flux_bytes = flx_bytes_pg( s );
   return GB_OK;
}

int gb_fluid_solve_device( gb_fluid_solver *s, const void *flu_in, void *flu_out,
                           const void *mag_in, void *mag_out, char *de_out,
                           void *flux, void *ele, int *pg_fail, int npg,
                           const gb_fluid_params *prm, void *stream )
{
   if ( s == nullptr ) return GB_E_INVALID;
   int rc = check_call( s, prm );
   if ( rc != GB_OK ) return rc;
   rc = check_arrays( s, flu_in, flu_out, de_out, flux, npg, prm );
   if ( rc != GB_OK || npg == 0 ) return rc;
   if ( is_mhd( s ) )
   {
      if ( mag_in == nullptr || mag_out == nullptr || ( prm->store_electric && ele == nullptr ) ) return GB_E_INVALID;
      if ( !aligned16( mag_in ) || !aligned16( mag_out ) ) return GB_E_ALIGN;
      const int chunk = ( npg < mhd_chunk( s ) ) ? npg : mhd_chunk( s );
      rc = ensure_scratch( s, 0, chunk );
      if ( rc != GB_OK ) return rc;
      s->last = (cudaStream_t)stream;
      return gb::ctu_solve( s->cfg, flu_in, mag_in, flu_out, mag_out, prm->store_flux ? flux : nullptr,
                            prm->store_electric ? ele : nullptr, npg, prm, s->d_scratch[0],
                            ctu_per_pg( s )*(size_t)chunk, (cudaStream_t)stream );
   }
   if ( is_ctu( s ) )
   {
      const int chunk = ( npg < mhd_chunk( s ) ) ? npg : mhd_chunk( s );
      rc = ensure_scratch( s, 0, chunk );
      if ( rc != GB_OK ) return rc;
      s->last = (cudaStream_t)stream;
      return gb::ctu_hydro_solve( s->cfg, flu_in, flu_out, prm->store_flux ? flux : nullptr, de_out, npg, prm,
                                  s->d_scratch[0], ctu_per_pg( s )*(size_t)chunk, (cudaStream_t)stream );
   }
   if ( is_rp( s ) )
   {
      s->last = (cudaStream_t)stream;
      return solve_rp( s, flu_in, flu_out, de_out, prm->store_flux ? flux : nullptr, pg_fail, npg, prm,
                       (cudaStream_t)stream, 0, mhd_chunk( s ) );
   }
   const double dt = prm->dt, dh = prm->dh;
   return solve_levels( s, flu_in, flu_out, de_out, prm->store_flux ? flux : nullptr, pg_fail, 1, &npg, &dt, &dh,
                        prm, (cudaStream_t)stream );
}

int gb_fluid_solve_levels_device( gb_fluid_solver *s, const void *flu_in, void *flu_out, char *de_out,
                                  void *flux, int *pg_fail, int nlevel, const int *level_npg,
                                  const double *level_dt, const double *level_dh,
                                  const gb_fluid_params *prm, void *stream )
{
   if ( s == nullptr || level_npg == nullptr || level_dt == nullptr || level_dh == nullptr ) return GB_E_INVALID;
   if ( nlevel < 1 || nlevel > GB_MAX_LEVEL ) return GB_E_INVALID;
   int rc = check_call( s, prm );
   if ( rc != GB_OK ) return rc;
   long long total = 0;
   for (int l=0; l<nlevel; l++)
   {
      if ( level_npg[l] < 0 || !( level_dh[l] > 0.0 ) || !( level_dt[l] >= 0.0 ) ) return GB_E_INVALID;
      total += level_npg[l];
   }
   if ( total > 0x7fffffff ) return GB_E_INVALID;
   rc = check_arrays( s, flu_in, flu_out, de_out, flux, (int)total, prm );
   if ( rc != GB_OK || total == 0 ) return rc;
   return solve_levels( s, flu_in, flu_out, de_out, prm->store_flux ? flux : nullptr, pg_fail, nlevel, level_npg,
                        level_dt, level_dh, prm, (cudaStream_t)stream );
}

int gb_fluid_solve_host_async( gb_fluid_solver *s, const void *flu_in, void *flu_out,
                               const void *mag_in, void *mag_out, char *de_out,
                               void *flux, void *ele, int npg, const gb_fluid_params *prm, void *stream )
{
   if ( s == nullptr ) return GB_E_INVALID;
   int rc = check_host_call( s, flu_in, flu_out, mag_in, mag_out, flux, ele, npg, prm );
   if ( rc != GB_OK || npg == 0 ) return rc;
   const cudaStream_t ext = (cudaStream_t)stream;
   if ( ext == nullptr ) return enqueue_host( s, flu_in, flu_out, mag_in, mag_out, de_out, flux, ele, npg, prm );
   // the solver's streams start after the work already on the caller's stream ...
   if ( cudaEventRecord( s->ev_start, ext ) != cudaSuccess ) return GB_E_CUDA;
   for (int q=0; q<gb_fluid_solver::NSTREAM; q++)
      if ( cudaStreamWaitEvent( s->streams[q], s->ev_start, 0 ) != cudaSuccess ) return GB_E_CUDA;
   rc = enqueue_host( s, flu_in, flu_out, mag_in, mag_out, de_out, flux, ele, npg, prm );
   // ... and the caller's stream waits for all of them (also after a failed enqueue, so that what
   // was enqueued is still ordered before the caller's later work)
   for (int q=0; q<gb_fluid_solver::NSTREAM; q++)
      if ( cudaEventRecord( s->ev_done[q], s->streams[q] ) != cudaSuccess ||
           cudaStreamWaitEvent( ext, s->ev_done[q], 0 ) != cudaSuccess ) return GB_E_CUDA;
   return rc;
}

int gb_fluid_synchronize( gb_fluid_solver *s )
{
   if ( s == nullptr ) return GB_E_INVALID;
   int rc = GB_OK;
   for (int q=0; q<gb_fluid_solver::NSTREAM; q++)
      if ( cudaStreamSynchronize( s->streams[q] ) != cudaSuccess ) rc = GB_E_CUDA;
   return rc;
}

int gb_fluid_solve_host( gb_fluid_solver *s, const void *flu_in, void *flu_out,
                         const void *mag_in, void *mag_out, char *de_out,
                         void *flux, void *ele, int npg, const gb_fluid_params *prm )
{
   if ( s == nullptr ) return GB_E_INVALID;
   int rc = check_host_call( s, flu_in, flu_out, mag_in, mag_out, flux, ele, npg, prm );
   if ( rc != GB_OK || npg == 0 ) return rc;
   rc = enqueue_host( s, flu_in, flu_out, mag_in, mag_out, de_out, flux, ele, npg, prm );
   const int rs = gb_fluid_synchronize( s );
   return ( rc != GB_OK ) ? rc : rs;
}

int gb_fluid_get_status( gb_fluid_solver *s, int *status )
{
   if ( s == nullptr || status == nullptr ) return GB_E_INVALID;
   if ( cudaDeviceSynchronize() != cudaSuccess ) return GB_E_CUDA;
   if ( cudaMemcpy( status, s->d_status, sizeof(int), cudaMemcpyDeviceToHost ) != cudaSuccess ) return GB_E_CUDA;
   if ( cudaMemset( s->d_status, 0, sizeof(int) ) != cudaSuccess ) return GB_E_CUDA;
   return GB_OK;
}

int gb_fluid_host_alloc( void **ptr, unsigned long long bytes )
{
   if ( ptr == nullptr ) return GB_E_INVALID;
   if ( cudaMallocHost( ptr, bytes ) != cudaSuccess ) { *ptr = nullptr; cudaGetLastError(); return GB_E_NOMEM; }
   return GB_OK;
}

int gb_fluid_host_free( void *ptr )
{
   return ( cudaFreeHost( ptr ) == cudaSuccess ) ? GB_OK : GB_E_CUDA;
}

} // extern "C"
