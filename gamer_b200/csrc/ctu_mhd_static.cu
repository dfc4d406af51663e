// CTU + MHD solve that allocates no device memory, for callers that cannot call cudaMalloc (their
// device memory is owned by their own pool allocator, or their time step must not pay the implicit
// synchronisation of an allocation).  The scratch of the multi-kernel pipeline lives in a
// file-scope __device__ array of fixed size (its own module, so it is loaded only when this entry
// point is used, and then held until the process exits).  Host code must not pass the array's
// name to a kernel (on the host it is only a stand-in symbol): the device address comes from
// cudaGetSymbolAddress, once per device.  Declared in include/gamer_b200_fluid.h as
// gb_ctu_mhd_solve_static.
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>
#include "../../include/gamer_b200_fluid.h"

namespace gb {
size_t ctu_scratch_bytes_per_pg( int precision );
int ctu_solve( const gb_fluid_config &cfg, const void *flu_in, const void *mag_in, void *flu_out, void *mag_out,
               void *flux, void *ele, int npg, const gb_fluid_params *prm, void *scratch, size_t scratch_bytes,
               cudaStream_t st );
}

static_assert( GB_CTU_STATIC_SCRATCH_BYTES % 256 == 0, "scratch size must keep 256-byte alignment" );

// one copy per device (a __device__ variable is instantiated in every context that loads the module)
static __device__ __align__(256) unsigned char g_ctu_static_scratch[GB_CTU_STATIC_SCRATCH_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_lock;
void *g_scratch_ptr[MAX_DEVICES] = {};

// device address of this device's copy of the scratch, looked up once per device.  The address
// belongs to the device's primary context (the one the runtime API uses): after a cudaDeviceReset
// the cached address is stale, so a process that resets a device must not call this entry point
// on it again; callers that run their own (non-primary) contexts are not supported either.
int scratch_for_current_device( void **ptr )
{
   int dev = 0;
   if ( cudaGetDevice( &dev ) != cudaSuccess ) { cudaGetLastError();  return GB_E_CUDA; }
   if ( dev < 0 || dev >= MAX_DEVICES ) return GB_E_UNSUPPORTED;
   std::lock_guard<std::mutex> lock( g_setup_lock );
   if ( g_scratch_ptr[dev] == nullptr )
   {
      void *p = nullptr;
      if ( cudaGetSymbolAddress( &p, g_ctu_static_scratch ) != cudaSuccess || p == nullptr )
      {
         cudaGetLastError();
         return GB_E_CUDA;
      }
      g_scratch_ptr[dev] = p;
   }
   *ptr = g_scratch_ptr[dev];
   return GB_OK;
}

bool aligned16( const void *p ) { return ( reinterpret_cast<uintptr_t>( p ) & 15u ) == 0; }

// patch groups one call can take: the scratch size over the pipeline's scratch per patch group
int static_capacity( int precision )
{
   return (int)( GB_CTU_STATIC_SCRATCH_BYTES / gb::ctu_scratch_bytes_per_pg( precision ) );
}

} // namespace

extern "C"
int gb_ctu_mhd_static_capacity( int precision, int *npg )
{
   if ( npg == nullptr || precision < GB_PREC_FP32 || precision > GB_PREC_FP64 ) return GB_E_INVALID;
   *npg = static_capacity( precision );
   return GB_OK;
}

extern "C"
int gb_ctu_mhd_solve_static( const gb_fluid_config *cfg, const void *flu_in, const void *mag_in,
                             void *flu_out, void *mag_out, void *flux, void *ele, int npg,
                             const gb_fluid_params *prm, void *stream )
{
   if ( cfg == nullptr || prm == nullptr ) return GB_E_INVALID;
   const gb_fluid_config c = *cfg;
   if ( c.scheme != GB_SCHEME_CTU || c.lr_scheme != GB_LR_PLM || c.rsolver != GB_RSOLVER_HLLD ||
        c.dual_energy != GB_DE_NONE || c.flu_nxt != 22 ) return GB_E_UNSUPPORTED;
   if ( c.precision < GB_PREC_FP32 || c.precision > GB_PREC_FP64 || !( c.gamma > 1.0 ) ) return GB_E_INVALID;
   if ( !( prm->dh > 0.0 ) || !( prm->dt >= 0.0 ) || prm->minmod_coeff < 0.0 ) return GB_E_INVALID;
   switch ( prm->lr_limiter ) {
      case GB_LIM_VANLEER: case GB_LIM_GMINMOD: case GB_LIM_ALBADA: case GB_LIM_VL_GMINMOD: case GB_LIM_CENTRAL: break;
      default: return GB_E_INVALID;
   }
   // the whole batch is one pass through the pipeline: it must fit the fixed scratch
   if ( npg < 0 || npg > static_capacity( c.precision ) ) return GB_E_INVALID;
   if ( npg == 0 ) return GB_OK;
   if ( flu_in == nullptr || flu_out == nullptr || mag_in == nullptr || mag_out == nullptr ) return GB_E_INVALID;
   if ( ( prm->store_flux && flux == nullptr ) || ( prm->store_electric && ele == nullptr ) ) return GB_E_INVALID;
   if ( !aligned16( flu_in ) || !aligned16( flu_out ) || !aligned16( mag_in ) || !aligned16( mag_out ) ) return GB_E_ALIGN;
   void *scratch = nullptr;
   const int rc = scratch_for_current_device( &scratch );
   if ( rc != GB_OK ) return rc;
   return gb::ctu_solve( c, flu_in, mag_in, flu_out, mag_out, prm->store_flux ? flux : nullptr,
                         prm->store_electric ? ele : nullptr, npg, prm, scratch, GB_CTU_STATIC_SCRATCH_BYTES,
                         (cudaStream_t)stream );
}
