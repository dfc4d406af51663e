// 1-D bulk copies (TMA, cp.async.bulk) global -> shared with an mbarrier, and bounded waits.
// No cluster multicast is used anywhere in this project.
#pragma once
#include "gb_common.cuh"

namespace gb {

GB_DEV uint32_t smem_u32( const void *p ) { return (uint32_t)__cvta_generic_to_shared( p ); }

GB_DEV void mbar_init( uint64_t *bar, uint32_t count )
{
   asm volatile( "mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"( smem_u32( bar ) ), "r"( count ) : "memory" );
}

GB_DEV void mbar_init_fence()
{
   asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
}

GB_DEV void mbar_expect_tx( uint64_t *bar, uint32_t bytes )
{
   asm volatile( "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"( smem_u32( bar ) ), "r"( bytes ) : "memory" );
}

// order earlier generic-proxy shared-memory accesses before later async-proxy (bulk copy) writes
GB_DEV void fence_proxy_async()
{
   asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" );
}

// bytes must be a multiple of 16 and both addresses 16-byte aligned (checked on the host)
GB_DEV void bulk_g2s( void *dst, const void *src, uint32_t bytes, uint64_t *bar )
{
   asm volatile( "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"( smem_u32( dst ) ), "l"( src ), "r"( bytes ), "r"( smem_u32( bar ) ) : "memory" );
}

GB_DEV bool mbar_try_wait( uint64_t *bar, uint32_t parity )
{
   uint32_t ok;
   asm volatile( "{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"( ok ) : "r"( smem_u32( bar ) ), "r"( parity ) : "memory" );
   return ok != 0;
}

// Wait for the phase with the given parity to complete.  Gives up after max_iter polls (each
// try_wait itself blocks for a bounded, hardware-defined time) and returns false.
GB_DEV bool mbar_wait_bounded( uint64_t *bar, uint32_t parity, uint32_t max_iter = 1u << 20 )
{
   for (uint32_t it=0; it<max_iter; it++)
      if ( mbar_try_wait( bar, parity ) ) return true;
   return false;
}

} // namespace gb
