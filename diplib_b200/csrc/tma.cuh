// Thin device-side wrappers of the sm_100a async-copy machinery used by the tile kernels:
// mbarriers and TMA tiled loads (cp.async.bulk.tensor, no multicast).  Every wait is bounded:
// after kWaitLimit polls a wait gives up and reports it, so a copy that never lands turns into
// a DIPCU_ERR_TIMEOUT status instead of a hung GPU.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace dipcu {

constexpr uint32_t kWaitLimit = 1u << 22;  // polls of ~0.1-1 us each: seconds, far above any copy

__device__ __forceinline__ uint32_t smem_u32( void const* p ) {
   return static_cast< uint32_t >( __cvta_generic_to_shared( p ));
}

__device__ __forceinline__ void mbar_init( uint64_t* bar, uint32_t count ) {
   asm volatile( "mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"( smem_u32( bar )), "r"( count ) : "memory" );
}

__device__ __forceinline__ void fence_mbar_init() {
   asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
}

__device__ __forceinline__ void fence_proxy_async() {
   asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" );
}

__device__ __forceinline__ void mbar_arrive_expect_tx( uint64_t* bar, uint32_t bytes ) {
   asm volatile( "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"( smem_u32( bar )), "r"( bytes ) : "memory" );
}

__device__ __forceinline__ void mbar_arrive( uint64_t* bar ) {
   asm volatile( "mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"( smem_u32( bar )) : "memory" );
}

// Named barrier over the first `threads` threads of the block (id 1..15; 0 is __syncthreads).
__device__ __forceinline__ void named_bar_sync( int id, int threads ) {
   asm volatile( "bar.sync %0, %1;" :: "r"( id ), "r"( threads ) : "memory" );
}

// Arrives at named barrier `id` without waiting (producer side of a producer/consumer pair).
__device__ __forceinline__ void named_bar_arrive( int id, int threads ) {
   asm volatile( "bar.arrive %0, %1;" :: "r"( id ), "r"( threads ) : "memory" );
}

// Bounded wait for the phase with parity `parity` to complete (at most `limit` polls).  Returns
// false on timeout.
__device__ __forceinline__ bool mbar_wait( uint64_t* bar, uint32_t parity, uint32_t limit = kWaitLimit ) {
   uint32_t addr = smem_u32( bar );
   for( uint32_t it = 0; it < limit; ++it ) {
      uint32_t done;
      asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"( done ) : "r"( addr ), "r"( parity ) : "memory" );
      if( done ) { return true; }
      if( it > 32 ) { __nanosleep( 128 ); }
   }
   return false;
}

// 4D tiled TMA load of one box into shared memory, completing on `bar`.  The innermost
// coordinate c0 must be a multiple of 16 bytes / element size (checked by the callers'
// tile geometry, which rounds the box start down to that boundary).
__device__ __forceinline__ void tma_load_4d( void* dst, CUtensorMap const* map, uint64_t* bar,
                                             int32_t c0, int32_t c1, int32_t c2, int32_t c3 ) {
   asm volatile(
         "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
         " [%0], [%1, {%2, %3, %4, %5}], [%6];"
         :: "r"( smem_u32( dst )), "l"( reinterpret_cast< uint64_t >( map )), "r"( c0 ), "r"( c1 ), "r"( c2 ), "r"( c3 ),
            "r"( smem_u32( bar ))
         : "memory" );
}

} // namespace dipcu
