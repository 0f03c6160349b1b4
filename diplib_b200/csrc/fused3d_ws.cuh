// K1-3D, warp-specialised: the fused 3D Gaussian FIR tile kernel for sm_100a.
//
// Work: the image is cut into tile columns (TX x 8 outputs in x-y, all of z, per batch image);
// the columns' output planes are split evenly over a persistent grid, so every CTA processes one
// or two contiguous z-chunks.  Roles inside a CTA, synchronised through mbarriers and named
// barriers (no block-wide barrier in the plane loop):
//   * NWI in-plane warps take plane pairs round-robin and stream their own pairs: lane 0 keeps
//     SPW pairs in flight with TMA tiled loads (one 2-plane box, or two 1-plane boxes at the z
//     boundary; box = the tile plus its x-y halo, raw input type) into the warp's stages, each on
//     its own mbarrier (bounded waits).  Per plane, warp-locally: the y pass (one column pair per
//     lane, all 8 rows, packed f32x2 arithmetic; y-edge tiles read through a row map) into the
//     warp's buffer, the x-edge fix of halo columns, the x pass (2x2 output points from float4
//     reads) into a shared ring of NS filtered planes;
//   * NWZ z warps: per block of RZ output planes, each thread streams its column pair's
//     RZ + 2 HZ ring values once, accumulates RZ outputs in registers and stores them.
// The ring holds two blocks plus the 2 HZ halo planes, so the in-plane warps fill block j + 1
// while the z warps read block j ("ready" / "free" named barriers per block parity).  Each input
// voxel crosses HBM once (the x-y halo re-reads of neighbouring tiles hit L2); each output voxel
// is written once.  Many loaders per CTA and 2-plane boxes keep enough TMA traffic in flight: a
// single loader thread issuing 1-plane boxes was limited to about one box per 150 ns per CTA.
//
// Tile geometry: the TMA box starts LEAD >= HX columns before the tile, LEAD a multiple of the
// TMA granule (16 bytes), so tiles start at multiples of TX and output rows are sector-aligned;
// the y pass works on aligned column pairs.
//
// Boundary conditions: z uses the mapped plane index as the TMA coordinate (an out-of-range
// coordinate gives TMA zero fill for "add zeros"), with the plane negated for the asymmetric
// conditions.  In x and y the kernel handles "mirror", "zero order", "add zeros" (and, for float
// input, "asym mirror") when every halo sample's source lies in the staged box, which the
// launcher guarantees (n > H); other cases run on the previous kernel.  Rows are remapped on
// load (the row map of y-edge tiles); columns after the y pass, which acts per column.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"
#include "fused3d_tma.cuh"
#include "tma.cuh"

namespace dipcu {

struct W5Args {
   CUtensorMap tmap2;       // 4D (x, y, z, batch) tiled map of the source, boxes of 2 planes
   CUtensorMap tmap1;       // the same with boxes of 1 plane (z-boundary planes)
   float* dst;
   int32_t n[ 3 ];
   int32_t nb;
   int64_t ds[ 3 ];
   int64_t db;
   int32_t bc[ 3 ];
   int32_t tiles_x, tiles_y;
   int32_t vec_store;       // float2 stores are 8-byte aligned
   int64_t units;           // tile columns x n[2]
   int32_t* status;
   float2 w[ 3 ][ kFusedMaxTaps ];  // per axis (x, y, z), centre first, duplicated for f32x2
};

constexpr int w5_pow2( int v ) { return v <= 1 ? 1 : 2 * w5_pow2(( v + 1 ) / 2 ); }
constexpr int w5_min( int a, int b ) { return a < b ? a : b; }

template< typename TIn, int HX, int HY, int HZ >
struct W5Geom {
   static constexpr int A = 16 / static_cast< int >( sizeof( TIn ));  // TMA x granule (samples)
   static constexpr int E = HX % 2;
   static constexpr int LEAD = ( HX + E + A - 1 ) / A * A;             // box columns before the tile (TMA granule)
   static constexpr int OFF = 0;                                       // tiles start at multiples of TX
   static constexpr int PPL = ( LEAD + HX + 48 <= 64 ) ? 1 : 2;        // y-pass column pairs per lane
   static constexpr int BW = 64 * PPL;                                 // box width
   static constexpr int TX = ( BW - LEAD - HX ) / A * A;               // outputs per tile row
   static constexpr int TY = 8;
   static constexpr int BH = TY + 2 * HY;                              // box height
   static constexpr int P0 = ( LEAD - HX ) / 2;                        // first y-pass column pair
   static constexpr int NPAIR = ( LEAD + TX + HX - 1 ) / 2 - P0 + 1;   // y-pass column pairs
   static constexpr int XQ = HX + 1 + E;                               // float4 reads per x-pass point group
   static constexpr int XITEMS = ( TX / 2 ) * ( TY / 2 );
   static constexpr int ZITEMS = ( TX / 2 ) * TY;
   // z ring: two blocks of RZ output planes in flight plus the 2 HZ planes of halo; RZ even, so
   // that blocks start on plane pairs.
   static constexpr int NS = w5_pow2( 2 * HZ + 8 );
   static constexpr int RZ = ( NS - 2 * HZ ) / 2 / 2 * 2;
   static constexpr int NWZ = ( ZITEMS + 63 ) / 64;                    // z-pass warps (~2 items per thread)
   static constexpr int NWI = 6;                                       // in-plane warps
   static constexpr int NWC = NWI + NWZ;
   static constexpr int NT = NWC * 32;
   static constexpr int PLANE_BYTES = BW * BH * static_cast< int >( sizeof( TIn ));
   static constexpr int STAGE_BYTES = 2 * PLANE_BYTES;                 // a stage holds a plane pair
   static constexpr int STAGE_STRIDE = ( STAGE_BYTES + 127 ) / 128 * 128;
   static constexpr int B2_BYTES = ( BW / 2 ) * ( TY / 2 ) * 16;      // per in-plane warp
   static constexpr int RING_PLANE = TX * TY;                          // floats
   static constexpr int XFIX_MAX = 2 * ( HX + 1 );                     // halo columns patched after the y pass
   static constexpr int FIXED = NWI * B2_BYTES + NS * RING_PLANE * 4 + 512;
   static constexpr int BUDGET = FIXED <= 80 * 1024 ? 110 * 1024 : 225 * 1024;
   // Stages per in-plane warp (each warp streams its own plane pairs).
   static constexpr int SPW = ( BUDGET - FIXED ) / ( NWI * STAGE_STRIDE ) >= 2 ? 2 : 1;
   static constexpr int D = NWI * SPW;
   static constexpr int OFF_B2 = D * STAGE_STRIDE;
   static constexpr int OFF_RING = OFF_B2 + NWI * B2_BYTES;
   static constexpr int OFF_TAB = OFF_RING + NS * RING_PLANE * 4;     // row map, row signs, column fixes
   static constexpr int OFF_BAR = ( OFF_TAB + BH * 8 + XFIX_MAX * 4 + 16 + 15 ) / 16 * 16;
   static constexpr int BYTES = OFF_BAR + D * 8 + 16;
   static_assert( TX >= 8 && TX % 2 == 0 && TX % A == 0, "tile width" );
   static_assert( LEAD >= HX && LEAD + TX + HX <= BW && 2 * ( P0 + NPAIR ) <= BW, "box width" );
   static_assert(( LEAD + TX - 2 - HX ) / 2 + XQ <= P0 + NPAIR, "x pass reads only y-pass columns" );
   static_assert( NPAIR <= 32 * PPL, "y-pass pairs per lane" );
   static_assert( RZ >= 2 && RZ % 2 == 0 && NS >= 2 * RZ + 2 * HZ, "z ring" );
   static_assert( NT <= 1024, "block size" );
   static_assert( PLANE_BYTES % 128 == 0 && STAGE_STRIDE % 128 == 0, "TMA destinations 128-byte aligned" );
   static_assert( PLANE_BYTES % 16 == 0 && OFF_B2 % 16 == 0 && OFF_RING % 16 == 0 && OFF_TAB % 16 == 0 &&
                  OFF_BAR % 16 == 0, "16-byte aligned sections" );
   static constexpr bool fits = BYTES <= 227 * 1024;
   static constexpr int MINB = BYTES <= 113 * 1024 ? 2 : 1;            // CTAs per SM the registers must allow
};

// Column pair (box columns 2p, 2p+1) of stage row r, as float.
template< typename TIn, int BW >
__device__ __forceinline__ float2 w5_pair( unsigned char const* stage, int r, int p );

template<>
__device__ __forceinline__ float2 w5_pair< uint16_t, 64 >( unsigned char const* stage, int r, int p ) {
   uint32_t w = reinterpret_cast< uint32_t const* >( stage )[ r * 32 + p ];
   uint32_t lo = __byte_perm( w, 0x4B000000u, 0x7610 );
   uint32_t hi = __byte_perm( w, 0x4B000000u, 0x7632 );
   return fadd2( make_float2( __uint_as_float( lo ), __uint_as_float( hi )), make_float2( -8388608.0f, -8388608.0f ));
}

template<>
__device__ __forceinline__ float2 w5_pair< uint16_t, 128 >( unsigned char const* stage, int r, int p ) {
   uint32_t w = reinterpret_cast< uint32_t const* >( stage )[ r * 64 + p ];
   uint32_t lo = __byte_perm( w, 0x4B000000u, 0x7610 );
   uint32_t hi = __byte_perm( w, 0x4B000000u, 0x7632 );
   return fadd2( make_float2( __uint_as_float( lo ), __uint_as_float( hi )), make_float2( -8388608.0f, -8388608.0f ));
}

template<>
__device__ __forceinline__ float2 w5_pair< float, 64 >( unsigned char const* stage, int r, int p ) {
   return reinterpret_cast< float2 const* >( stage )[ r * 32 + p ];
}

template<>
__device__ __forceinline__ float2 w5_pair< float, 128 >( unsigned char const* stage, int r, int p ) {
   return reinterpret_cast< float2 const* >( stage )[ r * 64 + p ];
}

// Bounded wait that gives up at once after any earlier give-up of the CTA (`abort`), so that a
// copy that never lands costs one timeout, not one per plane.
__device__ __forceinline__ bool w5_wait( uint64_t* bar, uint32_t parity, int volatile* abort, int32_t* status ) {
   if( *abort ) { return false; }
   if( mbar_wait( bar, parity )) { return true; }
   *abort = 1;
   atomicExch( status, DIPCU_ERR_TIMEOUT );
   return false;
}

// Named barriers of the consumer warps (0 is __syncthreads).
constexpr int kBarConsumers = 1;     // all warps: chunk start
constexpr int kBarReady = 2;         // + (block & 1): in-plane warps arrive, z warps wait
constexpr int kBarFree = 4;          // + (block & 1): z warps arrive, in-plane warps wait

// Issues the TMA load(s) of chunk plane pair `pq` (planes 2pq, 2pq+1 of the chunk, the second
// only if it exists) into `stage`, completing on `bar`.  Pairs inside the volume come as one
// 2-plane box; pairs at the z boundary as single planes at their mapped coordinates (-1: TMA zero
// fill for "add zeros").
template< int PLANE_BYTES >
__device__ __forceinline__ void w5_issue_pair( W5Args const& a, unsigned char* stage, uint64_t* bar, int pq, int nplanes,
                                               int zs, int hz, int bx, int by, int b ) {
   int const nz = a.n[ 2 ];
   int const z0 = zs - hz + 2 * pq;
   bool const two = 2 * pq + 1 < nplanes;
   if( two && z0 >= 0 && z0 + 1 < nz ) {
      mbar_arrive_expect_tx( bar, 2 * PLANE_BYTES );
      tma_load_4d( stage, &a.tmap2, bar, bx, by, z0, b );
      return;
   }
   mbar_arrive_expect_tx( bar, ( two ? 2 : 1 ) * PLANE_BYTES );
   for( int e = 0; e < ( two ? 2 : 1 ); ++e ) {
      int zc = z0 + e;
      if( zc < 0 || zc >= nz ) {
         bool neg;
         zc = ( a.bc[ 2 ] == BC_ADD_ZEROS ) ? -1 : static_cast< int >( bc_map_index( zc, nz, a.bc[ 2 ], &neg ));
      }
      tma_load_4d( stage + e * PLANE_BYTES, &a.tmap1, bar, bx, by, zc, b );
   }
}

template< typename TIn, int HX, int HY, int HZ, bool OX, bool OY, bool OZ >
__global__ void __launch_bounds__( W5Geom< TIn, HX, HY, HZ >::NT, W5Geom< TIn, HX, HY, HZ >::MINB ) fused3d_ws_kernel( W5Args const __grid_constant__ a ) {
   using G = W5Geom< TIn, HX, HY, HZ >;
   constexpr int TX = G::TX, TY = G::TY, BW = G::BW, BH = G::BH, NS = G::NS, RZ = G::RZ, SPW = G::SPW;
   constexpr int NWI = G::NWI, NWZ = G::NWZ, NWC = G::NWC, XQ = G::XQ, E = G::E;
   constexpr bool kFloat = std::is_same< TIn, float >::value;
   extern __shared__ __align__( 128 ) unsigned char smem[];
   uint64_t* full = reinterpret_cast< uint64_t* >( smem + G::OFF_BAR );     // [NWI][SPW]
   int volatile* abort = reinterpret_cast< int* >( full + G::D );
   float* ring = reinterpret_cast< float* >( smem + G::OFF_RING );
   int32_t* rmap = reinterpret_cast< int32_t* >( smem + G::OFF_TAB );        // [BH] source row
   float* rsgn = reinterpret_cast< float* >( rmap + BH );                     // [BH] sign (float input)
   uint32_t* xfix = reinterpret_cast< uint32_t* >( rsgn + BH );              // [XFIX_MAX] dst | src << 8 | neg << 16
   int* nxfix = reinterpret_cast< int* >( xfix + G::XFIX_MAX );

   int const tid = static_cast< int >( threadIdx.x );
   int const warp = tid >> 5, lane = tid & 31;
   if( tid == 0 ) {
      for( int d = 0; d < G::D; ++d ) { mbar_init( &full[ d ], 1 ); }
      *abort = 0;
      fence_mbar_init();
   }
   __syncthreads();
   // Programmatic dependent launch: the next launch in the stream may be scheduled now; global
   // memory is touched only after the previous grid has completed and its writes are visible.
   asm volatile( "griddepcontrol.launch_dependents;" ::: "memory" );
   asm volatile( "griddepcontrol.wait;" ::: "memory" );

   int const nx = a.n[ 0 ], ny = a.n[ 1 ], nz = a.n[ 2 ];
   int64_t const ub = ( static_cast< int64_t >( blockIdx.x ) * a.units ) / gridDim.x;
   int64_t const ue = ( static_cast< int64_t >( blockIdx.x + 1 ) * a.units ) / gridDim.x;
   uint32_t gpair = 0;    // plane pairs of this CTA before the current chunk
   uint32_t gblock = 0;   // z blocks of this CTA before the current chunk (barrier parity)
   uint32_t kdone = 0;    // pairs this in-plane warp consumed so far (its stage / parity sequence)

   for( int64_t u = ub; u < ue; ) {
      int64_t const tc = u / nz;
      int const zs = static_cast< int >( u - tc * nz );
      int const ze = static_cast< int >(( nz - zs < ue - u ) ? nz : zs + ( ue - u ));
      u += ze - zs;
      int const txi = static_cast< int >( tc % a.tiles_x );
      int64_t const tr = tc / a.tiles_x;
      int const tyi = static_cast< int >( tr % a.tiles_y );
      int const b = static_cast< int >( tr / a.tiles_y );
      int const x0 = txi * TX, y0 = tyi * TY;
      int const bx = x0 - G::LEAD, by = y0 - HY;
      int const nout_total = ze - zs;
      int const nplanes = nout_total + 2 * HZ;
      int const npairs = ( nplanes + 1 ) / 2;
      int const nblocks = ( nout_total + RZ - 1 ) / RZ;
      // This warp's first pair of the chunk (pairs go round-robin over the in-plane warps).
      int const pfirst = static_cast< int >(( static_cast< uint32_t >( warp + NWI ) - gpair % NWI ) % NWI );

      // Chunk start: every warp is done with the previous chunk (ring, tables).  In-plane warps
      // start streaming their first pairs before the tables are built.
      if( warp < NWI && lane == 0 ) {
         for( int k = 0; k < SPW; ++k ) {
            int const pq = pfirst + k * NWI;
            if( pq >= npairs ) { break; }
            int const st = static_cast< int >(( kdone + k ) % SPW );
            w5_issue_pair< G::PLANE_BYTES >( a, smem + ( warp * SPW + st ) * G::STAGE_STRIDE, &full[ warp * SPW + st ],
                                             pq, nplanes, zs, HZ, bx, by, b );
         }
      }
      named_bar_sync( kBarConsumers, NWC * 32 );
      bool const yedge = by < 0 || y0 + TY + HY > ny;
      bool const xedge = x0 - HX < 0 || x0 + TX + HX > nx;
      if( yedge ) {
         for( int r = tid; r < BH; r += NWC * 32 ) {
            int const yy = by + r;
            int src = r;
            float sg = 1.f;
            // Rows more than HY outside only feed outputs outside the image; "add zeros" rows
            // are TMA zero fill.
            if(( yy < 0 || yy >= ny ) && yy >= -HY && yy < ny + HY && a.bc[ 1 ] != BC_ADD_ZEROS ) {
               bool neg;
               int const si = static_cast< int >( bc_map_index( yy, ny, a.bc[ 1 ], &neg )) - by;
               if( si >= 0 && si < BH ) { src = si; sg = neg ? -1.f : 1.f; }
            }
            rmap[ r ] = src;
            rsgn[ r ] = sg;
         }
      }
      if( xedge && warp == NWC - 1 ) {
         // One warp: each lane tests one used box column; ballot-compacted list.
         constexpr int C_LO = G::LEAD - HX, C_HI = G::LEAD + TX + HX;
         int n = 0;
         for( int cc = C_LO; cc < C_HI; cc += 32 ) {
            int const c = cc + lane;
            int const xx = bx + c;
            uint32_t ent = 0;
            bool want = c < C_HI && !( xx >= 0 && xx < nx ) && xx >= -HX && xx < nx + HX && a.bc[ 0 ] != BC_ADD_ZEROS;
            if( want ) {
               bool neg;
               int const sc = static_cast< int >( bc_map_index( xx, nx, a.bc[ 0 ], &neg )) - bx;
               want = sc >= C_LO && sc < C_HI;
               ent = static_cast< uint32_t >( c ) | ( static_cast< uint32_t >( sc < 0 ? 0 : sc ) << 8 ) | ( neg ? 1u << 16 : 0u );
            }
            uint32_t const m = __ballot_sync( 0xffffffffu, want );
            int const slot = n + __popc( m & (( 1u << lane ) - 1u ));
            if( want && slot < G::XFIX_MAX ) { xfix[ slot ] = ent; }
            n += __popc( m );
         }
         if( lane == 0 ) { *nxfix = n < G::XFIX_MAX ? n : G::XFIX_MAX; }
      }
      named_bar_sync( kBarConsumers, NWC * 32 );
      int const nfx = xedge ? *nxfix : 0;

      if( warp < NWI ) {
         // ---- in-plane warps: per plane pair, y pass, x-edge fix, x pass -> ring
         float4* const b2 = reinterpret_cast< float4* >( smem + G::OFF_B2 + warp * G::B2_BYTES );   // [TY/2][BW/2]
         // The taps as register pairs (packed FMAs take register operands).
         float2 wyr[ HY + 1 ], wxr[ HX + 1 ];
#pragma unroll
         for( int k = 0; k <= HY; ++k ) { wyr[ k ] = a.w[ 1 ][ k ]; }
#pragma unroll
         for( int k = 0; k <= HX; ++k ) { wxr[ k ] = a.w[ 0 ][ k ]; }
         int pq = pfirst;
         for( int j = 0; j < nblocks; ++j ) {
            uint32_t const blk = gblock + static_cast< uint32_t >( j );
            if( j >= 2 ) { named_bar_sync( kBarFree + ( blk & 1u ), NWC * 32 ); }   // ring slots of block j - 2 read
            int const qb = ( j * RZ + RZ < nout_total ? j * RZ + RZ : nout_total ) + 2 * HZ;   // planes of blocks <= j
            for( ; 2 * pq < qb; pq += NWI ) {
               int const st = static_cast< int >( kdone % SPW );
               uint64_t* const bar = &full[ warp * SPW + st ];
               unsigned char* const stage = smem + ( warp * SPW + st ) * G::STAGE_STRIDE;
               w5_wait( bar, ( kdone / SPW ) & 1u, abort, a.status );
               int const np = ( 2 * pq + 1 < nplanes ) ? 2 : 1;
               for( int e = 0; e < np; ++e ) {
                  int const q = 2 * pq + e;
                  unsigned char const* const sp = stage + e * G::PLANE_BYTES;
                  // y pass: lane -> column pair(s), all TY rows
#pragma unroll
                  for( int pp = 0; pp < G::PPL; ++pp ) {
                     int const p = G::P0 + lane + 32 * pp;
                     if( lane + 32 * pp < G::NPAIR ) {
                        float2 v[ BH ];
                        if( !yedge ) {
#pragma unroll
                           for( int r = 0; r < BH; ++r ) { v[ r ] = w5_pair< TIn, BW >( sp, r, p ); }
                        } else {
#pragma unroll
                           for( int r = 0; r < BH; ++r ) {
                              v[ r ] = w5_pair< TIn, BW >( sp, rmap[ r ], p );
                              if( kFloat ) { v[ r ] = fmul2( make_float2( rsgn[ r ], rsgn[ r ] ), v[ r ] ); }
                           }
                        }
                        float2 o[ TY ];
#pragma unroll
                        for( int t = 0; t < TY; ++t ) {
                           float2 acc = OY ? make_float2( 0.f, 0.f ) : fmul2( wyr[ 0 ], v[ t + HY ] );
#pragma unroll
                           for( int k = 1; k <= HY; ++k ) {
                              float2 const ps = OY ? fsub2( v[ t + HY + k ], v[ t + HY - k ] ) : fadd2( v[ t + HY + k ], v[ t + HY - k ] );
                              acc = ffma2( wyr[ k ], ps, acc );
                           }
                           o[ t ] = acc;
                        }
#pragma unroll
                        for( int rp = 0; rp < TY / 2; ++rp ) {
                           b2[ rp * ( BW / 2 ) + p ] = make_float4( o[ 2 * rp ].x, o[ 2 * rp + 1 ].x, o[ 2 * rp ].y, o[ 2 * rp + 1 ].y );
                        }
                     }
                  }
                  __syncwarp();
                  if( e == np - 1 && lane == 0 ) {
                     // The stage is read: stream this warp's pair SPW ahead into it.
                     int const pn = pq + SPW * NWI;
                     if( pn < npairs ) {
                        w5_issue_pair< G::PLANE_BYTES >( a, stage, bar, pn, nplanes, zs, HZ, bx, by, b );
                     }
                  }
                  if( nfx > 0 ) {
                     // Halo columns outside the image: the y pass is per column, so a mirrored
                     // column's result is its source column's (negated for "asym mirror").
                     float2* const b2f = reinterpret_cast< float2* >( b2 );
                     for( int f = lane; f < nfx * ( TY / 2 ); f += 32 ) {
                        uint32_t const fe = xfix[ f / ( TY / 2 ) ];
                        int const rp = f % ( TY / 2 );
                        int const dc = static_cast< int >( fe & 0xffu ), sc = static_cast< int >(( fe >> 8 ) & 0xffu );
                        float2 val = b2f[ ( rp * ( BW / 2 ) + ( sc >> 1 )) * 2 + ( sc & 1 ) ];
                        if( fe & ( 1u << 16 )) { val = make_float2( -val.x, -val.y ); }
                        b2f[ ( rp * ( BW / 2 ) + ( dc >> 1 )) * 2 + ( dc & 1 ) ] = val;
                     }
                     __syncwarp();
                  }
                  // plane sign (asymmetric z conditions)
                  bool zneg = false;
                  {
                     int const zq = zs - HZ + q;
                     if( zq < 0 || zq >= nz ) { bc_map_index( zq, nz, a.bc[ 2 ], &zneg ); }
                  }
                  // x pass: 2x2 output points -> ring plane
                  float* const rs = ring + ( q & ( NS - 1 )) * G::RING_PLANE;
#pragma unroll
                  for( int it = lane; it < G::XITEMS; it += 32 ) {
                     int const cp = it % ( TX / 2 ), rp = it / ( TX / 2 );
                     float4 const* row = b2 + rp * ( BW / 2 ) + (( G::LEAD + 2 * cp - HX ) >> 1 );
                     float2 vx[ 2 * XQ ];
#pragma unroll
                     for( int m = 0; m < XQ; ++m ) {
                        float4 const f = row[ m ];
                        vx[ 2 * m ] = make_float2( f.x, f.y );
                        vx[ 2 * m + 1 ] = make_float2( f.z, f.w );
                     }
                     float2 out[ 2 ];
#pragma unroll
                     for( int c = 0; c < 2; ++c ) {
                        constexpr int C0 = HX + E;
                        float2 acc = OX ? make_float2( 0.f, 0.f ) : fmul2( wxr[ 0 ], vx[ C0 + c ] );
#pragma unroll
                        for( int k = 1; k <= HX; ++k ) {
                           float2 const ps = OX ? fsub2( vx[ C0 + c + k ], vx[ C0 + c - k ] ) : fadd2( vx[ C0 + c + k ], vx[ C0 + c - k ] );
                           acc = ffma2( wxr[ k ], ps, acc );
                        }
                        out[ c ] = zneg ? make_float2( -acc.x, -acc.y ) : acc;
                     }
                     *reinterpret_cast< float2* >( rs + ( 2 * rp ) * TX + 2 * cp ) = make_float2( out[ 0 ].x, out[ 1 ].x );
                     *reinterpret_cast< float2* >( rs + ( 2 * rp + 1 ) * TX + 2 * cp ) = make_float2( out[ 0 ].y, out[ 1 ].y );
                  }
                  __syncwarp();   // b2 reads done before this warp's next y pass
               }
               ++kdone;
            }
            // This warp's planes of blocks <= j are in the ring (arrive orders its ring writes).
            named_bar_arrive( kBarReady + ( blk & 1u ), NWC * 32 );
         }
      } else {
         // ---- z warps: per block, accumulate RZ outputs per column pair from the ring
         int const zt = tid - NWI * 32;
         // The full z kernel as register pairs (index k + HZ for tap k; odd kernels negated below 0).
         float2 wzr[ 2 * HZ + 1 ];
#pragma unroll
         for( int k = -HZ; k <= HZ; ++k ) {
            float2 const w = a.w[ 2 ][ k >= 0 ? k : -k ];
            wzr[ k + HZ ] = ( OZ && k < 0 ) ? make_float2( -w.x, -w.y ) : w;
         }
         for( int j = 0; j < nblocks; ++j ) {
            uint32_t const blk = gblock + static_cast< uint32_t >( j );
            named_bar_sync( kBarReady + ( blk & 1u ), NWC * 32 );
            int const ob = j * RZ;
            int const nout = nout_total - ob < RZ ? nout_total - ob : RZ;
#pragma unroll
            for( int it = zt; it < G::ZITEMS; it += NWZ * 32 ) {
               int const cp = it % ( TX / 2 ), y = it / ( TX / 2 );
               float2 acc[ RZ ];
#pragma unroll
               for( int t = 0; t < RZ; ++t ) { acc[ t ] = make_float2( 0.f, 0.f ); }
               float const* const col = ring + y * TX + 2 * cp;
#pragma unroll
               for( int i = 0; i < RZ + 2 * HZ; ++i ) {
                  float2 const v = *reinterpret_cast< float2 const* >( col + (( ob + i ) & ( NS - 1 )) * G::RING_PLANE );
#pragma unroll
                  for( int t = 0; t < RZ; ++t ) {
                     int const k = i - t - HZ;
                     if( k < -HZ || k > HZ ) { continue; }
                     if( OZ && k == 0 ) { continue; }
                     acc[ t ] = ffma2( wzr[ k + HZ ], v, acc[ t ] );
                  }
               }
               int const xo = x0 + 2 * cp, yo = y0 + y;
               if( yo < ny && xo >= 0 && xo < nx ) {
                  float* p = a.dst + static_cast< int64_t >( b ) * a.db + static_cast< int64_t >( yo ) * a.ds[ 1 ] + xo +
                             static_cast< int64_t >( zs + ob ) * a.ds[ 2 ];
                  bool const both = xo + 1 < nx;
#pragma unroll
                  for( int t = 0; t < RZ; ++t ) {
                     if( t < nout ) {
                        if( both && a.vec_store ) {
                           *reinterpret_cast< float2* >( p ) = acc[ t ];
                        } else {
                           p[ 0 ] = acc[ t ].x;
                           if( both ) { p[ 1 ] = acc[ t ].y; }
                        }
                     }
                     p += a.ds[ 2 ];
                  }
               }
            }
            // The in-plane warps overwrite these ring slots with block j + 2.
            if( j + 2 < nblocks ) { named_bar_arrive( kBarFree + ( blk & 1u ), NWC * 32 ); }
         }
      }
      gpair += static_cast< uint32_t >( npairs );
      gblock += static_cast< uint32_t >( nblocks );
   }
}

} // namespace dipcu
