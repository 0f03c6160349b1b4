// K1-2D, warp-per-tile: the fused 2D Gaussian FIR tile kernel for sm_100a.
//
// Every warp works alone on whole tiles (TX x 16 outputs of one image of the batch): the tiles
// are dealt round-robin over all warps of a persistent grid, and lane 0 of each warp keeps its
// next SPW tiles in flight with TMA tiled loads (box = the tile plus its x-y halo, raw input
// type) into the warp's own stages, each completing on its own mbarrier (bounded waits).  Per
// tile, warp-locally: the y pass (one column pair per lane, row blocks of RB outputs, packed f32x2
// arithmetic; y-edge tiles read through a row map) into the warp's buffer, the x-edge fix of the
// halo columns, and the x pass (a sliding register window over a strip of columns per lane) into
// a staging tile that one TMA store writes out (row-by-row coalesced stores where the destination
// layout does not allow TMA).
// No block barrier at all; each input pixel crosses HBM once and each output pixel is written
// once.
//
// The half-widths are a compile-time bucket B >= hx, hy with the taps in the parameters
// (zero beyond each axis' own h), and the symmetry of each axis is a runtime sign: an even kernel
// adds the mirrored tap pair, an odd one subtracts it, at the same cost.  So one instantiation per
// (input type, bucket) serves every sigma and derivative order up to that half-width.
//
// Tile geometry and boundary conditions are those of the 3D warp-specialised kernel (fused3d_ws):
// the TMA box starts LEAD >= B columns before the tile, LEAD a multiple of the TMA granule, so
// that tiles start at multiples of TX and every output row segment is sector-aligned; "mirror", "zero order", "add zeros" and, for float input,
// "asym mirror" in x and y when the image is larger than B along both axes.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "fused3d_ws.cuh"

namespace dipcu {

struct W2Args {
   CUtensorMap tmap;        // 4D (x, y, 1, batch) tiled map of the source
   CUtensorMap tout;        // the same for the destination, box = one tile (TMA stores)
   int32_t tma_store;       // destination layout allows TMA stores
   float* dst;
   int32_t n[ 2 ];
   int32_t nb;
   int64_t ds[ 2 ];
   int64_t db;
   int32_t bc[ 2 ];
   int32_t tiles_x, tiles_y;
   int32_t vec_store;       // float2 stores are 8-byte aligned
   int64_t ntiles;
   int32_t* status;
   float2 sgn[ 2 ];         // per axis: (1, 1) even kernel, (-1, -1) odd kernel
   float2 w[ 2 ][ kFusedMaxTaps ];  // per axis (x, y), centre first, zero beyond h
};

template< typename TIn, int B, int TYP = 16 >
struct W2Geom {
   static constexpr int A = 16 / static_cast< int >( sizeof( TIn ));  // TMA x granule (samples)
   static constexpr int E = B % 2;
   static constexpr int LEAD = ( B + E + A - 1 ) / A * A;              // box columns before the tile (TMA granule)
   static constexpr int OFF = 0;                                       // tiles start at multiples of TX
   static constexpr int BW = 64;                                       // box width: one column pair per lane
   static constexpr int TX = ( BW - LEAD - B ) / 8 * 8;                // outputs per tile row (4 strips of SW)
   static constexpr int TY = TYP;                                      // rows per tile (16 or 32)
   static constexpr int RB = B >= 9 ? 16 : 8;                          // y-pass rows per register block
   static constexpr int BH = TY + 2 * B;                               // box height
   static constexpr int P0 = ( LEAD - B ) / 2;                         // first y-pass column pair
   static constexpr int NPAIR = ( LEAD + TX + B - 1 ) / 2 - P0 + 1;    // y-pass column pairs (one per lane)
   static constexpr int SW = TX / 4;                                   // x-pass strip width (one lane: row pair x strip)
   static constexpr int NPX = SW / 2 + B + E;                          // column pairs a strip reads
   static constexpr int OTS = TX;                                      // row stride of the output staging tile (dense: TMA store)
   static constexpr int STAGE_BYTES = BW * BH * static_cast< int >( sizeof( TIn ));
   static constexpr int STAGE_STRIDE = ( STAGE_BYTES + 127 ) / 128 * 128;
   static constexpr int B2_BYTES = ( BW / 2 ) * ( TY / 2 ) * 16;
   static constexpr int XFIX_MAX = 2 * ( B + 1 );
   static constexpr int TAB_BYTES = ( BH * 8 + XFIX_MAX * 4 + 16 + 15 ) / 16 * 16;   // per warp
   static constexpr int OT_BYTES = ( TY * OTS * 4 + 127 ) / 128 * 128; // per warp
   static constexpr int PER_WARP = B2_BYTES + TAB_BYTES + OT_BYTES;
   // Warps per CTA and stages per warp: two CTAs per SM, as many warps as fit with 2 stages each
   // (3 when there is room), else 4 warps of 1 stage.
   static constexpr int FIT4_3 = 4 * ( 3 * STAGE_STRIDE + PER_WARP ) + 512 <= 112 * 1024;
   static constexpr int FIT4_2 = 4 * ( 2 * STAGE_STRIDE + PER_WARP ) + 512 <= 112 * 1024;
   static constexpr int FIT3_2 = 3 * ( 2 * STAGE_STRIDE + PER_WARP ) + 512 <= 112 * 1024;
   static constexpr int NW = ( FIT4_3 || FIT4_2 ) ? 4 : ( FIT3_2 ? 3 : 4 );
   static constexpr int SPW = FIT4_3 ? 3 : (( FIT4_2 || FIT3_2 ) ? 2 : 1 );
   static constexpr int NT = NW * 32;
   static constexpr int OFF_OT = 0;                                    // 128-byte aligned staging tiles first
   static constexpr int OFF_STAGE = NW * OT_BYTES;
   static constexpr int OFF_B2 = OFF_STAGE + NW * SPW * STAGE_STRIDE;
   static constexpr int OFF_TAB = OFF_B2 + NW * B2_BYTES;
   static constexpr int OFF_BAR = OFF_TAB + NW * TAB_BYTES;
   static constexpr int BYTES = OFF_BAR + NW * SPW * 8 + 16;
   static_assert( TX >= 8 && TX % 8 == 0 && TX % A == 0 && SW % 2 == 0, "tile width" );
   static_assert( TY % 16 == 0, "x-pass lanes: 8 row pairs x 4 strips per group of 16 rows" );
   static_assert(( LEAD + 3 * SW - B ) / 2 + NPX <= P0 + NPAIR, "x-pass reads only y-pass columns" );
   static_assert( LEAD >= B && LEAD + TX + B <= BW && 2 * ( P0 + NPAIR ) <= BW, "box width" );
   static_assert( NPAIR <= 32, "one column pair per lane" );
   static_assert( TY % RB == 0 && RB % 2 == 0, "row blocks" );
   static_assert( STAGE_BYTES % 128 == 0 && OFF_STAGE % 128 == 0 && STAGE_STRIDE % 128 == 0, "TMA destinations 128-byte aligned" );
   static_assert(( TX * 4 ) % 16 == 0, "TMA store rows of 16-byte multiples" );
   static constexpr bool fits = BYTES <= 113 * 1024;
};

template< typename TIn, int B, int TYP >
__global__ void __launch_bounds__( W2Geom< TIn, B, TYP >::NT, 2 ) fused2d_ws_kernel( W2Args const __grid_constant__ a ) {
   using G = W2Geom< TIn, B, TYP >;
   constexpr int TX = G::TX, TY = G::TY, BW = G::BW, BH = G::BH, SPW = G::SPW, RB = G::RB, E = G::E;
   constexpr int NW = G::NW;
   constexpr bool kFloat = std::is_same< TIn, float >::value;
   extern __shared__ __align__( 128 ) unsigned char smem[];
   int const tid = static_cast< int >( threadIdx.x );
   int const warp = tid >> 5, lane = tid & 31;
   uint64_t* const full = reinterpret_cast< uint64_t* >( smem + G::OFF_BAR ) + warp * SPW;
   int volatile* abort = reinterpret_cast< int* >( smem + G::OFF_BAR + NW * SPW * 8 );
   unsigned char* const stages = smem + G::OFF_STAGE + warp * SPW * G::STAGE_STRIDE;
   float4* const b2 = reinterpret_cast< float4* >( smem + G::OFF_B2 + warp * G::B2_BYTES );   // [TY/2][BW/2]
   unsigned char* const tab = smem + G::OFF_TAB + warp * G::TAB_BYTES;
   int32_t* const rmap = reinterpret_cast< int32_t* >( tab );                    // [BH]
   float* const rsgn = reinterpret_cast< float* >( rmap + BH );                   // [BH]
   uint32_t* const xfix = reinterpret_cast< uint32_t* >( rsgn + BH );            // [XFIX_MAX]
   float* const ot = reinterpret_cast< float* >( smem + G::OFF_OT + warp * G::OT_BYTES );   // [TY][TX]

   // Programmatic dependent launch: the next launch in the stream may be scheduled now, and this
   // grid touches global memory only once the previous one has completed and its writes are visible.
   asm volatile( "griddepcontrol.launch_dependents;" ::: "memory" );
   asm volatile( "griddepcontrol.wait;" ::: "memory" );
   if( tid == 0 ) { *abort = 0; }
   if( lane == 0 ) {
      for( int d = 0; d < SPW; ++d ) { mbar_init( &full[ d ], 1 ); }
      fence_mbar_init();
   }
   __syncthreads();

   int const nx = a.n[ 0 ], ny = a.n[ 1 ];
   int64_t const gw = static_cast< int64_t >( blockIdx.x ) * NW + warp;
   int64_t const nwarps = static_cast< int64_t >( gridDim.x ) * NW;
   float2 const sx = a.sgn[ 0 ], sy = a.sgn[ 1 ];

   auto geometry = [ & ]( int64_t t, int& x0, int& y0, int& b ) {
      int const txi = static_cast< int >( t % a.tiles_x );
      int64_t const r = t / a.tiles_x;
      int const tyi = static_cast< int >( r % a.tiles_y );
      b = static_cast< int >( r / a.tiles_y );
      x0 = txi * TX - G::OFF;
      y0 = tyi * TY;
   };
   auto issue = [ & ]( int64_t t, int st ) {
      int x0, y0, b;
      geometry( t, x0, y0, b );
      mbar_arrive_expect_tx( &full[ st ], G::STAGE_BYTES );
      tma_load_4d( stages + st * G::STAGE_STRIDE, &a.tmap, &full[ st ], x0 - G::LEAD, y0 - B, 0, b );
   };
   if( lane == 0 ) {
      for( int k = 0; k < SPW; ++k ) {
         int64_t const t = gw + k * nwarps;
         if( t < a.ntiles ) { issue( t, k ); }
      }
   }
   uint32_t kdone = 0;
   for( int64_t t = gw; t < a.ntiles; t += nwarps, ++kdone ) {
      int x0, y0, b;
      geometry( t, x0, y0, b );
      int const bx = x0 - G::LEAD, by = y0 - B;
      int const st = static_cast< int >( kdone % SPW );
      unsigned char* const sp = stages + st * G::STAGE_STRIDE;
      bool const yedge = by < 0 || y0 + TY + B > ny;
      bool const xedge = x0 - B < 0 || x0 + TX + B > nx;
      // Boundary tables of an edge tile (warp-local; the previous tile's reads are done).
      if( yedge ) {
         for( int r = lane; r < BH; r += 32 ) {
            int const yy = by + r;
            int src = r;
            float sg = 1.f;
            if(( yy < 0 || yy >= ny ) && yy >= -B && yy < ny + B && a.bc[ 1 ] != BC_ADD_ZEROS ) {
               bool neg;
               int const si = static_cast< int >( bc_map_index( yy, ny, a.bc[ 1 ], &neg )) - by;
               if( si >= 0 && si < BH ) { src = si; sg = neg ? -1.f : 1.f; }
            }
            rmap[ r ] = src;
            rsgn[ r ] = sg;
         }
      }
      int nfx = 0;
      if( xedge ) {
         constexpr int C_LO = G::LEAD - B, C_HI = G::LEAD + TX + B;
         for( int cc = C_LO; cc < C_HI; cc += 32 ) {
            int const c = cc + lane;
            int const xx = bx + c;
            uint32_t ent = 0;
            bool want = c < C_HI && !( xx >= 0 && xx < nx ) && xx >= -B && xx < nx + B && a.bc[ 0 ] != BC_ADD_ZEROS;
            if( want ) {
               bool neg;
               int const sc = static_cast< int >( bc_map_index( xx, nx, a.bc[ 0 ], &neg )) - bx;
               want = sc >= C_LO && sc < C_HI;
               ent = static_cast< uint32_t >( c ) | ( static_cast< uint32_t >( sc < 0 ? 0 : sc ) << 8 ) | ( neg ? 1u << 16 : 0u );
            }
            uint32_t const m = __ballot_sync( 0xffffffffu, want );
            int const slot = nfx + __popc( m & (( 1u << lane ) - 1u ));
            if( want && slot < G::XFIX_MAX ) { xfix[ slot ] = ent; }
            nfx += __popc( m );
         }
         nfx = nfx < G::XFIX_MAX ? nfx : G::XFIX_MAX;
      }
      __syncwarp();
      w5_wait( &full[ st ], ( kdone / SPW ) & 1u, abort, a.status );
      // y pass: lane -> column pair, row blocks of RB outputs
      if( lane < G::NPAIR ) {
         int const pc = G::P0 + lane;   // this lane's column pair
#pragma unroll
         for( int r0 = 0; r0 < TY; r0 += RB ) {
            float2 v[ RB + 2 * B ];
            if( !yedge ) {
#pragma unroll
               for( int r = 0; r < RB + 2 * B; ++r ) { v[ r ] = w5_pair< TIn, BW >( sp, r0 + r, pc ); }
            } else {
#pragma unroll
               for( int r = 0; r < RB + 2 * B; ++r ) {
                  v[ r ] = w5_pair< TIn, BW >( sp, rmap[ r0 + r ], pc );
                  if( kFloat ) { v[ r ] = fmul2( make_float2( rsgn[ r0 + r ], rsgn[ r0 + r ] ), v[ r ] ); }
               }
            }
            float2 o[ RB ];
#pragma unroll
            for( int t2 = 0; t2 < RB; ++t2 ) {
               float2 acc = fmul2( a.w[ 1 ][ 0 ], v[ t2 + B ] );
#pragma unroll
               for( int k = 1; k <= B; ++k ) {
                  float2 const ps = ffma2( sy, v[ t2 + B - k ], v[ t2 + B + k ] );
                  acc = ffma2( a.w[ 1 ][ k ], ps, acc );
               }
               o[ t2 ] = acc;
            }
#pragma unroll
            for( int rp = 0; rp < RB / 2; ++rp ) {
               b2[ ( r0 / 2 + rp ) * ( BW / 2 ) + pc ] =
                     make_float4( o[ 2 * rp ].x, o[ 2 * rp + 1 ].x, o[ 2 * rp ].y, o[ 2 * rp + 1 ].y );
            }
         }
      }
      __syncwarp();
      if( lane == 0 ) {
         // The stage is read: stream this warp's tile SPW ahead into it.
         int64_t const tn = t + SPW * nwarps;
         if( tn < a.ntiles ) { issue( tn, st ); }
      }
      if( nfx > 0 ) {
         // Halo columns outside the image take their source column's y-pass result.
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
      // x pass: lane -> (row pair, strip of SW columns); a sliding register window over the
      // strip's NPX column pairs, SW independent accumulators, results staged in `ot`.
      if( a.tma_store ) {
         // The previous tile's TMA store has finished reading `ot`.
         if( lane == 0 ) { asm volatile( "cp.async.bulk.wait_group.read 0;" ::: "memory" ); }
         __syncwarp();
      }
#pragma unroll 1
      for( int grp = 0; grp < TY / 16; ++grp ) {
         int const rp = ( lane >> 2 ) + 8 * grp, c0 = ( lane & 3 ) * G::SW;
         float4 const* row = b2 + rp * ( BW / 2 ) + (( G::LEAD + c0 - B ) >> 1 );
         float2 vx[ 2 * G::NPX ];
#pragma unroll
         for( int m = 0; m < G::NPX; ++m ) {
            float4 const f = row[ m ];
            vx[ 2 * m ] = make_float2( f.x, f.y );
            vx[ 2 * m + 1 ] = make_float2( f.z, f.w );
         }
         float2 out[ G::SW ];
#pragma unroll
         for( int c = 0; c < G::SW; ++c ) {
            constexpr int C0 = B + E;
            float2 acc = fmul2( a.w[ 0 ][ 0 ], vx[ C0 + c ] );
#pragma unroll
            for( int k = 1; k <= B; ++k ) {
               float2 const ps = ffma2( sx, vx[ C0 + c - k ], vx[ C0 + c + k ] );
               acc = ffma2( a.w[ 0 ][ k ], ps, acc );
            }
            out[ c ] = acc;
         }
#pragma unroll
         for( int c = 0; c < G::SW; c += 2 ) {
            *reinterpret_cast< float2* >( ot + ( 2 * rp ) * G::OTS + c0 + c ) = make_float2( out[ c ].x, out[ c + 1 ].x );
            *reinterpret_cast< float2* >( ot + ( 2 * rp + 1 ) * G::OTS + c0 + c ) = make_float2( out[ c ].y, out[ c + 1 ].y );
         }
      }
      if( a.tma_store ) {
         // One TMA store of the staged tile (clipped at the image edges by the tensor map).
         fence_proxy_async();
         __syncwarp();
         if( lane == 0 ) {
            asm volatile( "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
                          :: "l"( reinterpret_cast< uint64_t >( &a.tout )), "r"( x0 ), "r"( y0 ), "r"( 0 ), "r"( b ),
                             "r"( smem_u32( ot )) : "memory" );
            asm volatile( "cp.async.bulk.commit_group;" ::: "memory" );
         }
      } else {
         __syncwarp();
         // coalesced stores of the staged tile: lanes sweep rows in column pairs
         float* const dst_b = a.dst + static_cast< int64_t >( b ) * a.db;
#pragma unroll 4
         for( int e = lane; e < TY * ( TX / 2 ); e += 32 ) {
            int const r = e / ( TX / 2 ), cp = e - r * ( TX / 2 );
            int const xo = x0 + 2 * cp, yo = y0 + r;
            if( xo >= 0 && xo < nx && yo < ny ) {
               float2 const val = *reinterpret_cast< float2 const* >( ot + r * G::OTS + 2 * cp );
               float* const p = dst_b + static_cast< int64_t >( yo ) * a.ds[ 1 ] + xo;
               if( xo + 1 < nx && a.vec_store ) {
                  *reinterpret_cast< float2* >( p ) = val;
               } else {
                  p[ 0 ] = val.x;
                  if( xo + 1 < nx ) { p[ 1 ] = val.y; }
               }
            }
         }
      }
      __syncwarp();   // b2 and table reads done before the next tile
   }
   if( a.tma_store && lane == 0 ) { asm volatile( "cp.async.bulk.wait_group 0;" ::: "memory" ); }
}

} // namespace dipcu
