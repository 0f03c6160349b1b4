// K3-2D, warp-per-tile: the fused adjoint of the 2D Gaussian FIR with both sigma gradients.
//
// Forward (dip::GaussFIR on a 2D image, x first): y = C_y E_y C_x E_x x, with C_a the correlation
// with the axis' taps and E_a its boundary extension.  Its adjoint is
//    x_bar = F_x F_y y_bar,   F_a = E_a^T C_a^T,
// where C_a^T is the correlation with the flipped taps over the extended line (y_bar zero-padded)
// and E_a^T folds the result at each halo position j back onto its source m(j) (negated for
// "asym mirror").  The sigma gradients are
//    dL/dsigma_x = < x, F'_x F_y y_bar >,   dL/dsigma_y = < x, F_x F'_y y_bar >,
// with F'_a built from the analytic derivative of the normalised taps (kernel length fixed).
//
// Per tile (TX x 16 outputs), warp-locally, as in the forward warp-per-tile kernel (fused2d_ws):
// TMA brings y_bar with its halo (out-of-image samples are TMA zero fill, which is exactly the
// zero padding of C^T) and the tile of x; the y pass computes v = C_y^T y_bar and v' = C'_y^T y_bar
// from the same loads; y-edge tiles add the y fold (the tile that owns the fold's target row
// computes the halo value z(j) from its own staged rows); the x pass computes x_bar = C_x^T v,
// a = C'_x^T v and c = C_x^T v', x-edge tiles add the x fold, and a, c are dotted with x.  x_bar
// goes out through a staging tile (one TMA store, or coalesced stores); the dots are reduced per warp and added
// to the two sigma gradients (double) once per warp.  One kernel reads y_bar and x once and writes
// x_bar once.
//
// Boundary conditions: "mirror", "zero order", "asym mirror" and "add zeros" in x and y (the folds
// of these stay within H of the edge), images larger than the half-width bucket along both axes.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "fused2d_ws.cuh"

namespace dipcu {

struct A2Args {
   CUtensorMap tg;          // y_bar: 4D (x, y, 1, batch) float map, box (64, BH)
   CUtensorMap tx;          // x: the same layout in the input type, box (TX, 16)
   CUtensorMap tgx;         // x_bar, box = one tile (TMA stores)
   int32_t tma_store;       // x_bar layout allows TMA stores
   float* gx;               // x_bar (nullptr: not wanted)
   double* dsig[ 2 ];       // dL/dsigma_x, dL/dsigma_y accumulators (nullptr: not wanted)
   int32_t n[ 2 ];
   int32_t nb;
   int64_t gs1, gb;         // x_bar row and batch strides (x stride 1)
   int32_t bc[ 2 ];
   int32_t h[ 2 ];          // half-widths (the bucket may be larger)
   int32_t tiles_x, tiles_y;
   int32_t vec_store;
   int64_t ntiles;
   int32_t* status;
   float2 s[ 2 ];           // pair sign per axis: (1, 1) even kernel, (-1, -1) odd kernel
   float2 w[ 2 ][ kFusedMaxTaps ];    // adjoint taps: w_0, s * w_k (zero beyond h)
   float2 wd[ 2 ][ kFusedMaxTaps ];   // adjoint sigma-derivative taps
};

template< typename TIn, int B >
struct A2Geom {
   using G = W2Geom< float, B >;                                       // y_bar box / tile geometry
   static constexpr int TX = G::TX, TY = G::TY, BW = G::BW, BH = G::BH, LEAD = G::LEAD, P0 = G::P0;
   static constexpr int NPAIR = G::NPAIR, SW = G::SW, NPX = G::NPX, OTS = G::OTS, RB = G::RB;
   static constexpr int GBYTES = BW * BH * 4;                         // y_bar box
   static constexpr int XBYTES = TX * TY * static_cast< int >( sizeof( TIn ));
   static constexpr int STAGE_STRIDE = ( GBYTES + XBYTES + 127 ) / 128 * 128;
   static constexpr int B2_BYTES = ( BW / 2 ) * ( TY / 2 ) * 16;
   static constexpr int FOLD_MAX = 2 * B;
   static constexpr int TAB_BYTES = ( 2 * FOLD_MAX * 4 + 16 + 15 ) / 16 * 16;
   static constexpr int OT_BYTES = TY * OTS * 4;
   static constexpr int PER_WARP = 2 * B2_BYTES + TAB_BYTES + OT_BYTES;
   static constexpr int SPW = 2;
   static constexpr int NW = ( 110 * 1024 ) / ( SPW * STAGE_STRIDE + PER_WARP ) >= 4 ? 4 : 3;
   static constexpr int NT = NW * 32;
   static constexpr int OFF_OT = 0;                                    // 128-byte aligned staging tiles first
   static constexpr int OFF_STAGE = NW * OT_BYTES;
   static constexpr int OFF_B2 = OFF_STAGE + NW * SPW * STAGE_STRIDE;
   static constexpr int OFF_TAB = OFF_B2 + NW * 2 * B2_BYTES;
   static constexpr int OFF_BAR = OFF_TAB + NW * TAB_BYTES;
   static constexpr int BYTES = OFF_BAR + NW * SPW * 8 + 16;
   static_assert( GBYTES % 128 == 0 && ( XBYTES % 16 ) == 0 && OT_BYTES % 128 == 0, "TMA destinations and sources" );
   static_assert(( TX * static_cast< int >( sizeof( TIn ))) % 16 == 0, "x box rows of 16-byte multiples" );
   static constexpr bool fits = BYTES <= 113 * 1024;
};

// b2 holds a 2x2 point group per float4: (col 2p row 2r, col 2p row 2r+1, col 2p+1 row 2r,
// col 2p+1 row 2r+1); the float2 of column c, row pair r:
__device__ __forceinline__ int a2_b2col( int r, int c, int bw ) { return ( r * ( bw / 2 ) + ( c >> 1 )) * 2 + ( c & 1 ); }

template< typename TIn, int B >
__global__ void __launch_bounds__( A2Geom< TIn, B >::NT, 2 ) fused2d_adj_kernel( A2Args const __grid_constant__ a ) {
   using G = A2Geom< TIn, B >;
   constexpr int TX = G::TX, TY = G::TY, BW = G::BW, BH = G::BH, SPW = G::SPW, RB = G::RB, NW = G::NW;
   constexpr int LEAD = G::LEAD, SW = G::SW, NPX = G::NPX, OTS = G::OTS;
   constexpr int E = B % 2;
   extern __shared__ __align__( 128 ) unsigned char smem[];
   int const tid = static_cast< int >( threadIdx.x );
   int const warp = tid >> 5, lane = tid & 31;
   uint64_t* const full = reinterpret_cast< uint64_t* >( smem + G::OFF_BAR ) + warp * SPW;
   int volatile* abort = reinterpret_cast< int* >( smem + G::OFF_BAR + NW * SPW * 8 );
   unsigned char* const stages = smem + G::OFF_STAGE + warp * SPW * G::STAGE_STRIDE;
   float4* const b2 = reinterpret_cast< float4* >( smem + G::OFF_B2 + warp * 2 * G::B2_BYTES );    // v
   float4* const b2d = reinterpret_cast< float4* >( smem + G::OFF_B2 + warp * 2 * G::B2_BYTES + G::B2_BYTES );   // v'
   uint32_t* const yfold = reinterpret_cast< uint32_t* >( smem + G::OFF_TAB + warp * G::TAB_BYTES );   // tr | jb << 8 | neg << 16
   uint32_t* const xfold = yfold + G::FOLD_MAX;                                                          // tc | jb << 8 | neg << 16
   float* const ot = reinterpret_cast< float* >( smem + G::OFF_OT + warp * G::OT_BYTES );

   if( tid == 0 ) { *abort = 0; }
   if( lane == 0 ) {
      for( int d = 0; d < SPW; ++d ) { mbar_init( &full[ d ], 1 ); }
      fence_mbar_init();
   }
   __syncthreads();

   int const nx = a.n[ 0 ], ny = a.n[ 1 ];
   int64_t const gw = static_cast< int64_t >( blockIdx.x ) * NW + warp;
   int64_t const nwarps = static_cast< int64_t >( gridDim.x ) * NW;
   float2 const sx = a.s[ 0 ], sy = a.s[ 1 ];
   bool const want_gx = a.gx != nullptr;
   bool const want_sig = a.dsig[ 0 ] != nullptr;
   float dsx = 0.f, dsy = 0.f;   // this lane's parts of the two dot products

   auto geometry = [ & ]( int64_t t, int& x0, int& y0, int& b ) {
      int const txi = static_cast< int >( t % a.tiles_x );
      int64_t const r = t / a.tiles_x;
      int const tyi = static_cast< int >( r % a.tiles_y );
      b = static_cast< int >( r / a.tiles_y );
      x0 = txi * TX;
      y0 = tyi * TY;
   };
   auto issue = [ & ]( int64_t t, int st ) {
      int x0, y0, b;
      geometry( t, x0, y0, b );
      unsigned char* const sp = stages + st * G::STAGE_STRIDE;
      mbar_arrive_expect_tx( &full[ st ], G::GBYTES + ( want_sig ? G::XBYTES : 0 ));
      tma_load_4d( sp, &a.tg, &full[ st ], x0 - LEAD, y0 - B, 0, b );
      if( want_sig ) { tma_load_4d( sp + G::GBYTES, &a.tx, &full[ st ], x0, y0, 0, b ); }
   };
   if( lane == 0 ) {
      for( int k = 0; k < SPW; ++k ) {
         int64_t const t = gw + k * nwarps;
         if( t < a.ntiles ) { issue( t, k ); }
      }
   }
   // x value of tile row r, tile column c (zero fill outside the image).
   auto xval = [ & ]( unsigned char const* sp, int r, int c ) -> float {
      return to_f32< TIn >( reinterpret_cast< TIn const* >( sp + G::GBYTES )[ r * TX + c ] );
   };

   uint32_t kdone = 0;
   for( int64_t t = gw; t < a.ntiles; t += nwarps, ++kdone ) {
      int x0, y0, b;
      geometry( t, x0, y0, b );
      int const bx = x0 - LEAD, by = y0 - B;
      int const st = static_cast< int >( kdone % SPW );
      unsigned char* const sp = stages + st * G::STAGE_STRIDE;
      float const* const gbox = reinterpret_cast< float const* >( sp );
      // Fold tables: halo positions j within h of the image whose source lies in this tile.
      int nyf = 0, nxf = 0;
      if( y0 <= B || y0 + TY + B >= ny ) {
         int const hy = a.h[ 1 ];
         int const j = lane < hy ? -hy + lane : ( lane < 2 * hy ? ny + lane - hy : 0 );
         uint32_t ent = 0;
         bool want = lane < 2 * hy && a.bc[ 1 ] != BC_ADD_ZEROS;
         if( want ) {
            bool neg;
            int const m = static_cast< int >( bc_map_index( j, ny, a.bc[ 1 ], &neg ));
            want = m >= y0 && m < y0 + TY && m < ny;
            ent = static_cast< uint32_t >( m - y0 < 0 ? 0 : m - y0 ) | ( static_cast< uint32_t >( j - by ) << 8 ) |
                  ( neg ? 1u << 20 : 0u );
         }
         uint32_t const msk = __ballot_sync( 0xffffffffu, want );
         if( want ) { yfold[ __popc( msk & (( 1u << lane ) - 1u )) ] = ent; }
         nyf = __popc( msk );
      }
      if( x0 <= B || x0 + TX + B >= nx ) {
         int const hx = a.h[ 0 ];
         int const j = lane < hx ? -hx + lane : ( lane < 2 * hx ? nx + lane - hx : 0 );
         uint32_t ent = 0;
         bool want = lane < 2 * hx && a.bc[ 0 ] != BC_ADD_ZEROS;
         if( want ) {
            bool neg;
            int const m = static_cast< int >( bc_map_index( j, nx, a.bc[ 0 ], &neg ));
            want = m >= x0 && m < x0 + TX && m < nx;
            ent = static_cast< uint32_t >( m - x0 < 0 ? 0 : m - x0 ) | ( static_cast< uint32_t >( j - bx ) << 8 ) |
                  ( neg ? 1u << 20 : 0u );
         }
         uint32_t const msk = __ballot_sync( 0xffffffffu, want );
         if( want ) { xfold[ __popc( msk & (( 1u << lane ) - 1u )) ] = ent; }
         nxf = __popc( msk );
      }
      __syncwarp();
      w5_wait( &full[ st ], ( kdone / SPW ) & 1u, abort, a.status );

      // ---- y pass: v = C_y^T y_bar, v' = C'_y^T y_bar (lane -> column pair)
      int const pc = G::P0 + lane;
      if( lane < G::NPAIR ) {
#pragma unroll
         for( int r0 = 0; r0 < TY; r0 += RB ) {
            float2 v[ RB + 2 * B ];
#pragma unroll
            for( int r = 0; r < RB + 2 * B; ++r ) {
               v[ r ] = reinterpret_cast< float2 const* >( gbox )[ ( r0 + r ) * ( BW / 2 ) + pc ];
            }
            float2 o[ RB ], od[ RB ];
#pragma unroll
            for( int t2 = 0; t2 < RB; ++t2 ) {
               float2 acc = fmul2( a.w[ 1 ][ 0 ], v[ t2 + B ] );
               float2 accd = want_sig ? fmul2( a.wd[ 1 ][ 0 ], v[ t2 + B ] ) : make_float2( 0.f, 0.f );
#pragma unroll
               for( int k = 1; k <= B; ++k ) {
                  float2 const ps = ffma2( sy, v[ t2 + B - k ], v[ t2 + B + k ] );
                  acc = ffma2( a.w[ 1 ][ k ], ps, acc );
                  if( want_sig ) { accd = ffma2( a.wd[ 1 ][ k ], ps, accd ); }
               }
               o[ t2 ] = acc;
               od[ t2 ] = accd;
            }
#pragma unroll
            for( int rp = 0; rp < RB / 2; ++rp ) {
               b2[ ( r0 / 2 + rp ) * ( BW / 2 ) + pc ] = make_float4( o[ 2 * rp ].x, o[ 2 * rp + 1 ].x, o[ 2 * rp ].y, o[ 2 * rp + 1 ].y );
               if( want_sig ) {
                  b2d[ ( r0 / 2 + rp ) * ( BW / 2 ) + pc ] =
                        make_float4( od[ 2 * rp ].x, od[ 2 * rp + 1 ].x, od[ 2 * rp ].y, od[ 2 * rp + 1 ].y );
               }
            }
         }
         // y fold: row tr += sign * z(j), z(j) = C_y^T y_bar at halo row j (box row jb)
         for( int e = 0; e < nyf; ++e ) {
            uint32_t const fe = yfold[ e ];
            int const tr = static_cast< int >( fe & 0xffu ), jb = static_cast< int >(( fe >> 8 ) & 0xfffu );
            float const sg = ( fe & ( 1u << 20 )) ? -1.f : 1.f;
            auto row = [ & ]( int r ) -> float2 {
               return ( r >= 0 && r < BH ) ? reinterpret_cast< float2 const* >( gbox )[ r * ( BW / 2 ) + pc ] : make_float2( 0.f, 0.f );
            };
            float2 z = fmul2( a.w[ 1 ][ 0 ], row( jb ));
            float2 zd = want_sig ? fmul2( a.wd[ 1 ][ 0 ], row( jb )) : make_float2( 0.f, 0.f );
            for( int k = 1; k <= B; ++k ) {
               float2 const ps = ffma2( sy, row( jb - k ), row( jb + k ));
               z = ffma2( a.w[ 1 ][ k ], ps, z );
               if( want_sig ) { zd = ffma2( a.wd[ 1 ][ k ], ps, zd ); }
            }
            float* const b2f = reinterpret_cast< float* >( b2 );
            float* const b2df = reinterpret_cast< float* >( b2d );
            int const ia = a2_b2col( tr >> 1, 2 * pc, BW ) * 2 + ( tr & 1 );
            int const ib = a2_b2col( tr >> 1, 2 * pc + 1, BW ) * 2 + ( tr & 1 );
            b2f[ ia ] += sg * z.x;
            b2f[ ib ] += sg * z.y;
            if( want_sig ) {
               b2df[ ia ] += sg * zd.x;
               b2df[ ib ] += sg * zd.y;
            }
         }
      }
      __syncwarp();

      if( want_gx && a.tma_store ) {
         // The previous tile's TMA store has finished reading `ot`.
         if( lane == 0 ) { asm volatile( "cp.async.bulk.wait_group.read 0;" ::: "memory" ); }
         __syncwarp();
      }
      // ---- x pass: lane -> (row pair, strip of SW columns)
      int const rp = lane >> 2, c0 = ( lane & 3 ) * SW;
      constexpr int C0 = B + E;
      {
         float2 const* const bf = reinterpret_cast< float2 const* >( b2 );
         int const pbase = ( LEAD + c0 - B ) >> 1;
         float2 vx[ 2 * NPX ];
#pragma unroll
         for( int m = 0; m < NPX; ++m ) {
            float4 const f = b2[ rp * ( BW / 2 ) + pbase + m ];
            vx[ 2 * m ] = make_float2( f.x, f.y );
            vx[ 2 * m + 1 ] = make_float2( f.z, f.w );
         }
         (void) bf;
         float2 out[ SW ];
#pragma unroll
         for( int c = 0; c < SW; ++c ) {
            float2 acc = fmul2( a.w[ 0 ][ 0 ], vx[ C0 + c ] );
            float2 accd = want_sig ? fmul2( a.wd[ 0 ][ 0 ], vx[ C0 + c ] ) : make_float2( 0.f, 0.f );
#pragma unroll
            for( int k = 1; k <= B; ++k ) {
               float2 const ps = ffma2( sx, vx[ C0 + c - k ], vx[ C0 + c + k ] );
               acc = ffma2( a.w[ 0 ][ k ], ps, acc );
               if( want_sig ) { accd = ffma2( a.wd[ 0 ][ k ], ps, accd ); }
            }
            out[ c ] = acc;
            if( want_sig ) {
               dsx += accd.x * xval( sp, 2 * rp, c0 + c ) + accd.y * xval( sp, 2 * rp + 1, c0 + c );
            }
         }
         if( want_gx ) {
#pragma unroll
            for( int c = 0; c < SW; c += 2 ) {
               *reinterpret_cast< float2* >( ot + ( 2 * rp ) * OTS + c0 + c ) = make_float2( out[ c ].x, out[ c + 1 ].x );
               *reinterpret_cast< float2* >( ot + ( 2 * rp + 1 ) * OTS + c0 + c ) = make_float2( out[ c ].y, out[ c + 1 ].y );
            }
         }
      }
      if( want_sig ) {
         int const pbase = ( LEAD + c0 - B ) >> 1;
         float2 vx[ 2 * NPX ];
#pragma unroll
         for( int m = 0; m < NPX; ++m ) {
            float4 const f = b2d[ rp * ( BW / 2 ) + pbase + m ];
            vx[ 2 * m ] = make_float2( f.x, f.y );
            vx[ 2 * m + 1 ] = make_float2( f.z, f.w );
         }
#pragma unroll
         for( int c = 0; c < SW; ++c ) {
            float2 acc = fmul2( a.w[ 0 ][ 0 ], vx[ C0 + c ] );
#pragma unroll
            for( int k = 1; k <= B; ++k ) {
               float2 const ps = ffma2( sx, vx[ C0 + c - k ], vx[ C0 + c + k ] );
               acc = ffma2( a.w[ 0 ][ k ], ps, acc );
            }
            dsy += acc.x * xval( sp, 2 * rp, c0 + c ) + acc.y * xval( sp, 2 * rp + 1, c0 + c );
         }
      }
      __syncwarp();
      // ---- x fold: lane -> row pair (lanes 0 .. TY/2-1), all fold entries in turn
      if( nxf > 0 && lane < TY / 2 ) {
         int const r2 = lane;
         float2 const* const bv = reinterpret_cast< float2 const* >( b2 );
         float2 const* const bd = reinterpret_cast< float2 const* >( b2d );
         int const clo = 2 * G::P0, chi = 2 * ( G::P0 + G::NPAIR );   // columns the y pass computed
         for( int e = 0; e < nxf; ++e ) {
            uint32_t const fe = xfold[ e ];
            int const tc = static_cast< int >( fe & 0xffu ), jb = static_cast< int >(( fe >> 8 ) & 0xfffu );
            float const sg = ( fe & ( 1u << 20 )) ? -1.f : 1.f;
            auto col = [ & ]( float2 const* src, int c ) -> float2 {
               return ( c >= clo && c < chi && bx + c >= 0 && bx + c < nx ) ? src[ a2_b2col( r2, c, BW ) ] : make_float2( 0.f, 0.f );
            };
            float2 z = fmul2( a.w[ 0 ][ 0 ], col( bv, jb ));
            float2 za = want_sig ? fmul2( a.wd[ 0 ][ 0 ], col( bv, jb )) : make_float2( 0.f, 0.f );
            float2 zc = want_sig ? fmul2( a.w[ 0 ][ 0 ], col( bd, jb )) : make_float2( 0.f, 0.f );
            for( int k = 1; k <= B; ++k ) {
               float2 const ps = ffma2( sx, col( bv, jb - k ), col( bv, jb + k ));
               z = ffma2( a.w[ 0 ][ k ], ps, z );
               if( want_sig ) {
                  za = ffma2( a.wd[ 0 ][ k ], ps, za );
                  float2 const pd = ffma2( sx, col( bd, jb - k ), col( bd, jb + k ));
                  zc = ffma2( a.w[ 0 ][ k ], pd, zc );
               }
            }
            if( want_gx ) {
               ot[ ( 2 * r2 ) * OTS + tc ] += sg * z.x;
               ot[ ( 2 * r2 + 1 ) * OTS + tc ] += sg * z.y;
            }
            if( want_sig ) {
               float const x0v = xval( sp, 2 * r2, tc ), x1v = xval( sp, 2 * r2 + 1, tc );
               dsx += sg * ( za.x * x0v + za.y * x1v );
               dsy += sg * ( zc.x * x0v + zc.y * x1v );
            }
         }
      }
      __syncwarp();
      if( lane == 0 ) {
         // The stage is read: stream this warp's tile SPW ahead into it.
         int64_t const tn = t + SPW * nwarps;
         if( tn < a.ntiles ) { issue( tn, st ); }
      }
      if( want_gx && a.tma_store ) {
         fence_proxy_async();
         __syncwarp();
         if( lane == 0 ) {
            asm volatile( "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
                          :: "l"( reinterpret_cast< uint64_t >( &a.tgx )), "r"( x0 ), "r"( y0 ), "r"( 0 ), "r"( b ),
                             "r"( smem_u32( ot )) : "memory" );
            asm volatile( "cp.async.bulk.commit_group;" ::: "memory" );
         }
      } else if( want_gx ) {
         float* const dst_b = a.gx + static_cast< int64_t >( b ) * a.gb;
#pragma unroll 4
         for( int e = lane; e < TY * ( TX / 2 ); e += 32 ) {
            int const r = e / ( TX / 2 ), cp = e - r * ( TX / 2 );
            int const xo = x0 + 2 * cp, yo = y0 + r;
            if( xo < nx && yo < ny ) {
               float2 const val = *reinterpret_cast< float2 const* >( ot + r * OTS + 2 * cp );
               float* const p = dst_b + static_cast< int64_t >( yo ) * a.gs1 + xo;
               if( xo + 1 < nx && a.vec_store ) {
                  *reinterpret_cast< float2* >( p ) = val;
               } else {
                  p[ 0 ] = val.x;
                  if( xo + 1 < nx ) { p[ 1 ] = val.y; }
               }
            }
         }
      }
      __syncwarp();   // ot reads done before the next tile
   }
   if( want_gx && a.tma_store && lane == 0 ) { asm volatile( "cp.async.bulk.wait_group 0;" ::: "memory" ); }
   if( want_sig ) {
      double dx = dsx, dy = dsy;
#pragma unroll
      for( int o = 16; o > 0; o >>= 1 ) {
         dx += __shfl_xor_sync( 0xffffffffu, dx, o );
         dy += __shfl_xor_sync( 0xffffffffu, dy, o );
      }
      if( lane == 0 ) {
         atomicAdd( a.dsig[ 0 ], dx );
         atomicAdd( a.dsig[ 1 ], dy );
      }
   }
}

} // namespace dipcu
