// K1-3D: the fused 3D Gaussian FIR tile kernel for sm_100a (z-marching, TMA-pipelined).
//
// Work: the image is cut into tile columns (64 x 8 outputs in x-y, all of z, per batch image);
// the columns' output planes are split evenly over a persistent grid, so every CTA processes
// one or two contiguous z-chunks.  Per chunk the CTA marches through the input planes
// z - HZ .. z + HZ of its range:
//   1. one thread keeps D planes in flight with TMA tiled loads (box = the tile plus its x-y
//      halo, raw input type) into a ring of shared-memory stages, each completing on its own
//      mbarrier (bounded waits);
//   2. the y pass reads a landed stage, converts to float (exponent-bias insertion for
//      integer input), applies the boundary maps of edge tiles, and writes column pairs of
//      row-pair-interleaved float2s (double-buffered);
//   3. the x pass reads its 2x2 output points' neighbourhood as float4s and filters with packed
//      f32x2 FMAs;
//   4. the z pass keeps the last 2*HZ+1 planes' contributions in a register ring (the plane
//      loop is unrolled by the ring length so slots are static registers) and emits one output
//      plane per input plane.
// One block barrier per plane.  Each input voxel crosses HBM once (its tile's halo re-reads
// hit L2) and each output voxel is written once.
//
// Boundary conditions: x-y halos outside the image are either TMA zero fill ("add zeros"), or
// remapped inside the staged box ("mirror", "asym mirror", "zero order": the source of every
// halo sample of an edge tile lies in the box), or -- for "periodic" / "asym periodic" edge
// tiles -- gathered with plain loads.  z uses the mapped plane index as the TMA coordinate.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"
#include "fused.cuh"
#include "tma.cuh"

namespace dipcu {

struct Z3Args {
   CUtensorMap tmap;        // 4D (x, y, z, batch) tiled map of the source
   void const* src;
   float* dst;
   int64_t n[ 3 ];
   int64_t ss[ 3 ], ds[ 3 ];
   int64_t nb, sb, db;
   int32_t bc[ 3 ];
   int32_t tiles_x, tiles_y;
   int64_t units;           // tile columns x n[2]: output planes of all tile columns
   int32_t* status;         // set to DIPCU_ERR_TIMEOUT if a wait gives up
   float2 w[ 3 ][ kFusedMaxTaps ];  // per axis (x, y, z), centre first, duplicated for f32x2
};

template< typename TIn, int HX, int HY, int HZ >
struct Z3Geom {
   static constexpr int TX = 64, TY = 8, NT = 128, RY = 4;
   static constexpr int ALIGN = 16 / static_cast< int >( sizeof( TIn ));
   static constexpr int O0 = ( ALIGN - ( HX % ALIGN )) % ALIGN;      // box column of x0 - HX
   static constexpr int WXA = ( O0 + TX + 2 * HX + ALIGN - 1 ) / ALIGN * ALIGN;
   static constexpr int WY = TY + 2 * HY;
   static constexpr int NPAIR = TX / 2 + HX;                         // y-pass column pairs
   static constexpr int B2COLS = 2 * NPAIR;
   static constexpr int STAGE_BYTES = WXA * WY * static_cast< int >( sizeof( TIn ));
   static constexpr int STAGE_STRIDE = ( STAGE_BYTES + 127 ) / 128 * 128;
   // Planes in flight: about 48 KB of stages per CTA, between 3 and 8.
   static constexpr int D = ( 49152 / STAGE_STRIDE ) > 8 ? 8 : (( 49152 / STAGE_STRIDE ) < 3 ? 3 : ( 49152 / STAGE_STRIDE ));
   static constexpr int B2_FLOATS = ( TY / 2 ) * B2COLS * 2;
   static constexpr int OFF_B2 = D * STAGE_STRIDE;
   static constexpr int OFF_MAPS = OFF_B2 + 2 * B2_FLOATS * 4;
   static constexpr int OFF_GATHER = ( OFF_MAPS + ( WY + WXA ) * 2 + WY + WXA + 15 ) / 16 * 16;  // int32 gather rows/cols
   static constexpr int OFF_BAR = ( OFF_GATHER + ( WY + WXA ) * 4 + 15 ) / 16 * 16;
   static constexpr int OFF_RING = OFF_BAR + D * 8 + 16;                   // + fix-up list count
   static constexpr int RING_FLOATS = ( 2 * HZ + 1 ) * NT * 4;             // x-pass outputs per plane of a group
   static constexpr int OFF_FIX = OFF_RING + RING_FLOATS * 4;
   static constexpr int FIX_MAX = WY * ( TX + 2 * HX );                    // halo fix-up entries
   static constexpr int BYTES = OFF_FIX + FIX_MAX * 8;
   static_assert( TY % RY == 0 && RY % 2 == 0, "row blocks" );
   static_assert(( TX / 2 ) * ( TY / 2 ) == NT, "one 2x2 point group per thread" );
   static_assert( STAGE_BYTES % 16 == 0, "TMA box size" );
   static_assert( OFF_B2 % 16 == 0 && OFF_MAPS % 16 == 0 && OFF_GATHER % 16 == 0 && OFF_BAR % 16 == 0 &&
                  OFF_RING % 16 == 0 && OFF_FIX % 16 == 0,
                  "shared-memory sections must be 16-byte aligned" );
   static_assert(( B2_FLOATS * 4 ) % 16 == 0 && ( B2COLS * 2 * 4 ) % 16 == 0, "float4 accesses of B2" );
};

__device__ __forceinline__ float2 ffma2( float2 a, float2 b, float2 c ) { return __ffma2_rn( a, b, c ); }
__device__ __forceinline__ float2 fadd2( float2 a, float2 b ) { return __fadd2_rn( a, b ); }
__device__ __forceinline__ float2 fsub2( float2 a, float2 b ) { return __fadd2_rn( a, make_float2( -b.x, -b.y )); }
__device__ __forceinline__ float2 fmul2( float2 a, float2 b ) { return __fmul2_rn( a, b ); }

// Pair of raw samples of stage row r at box columns (O0 + 2 pair, O0 + 2 pair + 1), as float.
template< typename TIn >
struct PairLoader;

template<>
struct PairLoader< uint16_t > {
   template< int WXA, int O0 >
   static __device__ __forceinline__ float2 load( unsigned char const* stage, int r, int pair ) {
      // box columns O0 + 2 pair, O0 + 2 pair + 1
      uint32_t const* row = reinterpret_cast< uint32_t const* >( stage ) + r * ( WXA / 2 );
      uint32_t lo, hi;
      if( O0 % 2 == 0 ) {
         uint32_t w = row[ O0 / 2 + pair ];
         lo = __byte_perm( w, 0x4B000000u, 0x7610 );
         hi = __byte_perm( w, 0x4B000000u, 0x7632 );
      } else {
         uint32_t w0 = row[ ( O0 - 1 ) / 2 + pair ];
         uint32_t w1 = row[ ( O0 + 1 ) / 2 + pair ];
         lo = __byte_perm( w0, 0x4B000000u, 0x7632 );
         hi = __byte_perm( w1, 0x4B000000u, 0x7610 );
      }
      return fadd2( make_float2( __uint_as_float( lo ), __uint_as_float( hi )), make_float2( -8388608.0f, -8388608.0f ));
   }
   static __device__ __forceinline__ float one( unsigned char const* stage, int idx ) {
      return to_f32< uint16_t >( reinterpret_cast< uint16_t const* >( stage )[ idx ] );
   }
};

template<>
struct PairLoader< float > {
   template< int WXA, int O0 >
   static __device__ __forceinline__ float2 load( unsigned char const* stage, int r, int pair ) {
      float const* row = reinterpret_cast< float const* >( stage ) + r * WXA;
      if( O0 % 2 == 0 ) {
         return *reinterpret_cast< float2 const* >( row + O0 + 2 * pair );
      }
      return make_float2( row[ O0 + 2 * pair ], row[ O0 + 2 * pair + 1 ] );
   }
   static __device__ __forceinline__ float one( unsigned char const* stage, int idx ) {
      return reinterpret_cast< float const* >( stage )[ idx ];
   }
};

template< typename TIn, int HX, int HY, int HZ, bool OX, bool OY, bool OZ >
__global__ void __launch_bounds__( 128 ) fused3d_tma_kernel( Z3Args const __grid_constant__ a ) {
   using G = Z3Geom< TIn, HX, HY, HZ >;
   constexpr int M = 2 * HZ + 1;
   constexpr int TX = G::TX, TY = G::TY, D = G::D, RY = G::RY, WXA = G::WXA, WY = G::WY, NT = G::NT;
   constexpr int NC = TX + 2 * HX;                          // box columns the passes read
   constexpr bool kUnsigned = !std::is_same< TIn, float >::value;
   extern __shared__ __align__( 128 ) unsigned char smem[];
   unsigned char* stage = smem;
   float* B2 = reinterpret_cast< float* >( smem + G::OFF_B2 );
   int16_t* rmap = reinterpret_cast< int16_t* >( smem + G::OFF_MAPS );
   int16_t* cmap = rmap + WY;
   uint8_t* rfl = reinterpret_cast< uint8_t* >( cmap + WXA );
   uint8_t* cfl = rfl + WY;
   int32_t* grow = reinterpret_cast< int32_t* >( smem + G::OFF_GATHER );
   int32_t* gcol = grow + WY;
   uint64_t* bars = reinterpret_cast< uint64_t* >( smem + G::OFF_BAR );
   int* fix_count = reinterpret_cast< int* >( smem + G::OFF_BAR + D * 8 );
   float4* ring_in = reinterpret_cast< float4* >( smem + G::OFF_RING );   // [M][NT]
   uint32_t* fix = reinterpret_cast< uint32_t* >( smem + G::OFF_FIX );     // dst | src << 16 (+ flags in 2 words)

   int const tid = static_cast< int >( threadIdx.x );
   if( tid == 0 ) {
      for( int d = 0; d < D; ++d ) { mbar_init( &bars[ d ], 1 ); }
      fence_mbar_init();
   }
   __syncthreads();

   int64_t const nx = a.n[ 0 ], ny = a.n[ 1 ], nz = a.n[ 2 ];
   int64_t const ub = ( static_cast< int64_t >( blockIdx.x ) * a.units ) / gridDim.x;
   int64_t const ue = ( static_cast< int64_t >( blockIdx.x + 1 ) * a.units ) / gridDim.x;
   int const cp = tid % ( TX / 2 );   // column pair of this thread's 2x2 output group
   int const rp = tid / ( TX / 2 );   // row pair
   uint32_t phase = 0;                // bit d: parity of the next completion of stage d
   int64_t g = 0;                     // planes staged by this CTA so far (stage = g % D)

   for( int64_t u = ub; u < ue; ) {
      int64_t const tc = u / nz;
      int64_t const zs = u - tc * nz;
      int64_t const ze = ( nz < zs + ( ue - u )) ? nz : zs + ( ue - u );
      u += ze - zs;
      int64_t const txi = tc % a.tiles_x;
      int64_t const tr = tc / a.tiles_x;
      int64_t const tyi = tr % a.tiles_y;
      int64_t const b = tr / a.tiles_y;
      int64_t const x0 = txi * TX, y0 = tyi * TY;
      int32_t const xa = static_cast< int32_t >( x0 - HX - G::O0 );
      int32_t const ya = static_cast< int32_t >( y0 - HY );
      bool const inx = x0 - HX >= 0 && x0 + TX + HX <= nx;
      bool const iny = y0 - HY >= 0 && y0 + TY + HY <= ny;
      bool const interior = inx && iny;
      auto boxlocal = []( int32_t bc ) {
         return bc == BC_SYMMETRIC_MIRROR || bc == BC_ASYMMETRIC_MIRROR || bc == BC_ZERO_ORDER_EXTRAPOLATE || bc == BC_ADD_ZEROS;
      };
      bool gather = !(( inx || boxlocal( a.bc[ 0 ] )) && ( iny || boxlocal( a.bc[ 1 ] )));
      // Edge tiles with an inverting boundary condition on unsigned input keep per-sample maps in
      // the y pass (a negated sample has no unsigned representation in the stage).
      bool const asym_xy = ( !inx && ( a.bc[ 0 ] == BC_ASYMMETRIC_MIRROR || a.bc[ 0 ] == BC_ASYMMETRIC_PERIODIC )) ||
                           ( !iny && ( a.bc[ 1 ] == BC_ASYMMETRIC_MIRROR || a.bc[ 1 ] == BC_ASYMMETRIC_PERIODIC ));
      bool mapped = false;
      if( !interior ) {
         // Boundary maps of the tile.  For "box-local" conditions every halo sample's source lies
         // inside the staged box unless the tile sits far outside a small image; then, as for
         // periodic edges, the tile is staged by plain gathers instead.
         bool bad = false;
         for( int r = tid; r < WY; r += NT ) {
            int64_t yi; uint8_t fl;
            map_coord( ya + r, ny, a.bc[ 1 ], yi, fl );
            int64_t bi = yi - ya;
            bad |= !( fl & 2 ) && ( bi < 0 || bi >= WY );
            rmap[ r ] = static_cast< int16_t >(( bi < 0 || bi >= WY ) ? 0 : bi );
            rfl[ r ] = static_cast< uint8_t >( fl | (( ya + r < 0 || ya + r >= ny ) ? 4 : 0 ));
            grow[ r ] = static_cast< int32_t >( yi );
         }
         for( int c = tid; c < WXA; c += NT ) {
            int64_t xi; uint8_t fl;
            map_coord( xa + c, nx, a.bc[ 0 ], xi, fl );
            int64_t bi = xi - xa;
            bool needed = c >= G::O0 && c < G::O0 + NC;
            bad |= needed && !( fl & 2 ) && ( bi < 0 || bi >= WXA );
            cmap[ c ] = static_cast< int16_t >(( bi < 0 || bi >= WXA ) ? 0 : bi );
            cfl[ c ] = static_cast< uint8_t >( fl | (( xa + c < 0 || xa + c >= nx ) ? 4 : 0 ));
            gcol[ c ] = static_cast< int32_t >( xi );
         }
         if( tid == 0 ) { *fix_count = 0; }
         gather = __syncthreads_or( bad ) || gather;
         mapped = !gather && kUnsigned && asym_xy;
         if( !gather && !mapped ) {
            // Compact list of the box samples outside the image that the passes read, with the
            // in-box sample each copies (and whether it is zero or negated).
            for( int e = tid; e < WY * NC; e += NT ) {
               int r = e / NC;
               int c = G::O0 + ( e - r * NC );
               if(( rfl[ r ] | cfl[ c ] ) & 4 ) {
                  uint32_t dsti = static_cast< uint32_t >( r * WXA + c );
                  uint32_t srci = static_cast< uint32_t >( rmap[ r ] * WXA + cmap[ c ] );
                  uint32_t fl = (( rfl[ r ] | cfl[ c ] ) & 2 ) | (( rfl[ r ] ^ cfl[ c ] ) & 1 );
                  int i = atomicAdd( fix_count, 1 );
                  fix[ 2 * i ] = dsti | ( fl << 16 );
                  fix[ 2 * i + 1 ] = srci;
               }
            }
         }
      }
      int64_t const nplanes = ( ze - zs ) + 2 * HZ;
      auto zcoord = [ & ]( int64_t q, uint8_t& zfl ) -> int32_t {
         int64_t zi;
         map_coord( zs - HZ + q, nz, a.bc[ 2 ], zi, zfl );
         return ( zfl & 2 ) ? -1 : static_cast< int32_t >( zi );   // -1: TMA zero fill
      };
      auto issue = [ & ]( int64_t q ) {
         uint8_t zfl;
         int32_t zc = zcoord( q, zfl );
         int st = static_cast< int >(( g + q ) % D );
         mbar_arrive_expect_tx( &bars[ st ], G::STAGE_BYTES );
         tma_load_4d( stage + st * G::STAGE_STRIDE, &a.tmap, &bars[ st ], xa, ya, zc, static_cast< int32_t >( b ));
      };
      __syncthreads();   // maps and fix-up list visible; previous chunk's stages fully consumed
      int const nfix = ( interior || gather || mapped ) ? 0 : *fix_count;
      if( !gather && tid == 0 ) {
         for( int64_t q = 0; q < nplanes && q < D; ++q ) { issue( q ); }
      }
      int64_t const y_own = y0 + 2 * rp;
      int64_t const x_own = x0 + 2 * cp;
      float* const dst_b = a.dst + b * a.db;

      float2 acc0[ M ], acc1[ M ];   // ring: columns 2cp and 2cp+1, each a (row 2rp, row 2rp+1) pair
#pragma unroll
      for( int sl = 0; sl < M; ++sl ) { acc0[ sl ] = make_float2( 0.f, 0.f ); acc1[ sl ] = acc0[ sl ]; }

#pragma unroll 1
      for( int64_t q0 = 0; q0 < nplanes; q0 += M ) {
         int const jn = static_cast< int >(( nplanes - q0 ) < M ? ( nplanes - q0 ) : M );
         // ---- in-plane passes of up to M planes; x-pass outputs go to this thread's ring_in slots
#pragma unroll 1
         for( int j = 0; j < jn; ++j ) {
            int64_t const q = q0 + j;
            int const sidx = static_cast< int >(( g + q ) % D );
            unsigned char* st = stage + sidx * G::STAGE_STRIDE;
            bool timed_out = false;
            uint8_t zfl;
            int32_t const zc = zcoord( q, zfl );
            if( gather ) {
               // Plain-load staging of an edge tile whose halo sources leave the box.
               TIn const* src = static_cast< TIn const* >( a.src ) + b * a.sb + ( zc < 0 ? 0 : zc ) * a.ss[ 2 ];
               TIn* dstg = reinterpret_cast< TIn* >( st );
               for( int e = tid; e < WY * WXA; e += NT ) {
                  int r = e / WXA, c = e - r * WXA;
                  bool zero = ( zfl & 2 ) || (( rfl[ r ] | cfl[ c ] ) & 2 );
                  dstg[ e ] = zero ? TIn( 0 ) : src[ static_cast< int64_t >( grow[ r ] ) * a.ss[ 1 ] + gcol[ c ] ];
               }
               __syncthreads();
            } else {
               timed_out = !mbar_wait( &bars[ sidx ], ( phase >> sidx ) & 1u );
               phase ^= 1u << sidx;
               if( nfix > 0 ) {
                  TIn* sv = reinterpret_cast< TIn* >( st );
                  for( int i = tid; i < nfix; i += NT ) {
                     uint32_t d0 = fix[ 2 * i ];
                     TIn v = sv[ fix[ 2 * i + 1 ] ];
                     if( d0 & ( 2u << 16 )) { v = TIn( 0 ); }
                     else if( d0 & ( 1u << 16 )) { v = -v; }   // float input only (see `mapped`)
                     sv[ d0 & 0xffffu ] = v;
                  }
                  timed_out = __syncthreads_or( timed_out );
               }
            }
            // ---- y pass: column pairs x row blocks -> B2[q & 1]
            float* b2 = B2 + ( q & 1 ) * G::B2_FLOATS;
            constexpr int NYB = TY / RY;
#pragma unroll 1
            for( int item = tid; item < G::NPAIR * NYB; item += NT ) {
               int const pr = item % G::NPAIR;
               int const yb = item / G::NPAIR;
               float2 v[ RY + 2 * HY ];
               if( !mapped ) {
#pragma unroll
                  for( int i = 0; i < RY + 2 * HY; ++i ) {
                     v[ i ] = PairLoader< TIn >::template load< WXA, G::O0 >( st, yb * RY + i, pr );
                  }
               } else {
#pragma unroll
                  for( int i = 0; i < RY + 2 * HY; ++i ) {
                     int const r = yb * RY + i;
                     int const c = G::O0 + 2 * pr;
                     int const rr = rmap[ r ];
                     uint8_t const rf = rfl[ r ];
                     float e0 = 0.f, e1 = 0.f;
                     if( !(( rf | cfl[ c ] ) & 2 )) {
                        e0 = PairLoader< TIn >::one( st, rr * WXA + cmap[ c ] );
                        if(( rf ^ cfl[ c ] ) & 1 ) { e0 = -e0; }
                     }
                     if( !(( rf | cfl[ c + 1 ] ) & 2 )) {
                        e1 = PairLoader< TIn >::one( st, rr * WXA + cmap[ c + 1 ] );
                        if(( rf ^ cfl[ c + 1 ] ) & 1 ) { e1 = -e1; }
                     }
                     v[ i ] = make_float2( e0, e1 );
                  }
               }
               float2 o[ RY ];
#pragma unroll
               for( int t = 0; t < RY; ++t ) {
                  float2 acc = OY ? make_float2( 0.f, 0.f ) : fmul2( a.w[ 1 ][ 0 ], v[ t + HY ] );
#pragma unroll
                  for( int k = 1; k <= HY; ++k ) {
                     float2 pairsum = OY ? fsub2( v[ t + HY + k ], v[ t + HY - k ] ) : fadd2( v[ t + HY + k ], v[ t + HY - k ] );
                     acc = ffma2( a.w[ 1 ][ k ], pairsum, acc );
                  }
                  o[ t ] = acc;
               }
#pragma unroll
               for( int t = 0; t < RY; t += 2 ) {
                  int const rowpair = ( yb * RY + t ) / 2;
                  *reinterpret_cast< float4* >( b2 + ( rowpair * G::B2COLS + 2 * pr ) * 2 ) =
                        make_float4( o[ t ].x, o[ t + 1 ].x, o[ t ].y, o[ t + 1 ].y );
               }
            }
            timed_out = __syncthreads_or( timed_out );
            if( timed_out ) {
               if( tid == 0 ) { atomicExch( a.status, DIPCU_ERR_TIMEOUT ); }
               return;
            }
            // Stage sidx is free: refill it with the plane D ahead.
            if( !gather && tid == 0 && q + D < nplanes ) { issue( q + D ); }
            // ---- x pass: 2x2 points (rows 2rp, 2rp+1; columns 2cp, 2cp+1)
            float2 vx[ 2 * HX + 2 ];
            float4 const* row = reinterpret_cast< float4 const* >( b2 + ( rp * G::B2COLS + 2 * cp ) * 2 );
#pragma unroll
            for( int m = 0; m < HX + 1; ++m ) {
               float4 f = row[ m ];
               vx[ 2 * m ] = make_float2( f.x, f.y );
               vx[ 2 * m + 1 ] = make_float2( f.z, f.w );
            }
            float2 out[ 2 ];
#pragma unroll
            for( int e = 0; e < 2; ++e ) {
               float2 acc = OX ? make_float2( 0.f, 0.f ) : fmul2( a.w[ 0 ][ 0 ], vx[ e + HX ] );
#pragma unroll
               for( int k = 1; k <= HX; ++k ) {
                  float2 pairsum = OX ? fsub2( vx[ e + HX + k ], vx[ e + HX - k ] ) : fadd2( vx[ e + HX + k ], vx[ e + HX - k ] );
                  acc = ffma2( a.w[ 0 ][ k ], pairsum, acc );
               }
               out[ e ] = acc;
            }
            if( zfl & 1 ) {
               out[ 0 ] = make_float2( -out[ 0 ].x, -out[ 0 ].y );
               out[ 1 ] = make_float2( -out[ 1 ].x, -out[ 1 ].y );
            }
            ring_in[ j * NT + tid ] = make_float4( out[ 0 ].x, out[ 0 ].y, out[ 1 ].x, out[ 1 ].y );
         }
         // ---- z ring over the group (unrolled: slots are static registers).  Plane q feeds
         // outputs t = q - d (d = 0 .. 2HZ) at z offset d - HZ; output q - 2HZ completes.
#pragma unroll
         for( int j = 0; j < M; ++j ) {
            if( j >= jn ) { break; }
            int64_t const q = q0 + j;
            float4 const vin = ring_in[ j * NT + tid ];
            float2 const o0 = make_float2( vin.x, vin.y ), o1 = make_float2( vin.z, vin.w );
#pragma unroll
            for( int d = 0; d <= 2 * HZ; ++d ) {
               int const slot = ( j - d + M ) % M;
               int const kk = d - HZ;
               int const ak = kk < 0 ? -kk : kk;
               if( OZ && kk == 0 ) { continue; }
               float2 const c = ( OZ && kk < 0 ) ? make_float2( -a.w[ 2 ][ ak ].x, -a.w[ 2 ][ ak ].y ) : a.w[ 2 ][ ak ];
               if( d == 0 ) {
                  acc0[ slot ] = fmul2( c, o0 );
                  acc1[ slot ] = fmul2( c, o1 );
               } else {
                  acc0[ slot ] = ffma2( c, o0, acc0[ slot ] );
                  acc1[ slot ] = ffma2( c, o1, acc1[ slot ] );
               }
            }
            int64_t const to = q - 2 * HZ;
            if( to >= 0 && to < ze - zs ) {
               float2 const r0 = acc0[ ( j + 1 ) % M ];
               float2 const r1 = acc1[ ( j + 1 ) % M ];
               int64_t const z = zs + to;
               float* base = dst_b + z * a.ds[ 2 ];
#pragma unroll
               for( int e = 0; e < 2; ++e ) {
                  int64_t const y = y_own + e;
                  if( y < ny && x_own < nx ) {
                     float2 val = e == 0 ? make_float2( r0.x, r1.x ) : make_float2( r0.y, r1.y );
                     float* p = base + y * a.ds[ 1 ] + x_own;
                     if( x_own + 1 < nx && ( reinterpret_cast< uintptr_t >( p ) & 7 ) == 0 ) {
                        *reinterpret_cast< float2* >( p ) = val;
                     } else {
                        p[ 0 ] = val.x;
                        if( x_own + 1 < nx ) { p[ 1 ] = val.y; }
                     }
                  }
               }
            }
         }
      }
      g += nplanes;
   }
}

} // namespace dipcu
