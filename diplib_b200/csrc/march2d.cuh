// K1-2D, row march: the fused 2D Gaussian FIR kernel for sm_100a (single images and batches).
//
// Work item: a strip of TX = 128 output columns of one 2D image and a run of its rows [ya, yb).
// A CTA takes items one after the other (from a static list, or from a device work queue) and
// marches down the item's rows in steps of R = 24 input rows:
//   * x phase: the step's R input rows (the strip plus LEAD columns of halo on each side) land in
//     one of two shared-memory stages by TMA -- one box, or one box per row where rows lie outside
//     the image (the boundary condition's source row, or TMA zero fill for "add zeros") -- and are
//     filtered along x into a ring of x-filtered rows (each warp a row, each lane 4 outputs from
//     aligned float4 windows, taps in tap quads broadcast from shared memory);
//   * y phase: one step behind the rows it needs, the ring's rows are filtered along y into R output
//     rows (each thread a column pair and R / 4 rows with packed f32x2 FMAs, taps in blocks of 8,
//     R / 4 + 7 ring rows per block loaded ahead of the block's FMAs)
//     and stored straight to global memory (each warp 64 consecutive columns: 256-byte rows).
// One __syncthreads per step (x-phase results visible to the y phase); the ring of 128 rows holds
// at least (D + 2) R (D = ceil(2 hy / R)), so that a step's x phase never overwrites rows an earlier
// step's y phase may still read.  The next-but-one step's TMA goes out as soon as a stage is free.  Each input pixel
// crosses HBM once (the x-halo columns of neighbouring strips hit L2) and each output pixel is
// written once; the only recomputation is the x phase of the 2 hy rows of halo at the start of each
// item's row run.
//
// Half-widths up to 32 on each axis, runtime taps: the x filter is padded to the TMA granule
// LEAD >= hx on both sides (the x phase compiled per LEAD), the y filter to a multiple of 8 taps
// (the y phase compiled per number of tap blocks; the last block cut at 2 hy, so that no row beyond
// the filter's support is read).  Boundary conditions in x:
// every index-mapping one ("mirror", "asym mirror", "periodic", "asym periodic", "zero order") and
// "add zeros": halo columns outside the image are rewritten in the stage from their source column
// (a copy inside the box, or a load from the image where the source lies outside it), sign
// included; in y the same conditions through the rows' source coordinates and a per-row sign.
// These are the conditions whose extension of the x-filtered image equals the x-filtering of the
// extended input, which is what lets the two passes fuse (DIPlib extends each intermediate line
// itself, src/library/framework_separable.cpp:354-419).
#pragma once

#include <cuda.h>
#include <stdint.h>

#include <type_traits>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"
#include "tma.cuh"

namespace dipcu {

constexpr int kM2TX = 128;          // output columns per strip
constexpr int kM2R = 24;            // rows per step (and per y-phase block)
constexpr int kM2RT = kM2R / 4;     // output rows per thread in the y phase (a column pair per thread)
constexpr int kM2NT = 256;          // threads per CTA
constexpr int kM2MaxH = 32;         // largest half-width along either axis
constexpr int kM2MaxLead = 32;      // LEAD for hx = 32
constexpr int kM2MaxBW = kM2TX + 2 * kM2MaxLead;
constexpr int kM2Ring = 128;        // ring rows (a power of two >= (D + 2) R for every hy <= 32)
static_assert(( 2 + ( 2 * kM2MaxH + kM2R - 1 ) / kM2R ) * kM2R <= kM2Ring, "ring holds (D + 2) R rows" );
constexpr int kM2MaxFix = 2 * kM2MaxLead;
constexpr int kM2WxLen = 4 + 2 * kM2MaxLead + 8;   // 4 leading zeros, 2 LEAD + 1 taps, zero tail
constexpr int kM2WyLen = 9 * 8;      // 9 blocks of 8 taps (2 hy + 1 <= 65), as duplicated pairs

// One image of a launch.  `tmap` boxes are (bw, R) for the interior steps, `tmap1` (bw, 1) for
// rows at the image's edges; both 4D (x, y, 1, b).
struct alignas( 64 ) M2Image {
   CUtensorMap tmap;
   CUtensorMap tmap1;
   void const* src;           // the source (for gathers of x-halo columns whose source lies outside the box)
   int64_t ss1, ssb;          // source row and batch strides (samples)
   float* dst;
   int64_t ds1, dsb;          // destination row and batch strides
   int32_t nx, ny;
   int32_t bc[ 2 ];
   int32_t h[ 2 ];
   int32_t odd[ 2 ];
   int32_t lead;              // box columns before the strip (multiple of the TMA granule, >= h[0])
   int32_t bw;                // box width = 128 + 2 lead
   int32_t vec_out;           // destination rows take float2 stores (8-byte aligned origin, even row stride)
   int32_t tma;               // 1: stages filled by TMA; 0 (float images whose rows TMA cannot address):
                              // by per-thread 4-byte asynchronous copies
   float const* w[ 2 ];       // half kernels (centre first, h + 1 taps) in device memory; null: M2Args::w0
};

struct M2Item {
   int32_t img;               // image index (or batch index for a single image)
   int32_t x0;                // first output column of the strip
   int32_t ya, yb;            // output rows
};

struct M2Args {
   M2Image img0;              // the image of a single-image launch (images == nullptr)
   M2Image const* images;     // per-image table of a batch launch
   M2Item const* items;       // item list (batch); null: items from the single image's geometry
   int32_t nitems;
   int32_t nimages;           // entries of `images`
   int32_t* queue;            // device work counter (batch; zero before the launch); null: static
   int32_t* status;
   uint32_t wait_limit;       // polls before a wait for a copy gives up (0: kWaitLimit)
   int32_t stall_copies;      // test hook: the copies are announced but never issued, so every wait
                              // for one gives up (nothing is ever in flight)
   // single-image geometry: items = nb x strips x chunks, chunk = `lchunk` rows
   int32_t nb, strips, chunks, lchunk;
   float w0[ 2 ][ kM2MaxH + 1 ];   // single-image half kernels (x, y), centre first
};

struct M2Smem {
   static constexpr int STAGE_BYTES = kM2R * kM2MaxBW * 4;                       // float stage (u16 uses half)
   static constexpr int OFF_STAGE = 0;
   static constexpr int OFF_RING = OFF_STAGE + 2 * STAGE_BYTES;
   static constexpr int OFF_WX = OFF_RING + kM2Ring * kM2TX * 4;
   static constexpr int OFF_WY = OFF_WX + kM2WxLen * 4;
   static constexpr int OFF_ROWS = OFF_WY + kM2WyLen * 8;                        // [2][R] source row, [2][R] sign
   static constexpr int OFF_FIX = OFF_ROWS + 4 * kM2R * 4;                       // [kM2MaxFix] fix entries
   static constexpr int OFF_MISC = OFF_FIX + kM2MaxFix * 8;                      // 16 ints
   static constexpr int OFF_BAR = ( OFF_MISC + 64 + 15 ) / 16 * 16;
   static constexpr int BYTES = OFF_BAR + 4 * 8;                                // TMA and copy barriers per stage
   static_assert( OFF_RING % 128 == 0 && STAGE_BYTES % 128 == 0, "TMA destinations 128-byte aligned" );
   static_assert( OFF_WX % 16 == 0 && OFF_WY % 16 == 0, "float4 weight reads" );
   static_assert( BYTES <= 113 * 1024, "two CTAs per SM" );
};

// Column fix entry: destination box column, source (box column, or image column for a gather),
// flags.
struct M2Fix {
   int16_t dst;
   int16_t flags;             // bit 0: negate; bit 1: source is an image column (gather); bit 2: zero
   int32_t src;
};

template< typename TIn >
__device__ __forceinline__ float4 m2_load4( unsigned char const* stage, int rs, int row, int col ) {
   if constexpr( std::is_same< TIn, float >::value ) {
      return *reinterpret_cast< float4 const* >( stage + ( static_cast< size_t >( row ) * rs + col ) * 4 );
   } else {
      uint2 const u = *reinterpret_cast< uint2 const* >( stage + ( static_cast< size_t >( row ) * rs + col ) * 2 );
      // uint16 -> float exactly: the sample placed in the low mantissa bits of 2^23, minus 2^23.
      float4 r;
      r.x = __uint_as_float( __byte_perm( u.x, 0x4B000000u, 0x7610 )) - 8388608.0f;
      r.y = __uint_as_float( __byte_perm( u.x, 0x4B000000u, 0x7632 )) - 8388608.0f;
      r.z = __uint_as_float( __byte_perm( u.y, 0x4B000000u, 0x7610 )) - 8388608.0f;
      r.w = __uint_as_float( __byte_perm( u.y, 0x4B000000u, 0x7632 )) - 8388608.0f;
      return r;
   }
}

template< typename TIn >
__device__ __forceinline__ float m2_get( unsigned char const* stage, int rs, int row, int col ) {
   if constexpr( std::is_same< TIn, float >::value ) {
      return reinterpret_cast< float const* >( stage )[ static_cast< size_t >( row ) * rs + col ];
   } else {
      return static_cast< float >( reinterpret_cast< uint16_t const* >( stage )[ static_cast< size_t >( row ) * rs + col ] );
   }
}

template< typename TIn >
__device__ __forceinline__ void m2_put( unsigned char* stage, int rs, int row, int col, float v ) {
   if constexpr( std::is_same< TIn, float >::value ) {
      reinterpret_cast< float* >( stage )[ static_cast< size_t >( row ) * rs + col ] = v;
   } else {
      reinterpret_cast< uint16_t* >( stage )[ static_cast< size_t >( row ) * rs + col ] = static_cast< uint16_t >( v );
   }
}

// 4-byte asynchronous copy global -> shared; `bytes` 0 writes a zero (the source is not read).
__device__ __forceinline__ void m2_cp4( void* dst, void const* src, int bytes ) {
   asm volatile( "cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"( smem_u32( dst )), "l"( src ), "r"( bytes ) : "memory" );
}

// The mbarrier's pending count drops when all of this thread's earlier asynchronous copies have
// landed (the barrier's arrival count includes this arrival).
__device__ __forceinline__ void m2_cp_arrive( uint64_t* bar ) {
   asm volatile( "cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" :: "r"( smem_u32( bar )) : "memory" );
}

template< typename TIn >
__device__ __forceinline__ float m2_src_sample( M2Image const& im, int b, int row, int col ) {
   TIn const* p = static_cast< TIn const* >( im.src ) + static_cast< int64_t >( b ) * im.ssb +
                  static_cast< int64_t >( row ) * im.ss1 + col;
   return static_cast< float >( *p );
}

// x phase of one step for LEAD = 4 LQ: warp w filters stage rows w, w + 8, w + 16; lane l the
// outputs 4 l .. 4 l + 3 from the aligned window of 4 + 2 LEAD samples (1 + 2 LQ float4s).  The
// sample at window offset 4 m + e feeds output t with tap d = 4 m + e - t - LEAD; pairs with
// |d| > LEAD (the window's corners) are skipped at compile time, so each output takes 2 LEAD + 1
// FMAs (taps beyond hx are zero).
template< typename TIn, int LQ, int HX = 4 * LQ >
__device__ __forceinline__ void m2_xphase( unsigned char const* stage, int rs, int warp, int lane, float const* wx,
                                           float ( &acc )[ kM2R / 8 ][ 4 ] ) {
   constexpr int RW = kM2R / 8, NQ = 1 + 2 * LQ, LEAD = 4 * LQ;
   static_assert( HX <= LEAD, "the window holds the taps" );
   int const cb = 4 * lane;
#pragma unroll
   for( int m = 0; m < NQ; ++m ) {
      float4 const wl = *reinterpret_cast< float4 const* >( wx + 4 * m );
      float4 const wh = *reinterpret_cast< float4 const* >( wx + 4 * m + 4 );
      float const wv[ 8 ] = { wl.x, wl.y, wl.z, wl.w, wh.x, wh.y, wh.z, wh.w };
#pragma unroll
      for( int i = 0; i < RW; ++i ) {
         float4 const q = m2_load4< TIn >( stage, rs, warp + 8 * i, cb + 4 * m );
         float const qv[ 4 ] = { q.x, q.y, q.z, q.w };
#pragma unroll
         for( int e = 0; e < 4; ++e ) {
#pragma unroll
            for( int t = 0; t < 4; ++t ) {
               int const d = 4 * m + e - t - LEAD;
               if( d < -HX || d > HX ) { continue; }   // taps beyond hx are zero: skipped at compile time
               acc[ i ][ t ] = fmaf( wv[ 4 + e - t ], qv[ e ], acc[ i ][ t ] );   // wx[4 + 4m + e - t]
            }
         }
      }
   }
}

// y phase of one block for NYB tap blocks of 8, on column pairs with packed f32x2 FMAs: the
// thread's columns 2 cp, 2 cp + 1, output rows t0 .. t0 + RT - 1 (item offsets), from ring rows
// t0 + k, k in [0, 8 NYB); the last block reads only the rows up to t0 + RT - 1 + 2 hy (zeros
// beyond: `nlast` rows), so no row outside the filter's support is read.  Taps are duplicated pairs
// (w, w).  Ring rows are slots modulo kM2Ring; a block whose rows do not wrap reads them at immediate
// offsets.
template< int NYB >
__device__ __forceinline__ void m2_yphase( float const* ring, float2 const* wy2, int cp, int t0, int nlast,
                                           float2 ( &acc )[ kM2RT ] ) {
   constexpr int RT = kM2RT, NU = RT + 7, TX = kM2TX;
#pragma unroll
   for( int kb = 0; kb < NYB; ++kb ) {
      float2 wv[ 8 ];
#pragma unroll
      for( int h = 0; h < 4; ++h ) {
         float4 const w4 = *reinterpret_cast< float4 const* >( wy2 + 8 * kb + 2 * h );
         wv[ 2 * h ] = make_float2( w4.x, w4.y );
         wv[ 2 * h + 1 ] = make_float2( w4.z, w4.w );
      }
      int const sb = ( t0 + 8 * kb ) & ( kM2Ring - 1 );
      float2 v[ NU ];
      bool const last = kb == NYB - 1;
      if( sb + NU <= kM2Ring ) {
         float2 const* p = reinterpret_cast< float2 const* >( ring + sb * TX ) + cp;
#pragma unroll
         for( int u = 0; u < NU; ++u ) { v[ u ] = ( !last || u < nlast ) ? p[ u * ( TX / 2 ) ] : make_float2( 0.f, 0.f ); }
      } else {
#pragma unroll
         for( int u = 0; u < NU; ++u ) {
            v[ u ] = ( !last || u < nlast ) ? reinterpret_cast< float2 const* >( ring + (( sb + u ) & ( kM2Ring - 1 )) * TX )[ cp ]
                                            : make_float2( 0.f, 0.f );
         }
      }
#pragma unroll
      for( int u = 0; u < NU; ++u ) {
#pragma unroll
         for( int t = 0; t < RT; ++t ) {
            int const k = u - t;
            if( k >= 0 && k < 8 ) { acc[ t ] = __ffma2_rn( wv[ k ], v[ u ], acc[ t ] ); }
         }
      }
   }
}

template< typename TIn >
__global__ void __launch_bounds__( kM2NT, 2 ) march2d_kernel( M2Args const __grid_constant__ a ) {
   constexpr int R = kM2R, TX = kM2TX, NT = kM2NT;
   extern __shared__ __align__( 128 ) unsigned char smem[];
   unsigned char* const stages = smem + M2Smem::OFF_STAGE;
   float* const ring = reinterpret_cast< float* >( smem + M2Smem::OFF_RING );
   float* const wx = reinterpret_cast< float* >( smem + M2Smem::OFF_WX );
   float2* const wy2 = reinterpret_cast< float2* >( smem + M2Smem::OFF_WY );
   int32_t* const rsrc = reinterpret_cast< int32_t* >( smem + M2Smem::OFF_ROWS );   // [2][R]
   float* const rsgn = reinterpret_cast< float* >( rsrc + 2 * R );                   // [2][R]
   M2Fix* const fix = reinterpret_cast< M2Fix* >( smem + M2Smem::OFF_FIX );
   // misc: [0] item, [1] fixes, [2] abort, [4..5] stage row strides, [6..7] stage interior, [8..9] stage first row
   int32_t* const misc = reinterpret_cast< int32_t* >( smem + M2Smem::OFF_MISC );
   uint64_t* const full = reinterpret_cast< uint64_t* >( smem + M2Smem::OFF_BAR );   // [2] TMA, [2] copies
   int const tid = static_cast< int >( threadIdx.x );
   int const warp = tid >> 5, lane = tid & 31;

   // Stages and ring start as zeros (never uninitialised bits), then the barriers.
   for( int i = tid; i < M2Smem::OFF_WX / 16; i += NT ) { reinterpret_cast< float4* >( smem )[ i ] = make_float4( 0.f, 0.f, 0.f, 0.f ); }
   if( tid == 0 ) {
      mbar_init( &full[ 0 ], 1 );
      mbar_init( &full[ 1 ], 1 );
      mbar_init( &full[ 2 ], NT );               // every thread's copies of a stage
      mbar_init( &full[ 3 ], NT );
      misc[ 2 ] = 0;
      fence_mbar_init();
   }
   __syncthreads();
   uint32_t uses0 = 0, uses1 = 0;       // completed phases per stage (uniform over the CTA)
   uint32_t cuses0 = 0, cuses1 = 0;     // the same for the copy barriers
   uint32_t issued0 = 0, issued1 = 0;   // phases announced per stage (thread 0)
   uint32_t const wait_limit = a.wait_limit ? a.wait_limit : kWaitLimit;
   int volatile* const abort_flag = misc + 2;

   int32_t const total = a.items ? a.nitems : a.nb * a.strips * a.chunks;
   int32_t next = static_cast< int32_t >( blockIdx.x );
   for( ;; ) {
      // ---- next item
      int32_t it;
      if( a.queue ) {
         if( tid == 0 ) { misc[ 0 ] = atomicAdd( a.queue, 1 ); }
         __syncthreads();
         it = misc[ 0 ];
      } else {
         it = next;
         next += static_cast< int32_t >( gridDim.x );
      }
      if( it >= total || *abort_flag ) { break; }
      M2Item item;
      if( a.items ) {
         item = a.items[ it ];
         // An impossible item (a corrupted list) is skipped and reported, never followed.
         bool bad = item.img < 0 || item.img >= a.nimages;
         if( !bad ) {
            M2Image const& ib = a.images[ item.img ];
            bad = item.x0 < 0 || item.x0 >= ib.nx || item.x0 % TX != 0 || item.ya < 0 || item.yb > ib.ny || item.ya >= item.yb;
         }
         if( bad ) {
            if( tid == 0 ) { atomicExch( a.status, DIPCU_ERR_INVALID_ARG ); }
            __syncthreads();                          // every thread has read this item's index
            continue;
         }
      } else {
         int32_t const c = it % a.chunks;
         int32_t const t = it / a.chunks;
         item.x0 = ( t % a.strips ) * TX;
         item.img = t / a.strips;
         item.ya = c * a.lchunk;
         item.yb = min( item.ya + a.lchunk, a.img0.ny );
      }
      M2Image const& im = a.images ? a.images[ item.img ] : a.img0;
      int const b = a.images ? 0 : item.img;          // batch coordinate of a single-image launch
      int const nx = im.nx, ny = im.ny;
      int const hx = im.h[ 0 ], hy = im.h[ 1 ];
      int const lead = im.lead, bw = im.bw;
      int const x0 = item.x0, ya = item.ya, yb = item.yb;
      int const D = ( 2 * hy + R - 1 ) / R;
      int const qtot = yb - ya + 2 * hy;               // input rows of the item
      int const S = ( qtot + R - 1 ) / R;              // x steps
      int const J = ( yb - ya + R - 1 ) / R;           // y blocks
      int const nyb = ( 2 * hy + 1 + 7 ) / 8;          // y tap blocks of 8
      bool const xedge = x0 - lead < 0 || x0 + TX + lead > nx;
      float const sx = im.odd[ 0 ] ? -1.f : 1.f, sy = im.odd[ 1 ] ? -1.f : 1.f;

      // ---- set-up: weights, column fixes (edge strips)
      {
         float const* hwx = im.w[ 0 ] ? im.w[ 0 ] : a.w0[ 0 ];
         float const* hwy = im.w[ 1 ] ? im.w[ 1 ] : a.w0[ 1 ];
         // wx[4 + i], i in [0, 2 lead]: tap d = i - lead (zero beyond hx); wx[0..3] = 0; zero tail.
         for( int i = tid; i < kM2WxLen; i += NT ) {
            int const d = i - 4 - lead;
            float v = 0.f;
            if( i >= 4 && d >= -hx && d <= hx ) { v = d >= 0 ? hwx[ d ] : sx * hwx[ -d ]; }
            wx[ i ] = v;
         }
         // wy2[k] = (w, w), k in [0, 72): tap d = k - hy (zero beyond hy).
         for( int k = tid; k < kM2WyLen; k += NT ) {
            int const d = k - hy;
            float v = 0.f;
            if( d >= -hy && d <= hy ) { v = d >= 0 ? hwy[ d ] : sy * hwy[ -d ]; }
            wy2[ k ] = make_float2( v, v );
         }
         if( xedge && warp == 0 ) {
            int n = 0;
            for( int cc = 0; cc < bw; cc += 32 ) {
               int const c = cc + lane;
               int const xx = x0 - lead + c;
               // columns the stored outputs read (outputs beyond the image are never stored)
               bool want = c < bw && ( xx < 0 || xx >= nx ) && xx >= x0 - hx && xx < min( x0 + TX, nx ) + hx;
               M2Fix f{};
               if( want ) {
                  f.dst = static_cast< int16_t >( c );
                  if( im.bc[ 0 ] == BC_ADD_ZEROS ) {
                     f.flags = 4;
                  } else {
                     bool neg;
                     int const sc = static_cast< int >( bc_map_index( xx, nx, im.bc[ 0 ], &neg ));
                     int const sb = sc - ( x0 - lead );
                     bool const inbox = sb >= 0 && sb < bw && ( x0 - lead + sb ) >= 0 && ( x0 - lead + sb ) < nx;
                     f.flags = static_cast< int16_t >(( neg ? 1 : 0 ) | ( inbox ? 0 : 2 ));
                     f.src = inbox ? sb : sc;
                  }
               }
               uint32_t const m = __ballot_sync( 0xffffffffu, want );
               int const slot = n + __popc( m & (( 1u << lane ) - 1u ));
               if( want && slot < kM2MaxFix ) { fix[ slot ] = f; }
               n += __popc( m );
            }
            if( lane == 0 ) { misc[ 1 ] = n < kM2MaxFix ? n : kM2MaxFix; }
         }
      }
      __syncthreads();
      int const nfix = xedge ? misc[ 1 ] : 0;

      // Issues the TMA load(s) of step s into stage s & 1 and records its rows' sources and signs
      // and the stage's row stride: bw for one box of R rows, bw rounded up to 128 bytes for one
      // box per row (each TMA destination 128-byte aligned).
      auto issue = [ & ]( int s ) {
         int const st = s & 1;
         int const r0 = ya - hy + s * R;                 // absolute row of the step's first row
         unsigned char* const dst = stages + st * M2Smem::STAGE_BYTES;
         uint32_t const row_bytes = static_cast< uint32_t >( bw ) * sizeof( TIn );
         if( st ) { ++issued1; } else { ++issued0; }
         misc[ 8 + st ] = r0;
         if( r0 >= 0 && r0 + R <= ny ) {
            misc[ 6 + st ] = 1;                          // interior: rows r0 .. r0 + R - 1, signs +1
            misc[ 4 + st ] = bw;
            mbar_arrive_expect_tx( &full[ st ], R * row_bytes );
            if( !a.stall_copies ) { tma_load_4d( dst, &im.tmap, &full[ st ], x0 - lead, r0, 0, b ); }
         } else {
            uint32_t const pitch = ( row_bytes + 127u ) / 128u * 128u;
            misc[ 6 + st ] = 0;
            misc[ 4 + st ] = static_cast< int32_t >( pitch / sizeof( TIn ));
            mbar_arrive_expect_tx( &full[ st ], R * row_bytes );
            for( int r = 0; r < R; ++r ) {
               int yy = r0 + r;
               float sg = 1.f;
               if( yy < 0 || yy >= ny ) {
                  if( im.bc[ 1 ] == BC_ADD_ZEROS ) {
                     yy = -1;                           // TMA zero fill
                  } else {
                     bool neg;
                     yy = static_cast< int >( bc_map_index( yy, ny, im.bc[ 1 ], &neg ));
                     sg = neg ? -1.f : 1.f;
                  }
               }
               rsrc[ st * R + r ] = yy;
               rsgn[ st * R + r ] = sg;
               if( !a.stall_copies ) {
                  tma_load_4d( dst + static_cast< size_t >( r ) * pitch, &im.tmap1, &full[ st ], x0 - lead, yy, 0, b );
               }
            }
         }
      };

      // The per-thread copy path: warp w copies rows w, w + 8, w + 16 of step s (lane 0 records each
      // row's source and sign), its lanes the row's columns; columns and "add zeros" rows outside the
      // image become zeros (the column fixes then rewrite the boundary columns).
      bool const tma = im.tma != 0;
      auto copy = [ & ]( int s ) {
         int const st = s & 1;
         int const r0 = ya - hy + s * R;
         float* const dstf = reinterpret_cast< float* >( stages + st * M2Smem::STAGE_BYTES );
         float const* const base = static_cast< float const* >( im.src ) + static_cast< int64_t >( b ) * im.ssb;
#pragma unroll
         for( int i = 0; i < R / 8; ++i ) {
            int const r = warp + 8 * i;
            int yy = r0 + r;
            float sg = 1.f;
            if( yy < 0 || yy >= ny ) {
               if( im.bc[ 1 ] == BC_ADD_ZEROS ) {
                  yy = -1;
               } else {
                  bool neg;
                  yy = static_cast< int >( bc_map_index( yy, ny, im.bc[ 1 ], &neg ));
                  sg = neg ? -1.f : 1.f;
               }
            }
            if( lane == 0 ) { rsrc[ st * R + r ] = yy; rsgn[ st * R + r ] = sg; }
            float const* const srow = base + static_cast< int64_t >( yy < 0 ? 0 : yy ) * im.ss1;
            for( int c = lane; c < bw; c += 32 ) {
               int const xx = x0 - lead + c;
               bool const ok = yy >= 0 && xx >= 0 && xx < nx;
               m2_cp4( dstf + r * bw + c, ok ? srow + xx : base, ok ? 4 : 0 );
            }
         }
         m2_cp_arrive( &full[ 2 + st ] );
      };

      if( tma ) {
         if( tid == 0 ) {
            fence_proxy_async();                      // earlier generic writes to the stages first
            issue( 0 );
            if( S > 1 ) { issue( 1 ); }
         }
      } else {
         copy( 0 );
         if( S > 1 ) { copy( 1 ); }
      }

      int const nsteps = max( S, J + D );
      for( int s = 0; s < nsteps; ++s ) {
         int const st = s & 1;
         unsigned char* const stage = stages + st * M2Smem::STAGE_BYTES;
         if( s < S ) {
            // ---- wait for the step's rows (a give-up is reported and ends the CTA's work at the
            // next barrier; no later copy is issued)
            uint32_t const use = tma ? ( st ? uses1 : uses0 ) : ( st ? cuses1 : cuses0 );
            if( !*abort_flag && !mbar_wait( &full[ tma ? st : 2 + st ], use & 1u, wait_limit )) {
               *abort_flag = 1;
               atomicExch( a.status, DIPCU_ERR_TIMEOUT );
            }
            if( tma ) {
               if( st ) { ++uses1; } else { ++uses0; }
            } else {
               if( st ) { ++cuses1; } else { ++cuses0; }
            }
            int const rs = tma ? misc[ 4 + st ] : bw;     // the stage's row stride (samples)
            bool const interior = tma && misc[ 6 + st ] != 0;
            int const r0s = misc[ 8 + st ];
            if( nfix > 0 ) {
               if( !tma ) { __syncthreads(); }          // every warp's row table of this stage
               // Halo columns outside the image: their source column's sample (sign included).
               for( int e = tid; e < nfix * R; e += NT ) {
                  M2Fix const f = fix[ e % nfix ];
                  int const r = e / nfix;
                  float v = 0.f;
                  if( !( f.flags & 4 )) {
                     if( f.flags & 2 ) {
                        int const yy = interior ? r0s + r : rsrc[ st * R + r ];
                        v = yy >= 0 ? m2_src_sample< TIn >( im, b, yy, f.src ) : 0.f;
                     } else {
                        v = m2_get< TIn >( stage, rs, r, f.src );
                     }
                     if( f.flags & 1 ) { v = -v; }
                  }
                  // In-box sources are interior columns, never rewritten here, so the order of the
                  // rewrites does not matter.
                  m2_put< TIn >( stage, rs, r, f.dst, v );
               }
               __syncthreads();
            }
            // ---- x phase: warp w takes rows w, w + 8, w + 16; lane -> outputs 4 lane .. 4 lane + 3
            {
               constexpr int RW = R / 8;
               float acc[ RW ][ 4 ];
#pragma unroll
               for( int i = 0; i < RW; ++i ) {
#pragma unroll
                  for( int t = 0; t < 4; ++t ) { acc[ i ][ t ] = 0.f; }
               }
               // small half-widths exact (the window's LEAD is rounded up to the TMA granule, the
               // taps beyond hx are not evaluated); from LEAD 16 on the window's taps
               switch( lead == 4 * (( hx + 3 ) / 4 ) && hx <= 12 ? 100 + hx : lead / 4 ) {
                  case 101: m2_xphase< TIn, 1, 1 >( stage, rs, warp, lane, wx, acc ); break;
                  case 102: m2_xphase< TIn, 1, 2 >( stage, rs, warp, lane, wx, acc ); break;
                  case 103: m2_xphase< TIn, 1, 3 >( stage, rs, warp, lane, wx, acc ); break;
                  case 104: m2_xphase< TIn, 1, 4 >( stage, rs, warp, lane, wx, acc ); break;
                  case 105: m2_xphase< TIn, 2, 5 >( stage, rs, warp, lane, wx, acc ); break;
                  case 106: m2_xphase< TIn, 2, 6 >( stage, rs, warp, lane, wx, acc ); break;
                  case 107: m2_xphase< TIn, 2, 7 >( stage, rs, warp, lane, wx, acc ); break;
                  case 108: m2_xphase< TIn, 2, 8 >( stage, rs, warp, lane, wx, acc ); break;
                  case 109: m2_xphase< TIn, 3, 9 >( stage, rs, warp, lane, wx, acc ); break;
                  case 110: m2_xphase< TIn, 3, 10 >( stage, rs, warp, lane, wx, acc ); break;
                  case 111: m2_xphase< TIn, 3, 11 >( stage, rs, warp, lane, wx, acc ); break;
                  case 112: m2_xphase< TIn, 3, 12 >( stage, rs, warp, lane, wx, acc ); break;
                  case 1: m2_xphase< TIn, 1 >( stage, rs, warp, lane, wx, acc ); break;
                  case 2: m2_xphase< TIn, 2 >( stage, rs, warp, lane, wx, acc ); break;
                  case 3: m2_xphase< TIn, 3 >( stage, rs, warp, lane, wx, acc ); break;
                  case 4: m2_xphase< TIn, 4 >( stage, rs, warp, lane, wx, acc ); break;
                  case 5: m2_xphase< TIn, 5 >( stage, rs, warp, lane, wx, acc ); break;
                  case 6: m2_xphase< TIn, 6 >( stage, rs, warp, lane, wx, acc ); break;
                  case 7: m2_xphase< TIn, 7 >( stage, rs, warp, lane, wx, acc ); break;
                  default: m2_xphase< TIn, 8 >( stage, rs, warp, lane, wx, acc ); break;
               }
               int const cb = 4 * lane;
#pragma unroll
               for( int i = 0; i < RW; ++i ) {
                  int const r = warp + 8 * i;
                  int const q = s * R + r;                 // item input row
                  if( q < qtot ) {
                     float4 o = make_float4( acc[ i ][ 0 ], acc[ i ][ 1 ], acc[ i ][ 2 ], acc[ i ][ 3 ] );
                     if( !interior ) {
                        float const sg = rsgn[ st * R + r ];
                        o = make_float4( sg * o.x, sg * o.y, sg * o.z, sg * o.w );
                     }
                     *reinterpret_cast< float4* >( ring + ( q & ( kM2Ring - 1 )) * TX + cb ) = o;
                  }
               }
            }
         }
         __syncthreads();
         if( *abort_flag ) { break; }
         // ---- stage st is free: stream step s + 2 into it
         if( s + 2 < S ) {
            if( !tma ) {
               copy( s + 2 );
            } else if( tid == 0 ) {
               fence_proxy_async();                   // the column fixes' writes before the copy's
               issue( s + 2 );
            }
         }
         // ---- y phase: block j = s - D (output rows ya + jR ..), thread -> column, RT rows
         int const j = s - D;
         if( j >= 0 && j < J ) {
            constexpr int RT = kM2RT;
            int const cp = tid & ( TX / 2 - 1 );          // column pair
            int const g = tid >> 6;                      // row group
            int const t0 = j * R + RT * g;               // item output row offset of the thread's first row
            float2 acc[ RT ];
#pragma unroll
            for( int t = 0; t < RT; ++t ) { acc[ t ] = make_float2( 0.f, 0.f ); }
            // Output row t0 + t needs item input rows t0 + t + k, k in [0, 2 hy].
            int const nlast = RT - 1 + ( 2 * hy + 1 - 8 * ( nyb - 1 ));   // rows the last tap block reads
            switch( nyb ) {
               case 1: m2_yphase< 1 >( ring, wy2, cp, t0, nlast, acc ); break;
               case 2: m2_yphase< 2 >( ring, wy2, cp, t0, nlast, acc ); break;
               case 3: m2_yphase< 3 >( ring, wy2, cp, t0, nlast, acc ); break;
               case 4: m2_yphase< 4 >( ring, wy2, cp, t0, nlast, acc ); break;
               case 5: m2_yphase< 5 >( ring, wy2, cp, t0, nlast, acc ); break;
               case 6: m2_yphase< 6 >( ring, wy2, cp, t0, nlast, acc ); break;
               case 7: m2_yphase< 7 >( ring, wy2, cp, t0, nlast, acc ); break;
               case 8: m2_yphase< 8 >( ring, wy2, cp, t0, nlast, acc ); break;
               default: m2_yphase< 9 >( ring, wy2, cp, t0, nlast, acc ); break;
            }
            int const xo = x0 + 2 * cp;
            if( xo < nx ) {
               bool const both = xo + 1 < nx;
               float* p = im.dst + static_cast< int64_t >( b ) * im.dsb + static_cast< int64_t >( ya + t0 ) * im.ds1 + xo;
#pragma unroll
               for( int t = 0; t < RT; ++t ) {
                  if( ya + t0 + t < yb ) {
                     if( both && im.vec_out ) {
                        *reinterpret_cast< float2* >( p ) = acc[ t ];
                     } else {
                        p[ 0 ] = acc[ t ].x;
                        if( both ) { p[ 1 ] = acc[ t ].y; }
                     }
                  }
                  p += im.ds1;
               }
            }
         }
      }
      if( *abort_flag ) {
         // Before the CTA ends: the copies it announced and did not consume land first (bounded
         // waits again; a copy that never comes is given up on like the first).
         asm volatile( "cp.async.wait_all;" ::: "memory" );
         if( tid == 0 ) {
            for( ; uses0 < issued0; ++uses0 ) { mbar_wait( &full[ 0 ], uses0 & 1u, wait_limit ); }
            for( ; uses1 < issued1; ++uses1 ) { mbar_wait( &full[ 1 ], uses1 & 1u, wait_limit ); }
         }
         __syncthreads();
         break;
      }
      __syncthreads();   // the item's ring, stages and tables are done with
   }
}

// Host side (k_march2d.cu).  Fills one image's TMA maps and geometry; false when the kernel
// cannot take the image (layout, boundary conditions, half-widths).
template< typename TIn >
bool march2d_image( M2Image& im, void const* src, int64_t nx, int64_t ny, int64_t ss1, int64_t nb, int64_t ssb,
                    float* dst, int64_t ds1, int64_t dsb, int32_t const bc[ 2 ], int32_t const h[ 2 ], int32_t const odd[ 2 ] );
// Persistent CTAs the kernel runs with (two per SM).
int march2d_slots();
// One launch over a device item list pulled through the device counter `counter` (zero before the
// launch).  `stall` (a test hook): the copies are announced but never issued and every wait gives
// up after a short limit, so the kernel reports DIPCU_ERR_TIMEOUT with nothing in flight.
cudaError_t launch_march2d_items( M2Image const* d_images, int nimages, M2Item const* d_items, int nitems, int32_t* counter,
                                  int stall, cudaStream_t stream );

} // namespace dipcu
