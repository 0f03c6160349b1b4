// K4: batched Gaussian FIR -- many 2D sfloat images of uneven sizes, each with its own sigmas,
// derivative orders and boundary conditions, filtered by a few grouped launches captured as one
// CUDA graph.
//
// A plan (dipcu_batch_plan_*) classifies every image once and uploads per-group tables of image
// descriptors and (image, tile) work items, plus a device table of (sigma, order) per image axis.
// Each run:
//   1. builds every image's kernel weights on the device (K0, gauss_weights_kernel), so that a
//      captured run can be replayed after the sigma table is updated in place,
//   2. forks onto four side streams (parallel branches of the graph):
//      * the grouped line passes (images with half-widths 13-32 or layouts the tile path does not
//        take): one launch per half-width bucket of the x axis into a plan-owned intermediate,
//        a join, then one launch per bucket of the y axis into the outputs;
//      * the grouped warp-per-tile launches (both half-widths up to 12): one per bucket, each warp
//        streaming its own boxes (TMA where the rows allow, else per-lane copies, gathered with
//        wrapped indices at periodic edges) through the y and x passes, tiles out by TMA stores
//        where the destination allows;
//   3. runs the persistent queue kernel for whatever is left (#SMs x occupancy CTAs pop (image,
//      tile) items with one atomicAdd each and filter them with the fused 2D routine of the
//      image's half-width bucket, 4, 8, 16 or 32), and joins the branches.
// Taps beyond an image's own half-width are zero in every bucketed kernel.  The persistent
// kernel's tile shape is chosen by an autotuner that times the candidates on the plan's batch.
//
// Items that name a non-existent image or tile (a corrupted list) are skipped and reported as
// DIPCU_ERR_INVALID_ARG in the device status word; every wait in these kernels is bounded.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"
#include "fused.cuh"
#include "fused2d_ws.cuh"
#include "march2d.cuh"

namespace dipcu {

cudaError_t launch_gauss_weights( double const* sigmas, uint32_t const* orders, int count, double truncation,
                                  float* weights, float* dweights, int32_t* lengths, int stride, cudaStream_t stream );
int32_t* device_status_ptr();

namespace {

constexpr int kBankStride = 40;   // weight-bank entry: up to 33 taps (half-width 32), padded
constexpr int kBuckets[ 4 ] = { 4, 8, 16, 32 };

struct BatchImage {
   float const* src;
   float* dst;
   int64_t n[ 2 ];
   int64_t ss[ 2 ], ds[ 2 ];     // x strides are 1
   int32_t bc[ 2 ], h[ 2 ], odd[ 2 ];
   int32_t wofs[ 2 ];            // weight-bank offsets (floats) of the x and y kernels
   int32_t tiles_x, tiles_y;
   int32_t bucket;
   int32_t pad;
};

struct BatchItem {
   int32_t image, tile;
};

struct BatchArgs {
   BatchImage const* images;
   BatchItem const* items;
   float const* wbank;
   int32_t* counter;
   int32_t* status;
   int32_t nimages, nitems;
};

template< int HB, int TX, int TY >
struct BatchLayout {
   static constexpr int WX = TX + 2 * HB;
   static constexpr int WY = TY + 2 * HB;
   static constexpr int PB = AlignUp4< WX >::value + 4;
   static constexpr int A_FLOATS = AlignUp4< WY * WX >::value;
   static constexpr int B_FLOATS = TY * PB;
   static constexpr size_t bytes() {
      return ( A_FLOATS + B_FLOATS ) * sizeof( float ) + WY * sizeof( int64_t ) + WX * sizeof( int32_t ) + WY + WX + 16;
   }
};

// y pass of one column over RY output rows, centred at row HB of the staged block (push form:
// every staged sample feeds the outputs it reaches; tap indices are compile-time constants).
template< int HB, int RY, bool ODD >
__device__ __forceinline__ void batch_ypass( float const* A, int pitch, int c, int r0, float const ( &w )[ HB + 1 ],
                                             float* B, int pb ) {
   float acc[ RY ];
#pragma unroll
   for( int i = 0; i < RY; ++i ) { acc[ i ] = 0.0f; }
#pragma unroll
   for( int j = 0; j < RY + 2 * HB; ++j ) {
      float v = A[ ( r0 + j ) * pitch + c ];
#pragma unroll
      for( int i = 0; i < RY; ++i ) {
         int const k = j - i - HB;                   // input row = output row + k
         if( k >= -HB && k <= HB ) {
            float const wk = w[ k < 0 ? -k : k ];
            acc[ i ] = fmaf(( ODD && k < 0 ) ? -wk : wk, v, acc[ i ] );
         }
      }
   }
#pragma unroll
   for( int i = 0; i < RY; ++i ) { B[ ( r0 + i ) * pb + c ] = acc[ i ]; }
}

template< int HB, int RX, bool ODD >
__device__ __forceinline__ void batch_xpass( float const* Brow, int x, float const ( &w )[ HB + 1 ], float* out ) {
   constexpr int NV = AlignUp4< RX + 2 * HB >::value;
   float acc[ RX ];
#pragma unroll
   for( int i = 0; i < RX; ++i ) { acc[ i ] = 0.0f; }
   float4 const* p = reinterpret_cast< float4 const* >( Brow + x );
#pragma unroll
   for( int q = 0; q < NV / 4; ++q ) {
      float4 f = p[ q ];
      float const vv[ 4 ] = { f.x, f.y, f.z, f.w };
#pragma unroll
      for( int e = 0; e < 4; ++e ) {
         int const j = 4 * q + e;
#pragma unroll
         for( int i = 0; i < RX; ++i ) {
            int const k = j - i - HB;
            if( k >= -HB && k <= HB ) {
               float const wk = w[ k < 0 ? -k : k ];
               acc[ i ] = fmaf(( ODD && k < 0 ) ? -wk : wk, vv[ e ], acc[ i ] );
            }
         }
      }
   }
#pragma unroll
   for( int i = 0; i < RX; ++i ) { out[ i ] = acc[ i ]; }
}

template< int HB, int TX, int TY >
__device__ void batch_tile( BatchImage const& im, int tile, float const* wbank, unsigned char* smem_raw ) {
   using L = BatchLayout< HB, TX, TY >;
   constexpr int NT = 256, RY = 8, RX = 4;
   float* A = reinterpret_cast< float* >( smem_raw );
   float* B = A + L::A_FLOATS;
   int64_t* rowoff = reinterpret_cast< int64_t* >( B + L::B_FLOATS );
   int32_t* colidx = reinterpret_cast< int32_t* >( rowoff + L::WY );
   uint8_t* rfl = reinterpret_cast< uint8_t* >( colidx + L::WX );
   uint8_t* cfl = rfl + L::WY;
   int const tid = static_cast< int >( threadIdx.x );
   int64_t const tx = tile % im.tiles_x, ty = tile / im.tiles_x;
   int64_t const x0 = tx * TX, y0 = ty * TY;
   float wx[ HB + 1 ], wy[ HB + 1 ];
#pragma unroll
   for( int k = 0; k <= HB; ++k ) {
      wx[ k ] = k <= im.h[ 0 ] ? __ldg( wbank + im.wofs[ 0 ] + k ) : 0.0f;
      wy[ k ] = k <= im.h[ 1 ] ? __ldg( wbank + im.wofs[ 1 ] + k ) : 0.0f;
   }
   // Boundary maps of the staged block (HB halo on every side; beyond the image's own
   // half-width the taps are zero).
   for( int r = tid; r < L::WY; r += NT ) {
      int64_t yi; uint8_t fl;
      map_coord( y0 - HB + r, im.n[ 1 ], im.bc[ 1 ], yi, fl );
      rowoff[ r ] = yi * im.ss[ 1 ];
      rfl[ r ] = fl;
   }
   for( int c = tid; c < L::WX; c += NT ) {
      int64_t xi; uint8_t fl;
      map_coord( x0 - HB + c, im.n[ 0 ], im.bc[ 0 ], xi, fl );
      colidx[ c ] = static_cast< int32_t >( xi );
      cfl[ c ] = fl;
   }
   __syncthreads();
   for( int e = tid; e < L::WY * L::WX; e += NT ) {
      int r = e / L::WX;
      int c = e - r * L::WX;
      uint8_t fl = static_cast< uint8_t >( rfl[ r ] | cfl[ c ] );
      float v = 0.0f;
      if( !( fl & 2 )) {
         v = im.src[ rowoff[ r ] + colidx[ c ] ];
         if(( rfl[ r ] ^ cfl[ c ] ) & 1 ) { v = -v; }
      }
      A[ e ] = v;
   }
   __syncthreads();
   for( int item = tid; item < L::WX * ( TY / RY ); item += NT ) {
      int c = item % L::WX;
      int rb = item / L::WX;
      if( im.odd[ 1 ] ) { batch_ypass< HB, RY, true >( A, L::WX, c, rb * RY, wy, B, L::PB ); }
      else { batch_ypass< HB, RY, false >( A, L::WX, c, rb * RY, wy, B, L::PB ); }
   }
   __syncthreads();
   constexpr int NSEG = TX / RX;
   for( int item = tid; item < TY * NSEG; item += NT ) {
      int s = item % NSEG;
      int r = item / NSEG;
      int64_t y = y0 + r;
      int64_t x = x0 + s * RX;
      if( y >= im.n[ 1 ] || x >= im.n[ 0 ] ) { continue; }
      float out[ RX ];
      if( im.odd[ 0 ] ) { batch_xpass< HB, RX, true >( B + r * L::PB, s * RX, wx, out ); }
      else { batch_xpass< HB, RX, false >( B + r * L::PB, s * RX, wx, out ); }
      store_row< RX >( im.dst + y * im.ds[ 1 ] + x, x, im.n[ 0 ], out );
   }
   __syncthreads();   // smem reused by the next item
}

template< int TX, int TY >
__global__ void __launch_bounds__( 256 ) batch_kernel( BatchArgs const __grid_constant__ a ) {
   extern __shared__ float4 smem4[];
   __shared__ int item_s;
   unsigned char* smem = reinterpret_cast< unsigned char* >( smem4 );
   for( ;; ) {
      if( threadIdx.x == 0 ) { item_s = atomicAdd( a.counter, 1 ); }
      __syncthreads();
      int const it = item_s;
      __syncthreads();
      if( it >= a.nitems ) { break; }
      BatchItem const item = a.items[ it ];
      if( item.image < 0 || item.image >= a.nimages ) {
         if( threadIdx.x == 0 ) { atomicExch( a.status, DIPCU_ERR_INVALID_ARG ); }
         continue;
      }
      BatchImage const im = a.images[ item.image ];
      if( item.tile < 0 || item.tile >= im.tiles_x * im.tiles_y || im.bucket < 0 || im.bucket > 3 ) {
         if( threadIdx.x == 0 ) { atomicExch( a.status, DIPCU_ERR_INVALID_ARG ); }
         continue;
      }
      switch( im.bucket ) {
         case 0: batch_tile< 4, TX, TY >( im, item.tile, a.wbank, smem ); break;
         case 1: batch_tile< 8, TX, TY >( im, item.tile, a.wbank, smem ); break;
         case 2: batch_tile< 16, TX, TY >( im, item.tile, a.wbank, smem ); break;
         default: batch_tile< 32, TX, TY >( im, item.tile, a.wbank, smem ); break;
      }
   }
}

// ---- grouped warp-per-tile path: images with half-widths up to 12 and x-y boundary conditions
// the 2D tile kernel takes (fused2d_ws.cuh) run through a variant of that kernel with per-image
// tables: a TMA map per image in device memory and a work list of (image, tile) items, dealt
// round-robin over the warps of a persistent grid.  Taps come from the plan's weight bank per
// tile (zero beyond each axis' half-width), so a sigma-table update replays correctly.  Images
// whose row stride is not a multiple of 16 bytes (TMA global strides are) get the same boxes
// from per-lane cp.async copies with zero fill (8 bytes per lane and row when the row stride and
// width are even, else 4); every stage fill commits one copy group (empty for TMA boxes), so
// waiting until SPW - 1 groups are pending finds the current stage's copies done.  Edge tiles of
// images with "periodic" edges fill their boxes the same way, with the indices wrapped.  Output tiles
// go out as one TMA store each where the destination layout allows, else as per-lane stores.

struct alignas( 128 ) G2Image {
   CUtensorMap tmap;        // 4D (x, y, 1, 1) tiled map of the source, box = tile + halo (if tma)
   CUtensorMap tout;        // 4D tiled map of the destination, box = tile (if tma_store)
   float const* src;        // the source, for images whose layout TMA cannot take
   int64_t ss1;             // source row stride (x stride 1)
   int32_t tma;             // 1: boxes by TMA; 0: by per-lane asynchronous copies
   int32_t pair8;           // per-lane copies of 8 bytes (column pairs wholly inside or outside)
   int32_t tma_store;       // 1: output tiles by TMA stores
   float* dst;
   int64_t ds1;             // destination row stride (x stride 1)
   int32_t n[ 2 ];
   int32_t bc[ 2 ];
   int32_t h[ 2 ];
   int32_t wofs[ 2 ];       // weight-bank offsets of the x and y kernels
   int32_t odd[ 2 ];
   int32_t tiles_x, tiles_y;
   int32_t vec_store;       // float2 stores are 8-byte aligned
   int32_t wrap[ 2 ];       // "periodic" / "asym periodic" along x, y: edge tiles gather their boxes
};

struct G2Args {
   G2Image const* images;
   BatchItem const* items;
   float const* wbank;
   int32_t* status;
   int32_t nimages;
   int32_t nitems;
};

constexpr int kG2Buckets[ 4 ] = { 4, 6, 9, 12 };

template< int B >
struct G2Geom {
   using G = W2Geom< float, B, 32 >;
   static constexpr int WT = 2 * ( B + 1 );                            // taps per warp: x then y, float2
   static constexpr int OFF_WT = ( G::BYTES + 15 ) / 16 * 16;
   static constexpr int BYTES = OFF_WT + G::NW * WT * 8;
   static_assert( WT <= 32, "one tap per lane" );
   static_assert( BYTES <= 113 * 1024, "two CTAs per SM" );
};

template< int B >
__global__ void __launch_bounds__( W2Geom< float, B, 32 >::NT, 2 ) batch_ws_kernel( G2Args const __grid_constant__ a ) {
   using G = W2Geom< float, B, 32 >;
   using GG = G2Geom< B >;
   constexpr int TX = G::TX, TY = G::TY, BW = G::BW, BH = G::BH, SPW = G::SPW, RB = G::RB, E = G::E;
   constexpr int NW = G::NW;
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
   float2* const wt = reinterpret_cast< float2* >( smem + GG::OFF_WT ) + warp * GG::WT;    // x taps, then y taps
   float2 const* const wtx = wt;
   float2 const* const wty = wt + ( B + 1 );

   if( tid == 0 ) { *abort = 0; }
   if( lane == 0 ) {
      for( int d = 0; d < SPW; ++d ) { mbar_init( &full[ d ], 1 ); }
      fence_mbar_init();
   }
   __syncthreads();

   int64_t const gw = static_cast< int64_t >( blockIdx.x ) * NW + warp;
   int64_t const nwarps = static_cast< int64_t >( gridDim.x ) * NW;
   // Item t's image and tile, or false for an item that names no image or tile (skipped and
   // reported; its stage phase is completed without a copy so the stage sequence stays aligned).
   auto lookup = [ & ]( int64_t t, G2Image const*& im, int& x0, int& y0 ) -> bool {
      BatchItem const it = a.items[ t ];
      if( it.image < 0 || it.image >= a.nimages ) { return false; }
      im = a.images + it.image;
      if( it.tile < 0 || it.tile >= im->tiles_x * im->tiles_y ) { return false; }
      x0 = ( it.tile % im->tiles_x ) * TX;
      y0 = ( it.tile / im->tiles_x ) * TY;
      return true;
   };
   // Warp-wide: fills stage `st` with item t's box (nothing for t past the end) and commits
   // one copy group.
   auto issue = [ & ]( int64_t t, int st ) {
      if( t < a.nitems ) {
         G2Image const* im;
         int x0, y0;
         bool const ok = lookup( t, im, x0, y0 );
         // A tile that reads samples past a periodic edge gathers its box with wrapped indices.
         bool const gather = ok && (( im->wrap[ 0 ] && ( x0 - B < 0 || x0 + TX + B > im->n[ 0 ] )) ||
                                    ( im->wrap[ 1 ] && ( y0 - B < 0 || y0 + TY + B > im->n[ 1 ] )));
         if( gather ) {
            if( lane == 0 ) { mbar_arrive( &full[ st ] ); }
            // Box rows of BW floats, two columns per lane.  Along a periodic axis every index
            // outside the image is wrapped (negated for "asym periodic": a plain load and store);
            // along the other axis it is zero-filled, as in the copies below.
            int const nx = im->n[ 0 ], ny = im->n[ 1 ];
            int const by = y0 - B, xa = x0 - G::LEAD + 2 * lane;
            int cx[ 2 ];
            bool cin[ 2 ], cneg[ 2 ];
#pragma unroll
            for( int h = 0; h < 2; ++h ) {
               int const x = xa + h;
               cx[ h ] = x;
               cin[ h ] = x >= 0 && x < nx;
               cneg[ h ] = false;
               if( !cin[ h ] && im->wrap[ 0 ] ) {
                  bool ng;
                  cx[ h ] = static_cast< int >( bc_map_index( x, nx, im->bc[ 0 ], &ng ));
                  cin[ h ] = true;
                  cneg[ h ] = ng;
               }
            }
            float* const dst = reinterpret_cast< float* >( stages + st * G::STAGE_STRIDE );
            for( int r = 0; r < BH; ++r ) {
               int const y = by + r;
               int ry = y;
               bool rin = y >= 0 && y < ny, rneg = false;
               if( !rin && im->wrap[ 1 ] ) {
                  bool ng;
                  ry = static_cast< int >( bc_map_index( y, ny, im->bc[ 1 ], &ng ));
                  rin = true;
                  rneg = ng;
               }
#pragma unroll
               for( int h = 0; h < 2; ++h ) {
                  bool const in = rin && cin[ h ];
                  float const* src = in ? im->src + static_cast< int64_t >( ry ) * im->ss1 + cx[ h ] : im->src;
                  float* const d = dst + r * BW + 2 * lane + h;
                  if( in && ( rneg != cneg[ h ] )) {
                     *d = -__ldg( src );
                  } else {
                     asm volatile( "cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"( smem_u32( d )), "l"( src ), "r"( in ? 4 : 0 ) : "memory" );
                  }
               }
            }
         } else if( ok && im->tma ) {
            if( lane == 0 ) {
               mbar_arrive_expect_tx( &full[ st ], G::STAGE_BYTES );
               tma_load_4d( stages + st * G::STAGE_STRIDE, &im->tmap, &full[ st ], x0 - G::LEAD, y0 - B, 0, 0 );
            }
         } else {
            if( lane == 0 ) { mbar_arrive( &full[ st ] ); }
            if( ok ) {
               // Box rows of BW floats, two columns per lane; outside the image: zero fill.
               int const nx = im->n[ 0 ], ny = im->n[ 1 ];
               int const by = y0 - B, xa = x0 - G::LEAD + 2 * lane;
               bool const in0 = xa >= 0 && xa < nx, in1 = xa + 1 >= 0 && xa + 1 < nx;
               float const* const src0 = im->src;
               int64_t const ss1 = im->ss1;
               int64_t off = static_cast< int64_t >( by ) * ss1 + xa;   // used only inside the image
               uint32_t d = smem_u32( stages + st * G::STAGE_STRIDE ) + 8u * static_cast< uint32_t >( lane );
               if( im->pair8 ) {
#pragma unroll 4
                  for( int r = 0; r < BH; ++r, off += ss1, d += BW * 4 ) {
                     bool const in = static_cast< unsigned >( by + r ) < static_cast< unsigned >( ny ) && in0;
                     asm volatile( "cp.async.ca.shared.global [%0], [%1], 8, %2;"
                                   :: "r"( d ), "l"( in ? src0 + off : src0 ), "r"( in ? 8 : 0 ) : "memory" );
                  }
               } else {
#pragma unroll 4
                  for( int r = 0; r < BH; ++r, off += ss1, d += BW * 4 ) {
                     bool const yin = static_cast< unsigned >( by + r ) < static_cast< unsigned >( ny );
                     bool const i0 = yin && in0, i1 = yin && in1;
                     asm volatile( "cp.async.ca.shared.global [%0], [%1], 4, %2;"
                                   :: "r"( d ), "l"( i0 ? src0 + off : src0 ), "r"( i0 ? 4 : 0 ) : "memory" );
                     asm volatile( "cp.async.ca.shared.global [%0], [%1], 4, %2;"
                                   :: "r"( d + 4u ), "l"( i1 ? src0 + off + 1 : src0 ), "r"( i1 ? 4 : 0 ) : "memory" );
                  }
               }
            }
         }
      }
      asm volatile( "cp.async.commit_group;" ::: "memory" );
   };
   for( int k = 0; k < SPW; ++k ) { issue( gw + k * nwarps, k ); }
   uint32_t kdone = 0;
   for( int64_t t = gw; t < a.nitems; t += nwarps, ++kdone ) {
      int const st = static_cast< int >( kdone % SPW );
      unsigned char* const sp = stages + st * G::STAGE_STRIDE;
      G2Image const* im = nullptr;
      int x0 = 0, y0 = 0;
      bool const valid = lookup( t, im, x0, y0 );
      if( !valid ) {
         w5_wait( &full[ st ], ( kdone / SPW ) & 1u, abort, a.status );
         asm volatile( "cp.async.wait_group %0;" :: "n"( SPW - 1 ) : "memory" );
         __syncwarp();
         if( lane == 0 ) { atomicExch( a.status, DIPCU_ERR_INVALID_ARG ); }
         issue( t + SPW * nwarps, st );
         __syncwarp();
         continue;
      }
      int const nx = im->n[ 0 ], ny = im->n[ 1 ];
      int const bcx = im->bc[ 0 ], bcy = im->bc[ 1 ];
      int const bx = x0 - G::LEAD, by = y0 - B;
      bool const yedge = by < 0 || y0 + TY + B > ny;
      bool const xedge = x0 - B < 0 || x0 + TX + B > nx;
      // Taps of this image (the previous tile's reads of `wt` are done).
      if( lane < GG::WT ) {
         int const ax = lane / ( B + 1 ), k = lane - ax * ( B + 1 );
         float const w = k <= im->h[ ax ] ? __ldg( a.wbank + im->wofs[ ax ] + k ) : 0.f;
         wt[ lane ] = make_float2( w, w );
      }
      float2 const sx = im->odd[ 0 ] ? make_float2( -1.f, -1.f ) : make_float2( 1.f, 1.f );
      float2 const sy = im->odd[ 1 ] ? make_float2( -1.f, -1.f ) : make_float2( 1.f, 1.f );
      // Boundary tables of an edge tile.
      if( yedge ) {
         for( int r = lane; r < BH; r += 32 ) {
            int const yy = by + r;
            int src = r;
            float sg = 1.f;
            if(( yy < 0 || yy >= ny ) && yy >= -B && yy < ny + B && bcy != BC_ADD_ZEROS ) {
               bool neg;
               int const si = static_cast< int >( bc_map_index( yy, ny, bcy, &neg )) - by;
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
            bool want = c < C_HI && !( xx >= 0 && xx < nx ) && xx >= -B && xx < nx + B && bcx != BC_ADD_ZEROS;
            if( want ) {
               bool neg;
               int const sc = static_cast< int >( bc_map_index( xx, nx, bcx, &neg )) - bx;
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
      asm volatile( "cp.async.wait_group %0;" :: "n"( SPW - 1 ) : "memory" );
      __syncwarp();
      // y pass: lane -> column pair, row blocks of RB outputs
      if( lane < G::NPAIR ) {
         int const pc = G::P0 + lane;
#pragma unroll
         for( int r0 = 0; r0 < TY; r0 += RB ) {
            float2 v[ RB + 2 * B ];
            if( !yedge ) {
#pragma unroll
               for( int r = 0; r < RB + 2 * B; ++r ) { v[ r ] = w5_pair< float, BW >( sp, r0 + r, pc ); }
            } else {
#pragma unroll
               for( int r = 0; r < RB + 2 * B; ++r ) {
                  v[ r ] = w5_pair< float, BW >( sp, rmap[ r0 + r ], pc );
                  v[ r ] = fmul2( make_float2( rsgn[ r0 + r ], rsgn[ r0 + r ] ), v[ r ] );
               }
            }
            float2 o[ RB ];
#pragma unroll
            for( int t2 = 0; t2 < RB; ++t2 ) {
               float2 acc = fmul2( wty[ 0 ], v[ t2 + B ] );
#pragma unroll
               for( int k = 1; k <= B; ++k ) {
                  float2 const ps = ffma2( sy, v[ t2 + B - k ], v[ t2 + B + k ] );
                  acc = ffma2( wty[ k ], ps, acc );
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
      // The stage is read: stream this warp's item SPW ahead into it.
      issue( t + SPW * nwarps, st );
      if( nfx > 0 ) {
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
      // x pass: lane -> (row pair, strip of SW columns), results staged in `ot` (after any
      // earlier TMA store of this warp has finished reading it)
      if( lane == 0 ) { asm volatile( "cp.async.bulk.wait_group.read 0;" ::: "memory" ); }
      __syncwarp();
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
            float2 acc = fmul2( wtx[ 0 ], vx[ C0 + c ] );
#pragma unroll
            for( int k = 1; k <= B; ++k ) {
               float2 const ps = ffma2( sx, vx[ C0 + c - k ], vx[ C0 + c + k ] );
               acc = ffma2( wtx[ k ], ps, acc );
            }
            out[ c ] = acc;
         }
#pragma unroll
         for( int c = 0; c < G::SW; c += 2 ) {
            *reinterpret_cast< float2* >( ot + ( 2 * rp ) * G::OTS + c0 + c ) = make_float2( out[ c ].x, out[ c + 1 ].x );
            *reinterpret_cast< float2* >( ot + ( 2 * rp + 1 ) * G::OTS + c0 + c ) = make_float2( out[ c ].y, out[ c + 1 ].y );
         }
      }
      if( im->tma_store ) {
         // One TMA store of the staged tile (clipped at the image edges by the tensor map).
         fence_proxy_async();
         __syncwarp();
         if( lane == 0 ) {
            asm volatile( "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
                          :: "l"( reinterpret_cast< uint64_t >( &im->tout )), "r"( x0 ), "r"( y0 ), "r"( 0 ), "r"( 0 ),
                             "r"( smem_u32( ot )) : "memory" );
            asm volatile( "cp.async.bulk.commit_group;" ::: "memory" );
         }
         __syncwarp();
         continue;
      }
      __syncwarp();
      // Per-lane stores of the staged tile: lane -> column pair, down the tile's rows (a warp
      // store covers TX / 2 consecutive pairs of one row).
      static_assert( TX / 2 <= 32, "one column pair per lane" );
      int const xo = x0 + 2 * lane;
      if( lane < TX / 2 && xo < nx ) {
         int const rows = ny - y0 < TY ? ny - y0 : TY;
         int64_t const ds1 = im->ds1;
         float* p = im->dst + static_cast< int64_t >( y0 ) * ds1 + xo;
         float const* q = ot + 2 * lane;
         if( xo + 1 < nx && im->vec_store ) {
#pragma unroll 8
            for( int r = 0; r < rows; ++r, p += ds1, q += G::OTS ) { *reinterpret_cast< float2* >( p ) = *reinterpret_cast< float2 const* >( q ); }
         } else {
            bool const two = xo + 1 < nx;
#pragma unroll 8
            for( int r = 0; r < rows; ++r, p += ds1, q += G::OTS ) {
               p[ 0 ] = q[ 0 ];
               if( two ) { p[ 1 ] = q[ 1 ]; }
            }
         }
      }
      __syncwarp();   // b2, tables, taps and staging reads done before the next tile
   }
   if( lane == 0 ) { asm volatile( "cp.async.bulk.wait_group 0;" ::: "memory" ); }
}

template< int B >
cudaError_t launch_batch_ws( G2Args const& a, int grid, cudaStream_t st ) {
   batch_ws_kernel< B ><<< grid, W2Geom< float, B, 32 >::NT, G2Geom< B >::BYTES, st >>>( a ); count_launch();
   return cudaGetLastError();
}

template< int B >
int batch_ws_grid() {
   static std::mutex mu;
   static std::map< int, int > cache;
   int dev = 0;
   cudaGetDevice( &dev );
   std::lock_guard< std::mutex > lock( mu );
   auto it = cache.find( dev );
   if( it != cache.end() ) { return it->second; }
   auto kern = batch_ws_kernel< B >;
   size_t const smem = G2Geom< B >::BYTES;
   if( cudaFuncSetAttribute( kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( smem )) != cudaSuccess ) {
      return -1;
   }
   int per_sm = 0, sms = 148;
   if( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, kern, W2Geom< float, B, 32 >::NT, smem ) != cudaSuccess || per_sm < 1 ) {
      return -1;
   }
   cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
   cache[ dev ] = std::min( per_sm, 2 ) * sms;
   return cache[ dev ];
}

int g2_tile_x( int b ) {
   switch( b ) {
      case 0: return W2Geom< float, 4, 32 >::TX;
      case 1: return W2Geom< float, 6, 32 >::TX;
      case 2: return W2Geom< float, 9, 32 >::TX;
      default: return W2Geom< float, 12, 32 >::TX;
   }
}

int g2_box_h( int b ) {
   switch( b ) {
      case 0: return W2Geom< float, 4, 32 >::BH;
      case 1: return W2Geom< float, 6, 32 >::BH;
      case 2: return W2Geom< float, 9, 32 >::BH;
      default: return W2Geom< float, 12, 32 >::BH;
   }
}

int g2_grid( int b ) {
   switch( b ) {
      case 0: return batch_ws_grid< 4 >();
      case 1: return batch_ws_grid< 6 >();
      case 2: return batch_ws_grid< 9 >();
      default: return batch_ws_grid< 12 >();
   }
}

cudaError_t g2_launch( int b, G2Args const& a, int grid, cudaStream_t st ) {
   switch( b ) {
      case 0: return launch_batch_ws< 4 >( a, grid, st );
      case 1: return launch_batch_ws< 6 >( a, grid, st );
      case 2: return launch_batch_ws< 9 >( a, grid, st );
      default: return launch_batch_ws< 12 >( a, grid, st );
   }
}

// ---- grouped line passes: every other image (half-widths 13 .. 32, layouts the tile path does not take) as two
// passes -- along x into a plan-owned intermediate, then along y into the output -- with the
// register-window line kernels of the fast float path (k_line.cu), one table of images and work
// lists per pass and per half-width bucket of that pass' axis (4, 8, 12, 16, 24, 32): one launch
// each, the y passes after every x pass.  Taps come from the weight bank per work item (zero
// beyond the axis' half-width).

struct BLImage {
   float const* src;
   float* dst;
   float* tmp;              // n0 x n1 intermediate (dense rows)
   int64_t ss1, ds1;        // source and destination row strides (x stride 1)
   int32_t n0, n1;
   int32_t h[ 2 ], odd[ 2 ], bc[ 2 ], wofs[ 2 ];
   int32_t nseg;            // x pass: segments of 512 outputs per row
   int32_t ncb;             // y pass: column blocks of 128 per row block
};

struct BLArgs {
   BLImage const* images;
   BatchItem const* items;
   float const* wbank;
   int32_t* status;
   int32_t nimages;
   int32_t nitems;
};

constexpr int kNBL = 6;      // half-width buckets of the line passes, per axis
constexpr int kBLBuckets[ kNBL ] = { 4, 8, 12, 16, 24, 32 };
constexpr int kBLT = 256;    // x pass: outputs per item
constexpr int kBLXT = 64;    // x pass: threads per CTA (4 outputs each)
constexpr int kBLR = 16;     // y pass: rows per item

// Sample j of a line (base, stride st, length n), extended with the boundary condition.
__device__ __forceinline__ float bl_load( float const* base, int64_t st, int64_t j, int64_t n, int32_t bc ) {
   if( j >= 0 && j < n ) { return __ldg( base + j * st ); }
   if( bc == BC_ADD_ZEROS ) { return 0.f; }
   bool neg;
   int64_t const i = bc_map_index( j, n, bc, &neg );
   float const v = __ldg( base + i * st );
   return neg ? -v : v;
}

// Stages sample j of a line into `dst` (shared memory): an asynchronous 4-byte copy, zero fill
// for "add zeros", a plain load and store for sources the boundary condition negates.
__device__ __forceinline__ void bl_stage( float* dst, float const* base, int64_t j, int64_t n, int32_t bc ) {
   float const* src = base;
   int32_t bytes = 4;
   if( j >= 0 && j < n ) {
      src += j;
   } else if( bc == BC_ADD_ZEROS ) {
      bytes = 0;
   } else {
      bool neg;
      src += bc_map_index( j, n, bc, &neg );
      if( neg ) {
         *dst = -__ldg( src );
         return;
      }
   }
   asm volatile( "cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"( smem_u32( dst )), "l"( src ), "r"( bytes ) : "memory" );
}

template< int HB >
__global__ void __launch_bounds__( kBLXT ) batch_line_x_kernel( BLArgs const __grid_constant__ a ) {
   constexpr int W = kBLT + 2 * HB, WP = ( W + 3 ) / 4 * 4;
   constexpr int RX = kBLT / kBLXT;
   __shared__ __align__( 16 ) float tile[ 2 ][ WP ];
   __shared__ float ws[ 2 ][ HB + 1 ];
   int const tid = static_cast< int >( threadIdx.x );
   // Item t's image, row and segment start, or null for an item that names no image or row.
   auto lookup = [ & ]( int64_t t, int& row, int64_t& a0 ) -> BLImage const* {
      BatchItem const it = a.items[ t ];
      BLImage const* im = ( it.image >= 0 && it.image < a.nimages ) ? a.images + it.image : nullptr;
      if( !im || it.tile < 0 || it.tile >= im->n1 * im->nseg ) { return nullptr; }
      row = it.tile / im->nseg;
      a0 = static_cast< int64_t >( it.tile - row * im->nseg ) * kBLT;
      return im;
   };
   // Double-buffered: the copies of the next item land while this one is filtered.
   auto issue = [ & ]( int64_t t, int buf ) {
      if( t < a.nitems ) {
         int row;
         int64_t a0;
         BLImage const* im = lookup( t, row, a0 );
         if( im ) {
            if( tid <= HB ) { ws[ buf ][ tid ] = tid <= im->h[ 0 ] ? __ldg( a.wbank + im->wofs[ 0 ] + tid ) : 0.f; }
            float const* srow = im->src + static_cast< int64_t >( row ) * im->ss1;
            // Segments inside the row whose first sample is 16- (8-) byte aligned go as 16- (8-)
            // byte copies (W and a0 - HB are multiples of 4).
            float const* const g = srow + ( a0 - HB );
            uintptr_t const ga = reinterpret_cast< uintptr_t >( g );
            if( a0 - HB >= 0 && a0 - HB + W <= im->n0 && ( ga & 7 ) == 0 ) {
               if(( ga & 15 ) == 0 ) {
                  for( int e = 4 * tid; e < W; e += 4 * kBLXT ) {
                     asm volatile( "cp.async.cg.shared.global [%0], [%1], 16;" :: "r"( smem_u32( &tile[ buf ][ e ] )), "l"( g + e ) : "memory" );
                  }
               } else {
                  for( int e = 2 * tid; e < W; e += 2 * kBLXT ) {
                     asm volatile( "cp.async.ca.shared.global [%0], [%1], 8;" :: "r"( smem_u32( &tile[ buf ][ e ] )), "l"( g + e ) : "memory" );
                  }
               }
            } else {
               for( int e = tid; e < W; e += kBLXT ) { bl_stage( &tile[ buf ][ e ], srow, a0 - HB + e, im->n0, im->bc[ 0 ] ); }
            }
         }
      }
      asm volatile( "cp.async.commit_group;" ::: "memory" );
   };
   issue( blockIdx.x, 0 );
   int k = 0;
   for( int64_t t = blockIdx.x; t < a.nitems; t += gridDim.x, ++k ) {
      int const buf = k & 1;
      issue( t + gridDim.x, buf ^ 1 );
      asm volatile( "cp.async.wait_group 1;" ::: "memory" );
      __syncthreads();
      int row;
      int64_t a0;
      BLImage const* im = lookup( t, row, a0 );
      if( !im ) {   // uniform over the CTA
         if( tid == 0 ) { atomicExch( a.status, DIPCU_ERR_INVALID_ARG ); }
      } else {
         int64_t const n = im->n0;
         float v[ RX + 2 * HB + 4 ];
         float4 const* w4 = reinterpret_cast< float4 const* >( tile[ buf ] + tid * RX );
#pragma unroll
         for( int q = 0; q < ( RX + 2 * HB + 3 ) / 4; ++q ) {
            float4 const f = w4[ q ];
            v[ 4 * q ] = f.x; v[ 4 * q + 1 ] = f.y; v[ 4 * q + 2 ] = f.z; v[ 4 * q + 3 ] = f.w;
         }
         float const sg = im->odd[ 0 ] ? -1.f : 1.f;
         float acc[ RX ];
#pragma unroll
         for( int r = 0; r < RX; ++r ) { acc[ r ] = ws[ buf ][ 0 ] * v[ HB + r ]; }   // the centre tap is 0 for odd kernels
#pragma unroll
         for( int kk = 1; kk <= HB; ++kk ) {
            float const w = ws[ buf ][ kk ];
#pragma unroll
            for( int r = 0; r < RX; ++r ) { acc[ r ] = fmaf( w, fmaf( sg, v[ HB + r - kk ], v[ HB + r + kk ] ), acc[ r ] ); }
         }
         float* const trow = im->tmp + static_cast< int64_t >( row ) * n;
#pragma unroll
         for( int r = 0; r < RX; ++r ) {
            int64_t const i = a0 + tid * RX + r;
            if( i < n ) { trow[ i ] = acc[ r ]; }
         }
      }
      __syncthreads();   // this buffer and its taps are refilled two items later
   }
   asm volatile( "cp.async.wait_group 0;" ::: "memory" );
}

template< int HB >
__global__ void __launch_bounds__( 128 ) batch_line_y_kernel( BLArgs const __grid_constant__ a ) {
   __shared__ float ws[ 2 ][ HB + 1 ];   // taps of the current and the next item
   int const tid = static_cast< int >( threadIdx.x );
   int k = 0;
   for( int64_t t = blockIdx.x; t < a.nitems; t += gridDim.x, ++k ) {
      float* const wk = ws[ k & 1 ];
      BatchItem const it = a.items[ t ];
      BLImage const* im = ( it.image >= 0 && it.image < a.nimages ) ? a.images + it.image : nullptr;
      int const nrb = im ? ( im->n1 + kBLR - 1 ) / kBLR : 0;
      if( !im || it.tile < 0 || it.tile >= im->ncb * nrb ) {   // uniform over the CTA
         if( tid == 0 ) { atomicExch( a.status, DIPCU_ERR_INVALID_ARG ); }
         __syncthreads();   // keeps one barrier per item, so the tap buffers alternate safely
         continue;
      }
      // This buffer was last read two items ago, before the previous item's barrier.
      if( tid <= HB ) { wk[ tid ] = tid <= im->h[ 1 ] ? __ldg( a.wbank + im->wofs[ 1 ] + tid ) : 0.f; }
      __syncthreads();
      int const rb = it.tile / im->ncb, cb = it.tile - rb * im->ncb;
      int64_t const c = static_cast< int64_t >( cb ) * 128 + tid;
      if( c >= im->n0 ) { continue; }
      int64_t const n = im->n1, n0 = im->n0, i0 = static_cast< int64_t >( rb ) * kBLR;
      int32_t const bc = im->bc[ 1 ];
      float const* col = im->tmp + c;
      float v[ kBLR + 2 * HB ];
      if( i0 - HB >= 0 && i0 + kBLR + HB <= n ) {
         float const* p = col + ( i0 - HB ) * n0;
#pragma unroll
         for( int j = 0; j < kBLR + 2 * HB; ++j ) { v[ j ] = __ldg( p + j * n0 ); }
      } else {
#pragma unroll
         for( int j = 0; j < kBLR + 2 * HB; ++j ) { v[ j ] = bl_load( col, n0, i0 - HB + j, n, bc ); }
      }
      float const sg = im->odd[ 1 ] ? -1.f : 1.f;
      float acc[ kBLR ];
#pragma unroll
      for( int r = 0; r < kBLR; ++r ) { acc[ r ] = wk[ 0 ] * v[ HB + r ]; }
#pragma unroll
      for( int kk = 1; kk <= HB; ++kk ) {
         float const w = wk[ kk ];
#pragma unroll
         for( int r = 0; r < kBLR; ++r ) { acc[ r ] = fmaf( w, fmaf( sg, v[ HB + r - kk ], v[ HB + r + kk ] ), acc[ r ] ); }
      }
      float* const dcol = im->dst + c;
#pragma unroll
      for( int r = 0; r < kBLR; ++r ) {
         int64_t const i = i0 + r;
         if( i < n ) { dcol[ i * im->ds1 ] = acc[ r ]; }
      }
   }
}

template< int HB >
void bl_launch_hb( bool ypass, BLArgs const& a, unsigned grid, cudaStream_t st ) {
   if( ypass ) { batch_line_y_kernel< HB ><<< grid, 128, 0, st >>>( a ); count_launch(); } else { batch_line_x_kernel< HB ><<< grid, kBLXT, 0, st >>>( a ); count_launch(); }
}

cudaError_t bl_launch( int b, bool ypass, BLArgs const& a, cudaStream_t st ) {
   int64_t const cap = ypass ? 148 * 8 : 148 * 16;
   int64_t g = a.nitems < cap ? a.nitems : cap;
   if( g < 1 ) { g = 1; }
   unsigned const grid = static_cast< unsigned >( g );
   switch( b ) {
      case 0: bl_launch_hb< 4 >( ypass, a, grid, st ); break;
      case 1: bl_launch_hb< 8 >( ypass, a, grid, st ); break;
      case 2: bl_launch_hb< 12 >( ypass, a, grid, st ); break;
      case 3: bl_launch_hb< 16 >( ypass, a, grid, st ); break;
      case 4: bl_launch_hb< 24 >( ypass, a, grid, st ); break;
      default: bl_launch_hb< 32 >( ypass, a, grid, st ); break;
   }
   return cudaGetLastError();
}

// Candidate tile shapes (the autotuner's search space).
struct TileShape { int tx, ty; };
constexpr TileShape kShapes[ 3 ] = { { 64, 32 }, { 64, 16 }, { 128, 32 } };

template< int TX, int TY >
size_t batch_smem() { return BatchLayout< 32, TX, TY >::bytes(); }

size_t shape_smem( int s ) {
   switch( s ) {
      case 0: return batch_smem< 64, 32 >();
      case 1: return batch_smem< 64, 16 >();
      default: return batch_smem< 128, 32 >();
   }
}

void const* shape_kernel( int s ) {
   switch( s ) {
      case 0: return reinterpret_cast< void const* >( &batch_kernel< 64, 32 > );
      case 1: return reinterpret_cast< void const* >( &batch_kernel< 64, 16 > );
      default: return reinterpret_cast< void const* >( &batch_kernel< 128, 32 > );
   }
}

cudaError_t launch_shape( int s, int grid, BatchArgs const& a, cudaStream_t st ) {
   size_t smem = shape_smem( s );
   switch( s ) {
      case 0: batch_kernel< 64, 32 ><<< grid, 256, smem, st >>>( a ); count_launch(); break;
      case 1: batch_kernel< 64, 16 ><<< grid, 256, smem, st >>>( a ); count_launch(); break;
      default: batch_kernel< 128, 32 ><<< grid, 256, smem, st >>>( a ); count_launch(); break;
   }
   return cudaGetLastError();
}

int shape_grid( int s ) {
   static std::mutex mu;
   static std::map< std::pair< int, int >, int > cache;
   int dev = 0;
   cudaGetDevice( &dev );
   std::lock_guard< std::mutex > lock( mu );
   auto key = std::make_pair( s, dev );
   auto it = cache.find( key );
   if( it != cache.end() ) { return it->second; }
   size_t smem = shape_smem( s );
   if( cudaFuncSetAttribute( shape_kernel( s ), cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( smem )) != cudaSuccess ) {
      return -1;
   }
   int per_sm = 0, sms = 148;
   if( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, shape_kernel( s ), 256, smem ) != cudaSuccess || per_sm < 1 ) {
      return -1;
   }
   cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
   cache[ key ] = per_sm * sms;
   return per_sm * sms;
}

// Autotune results: batch signature -> tile shape.
std::mutex g_tune_mu;
std::map< std::string, int > g_tune_cache;

} // namespace

} // namespace dipcu

using namespace dipcu;

struct dipcu_batch_plan {
   int device = 0;
   int count = 0;
   int shape = 0;
   int grid = 0;
   double truncation = 3.0;
   std::vector< BatchImage > images;       // host copy (tiles depend on the shape)
   std::vector< double > sig_host;
   std::vector< uint32_t > ord_host;
   BatchImage* d_images = nullptr;
   BatchItem* d_items = nullptr;
   double* d_sigmas = nullptr;
   uint32_t* d_orders = nullptr;
   float* d_bank = nullptr;
   int32_t* d_counter = nullptr;
   int nitems = 0;
   // Grouped warp-per-tile path, per half-width bucket (4, 6, 9, 12).
   std::vector< int > gbucket;             // per image: bucket index, or -1 (persistent tile kernel)
   G2Image* d_gimg[ 4 ] = {};
   BatchItem* d_gitems[ 4 ] = {};
   int g_nimg[ 4 ] = {}, g_nitems[ 4 ] = {}, g_grid[ 4 ] = {};
   // Grouped line passes: one image table, work items per pass and per half-width bucket of
   // that pass' axis (4, 8, 12, 16, 24, 32), and their intermediate.
   BLImage* d_limg = nullptr;
   BatchItem* d_lxitems[ kNBL ] = {};
   BatchItem* d_lyitems[ kNBL ] = {};
   int l_nimg = 0, l_nx[ kNBL ] = {}, l_ny[ kNBL ] = {};
   float* d_tmp = nullptr;
   // Fork / join: side stream s runs the x passes of the line buckets b = s (mod 4), then -- once
   // every stream's x passes are done (ev_x) -- their y passes, then warp-per-tile bucket s;
   // the streams run concurrently with each other and the persistent kernel (parallel branches
   // of the captured graph).
   cudaStream_t side[ 4 ] = {};
   cudaEvent_t ev_fork = nullptr, ev_join[ 4 ] = {}, ev_x[ 4 ] = {};
   cudaStream_t cap_stream = nullptr;
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   // Row-march path (march2d.cuh): every image it takes, in one persistent launch that pulls
   // (image, strip, row run) items from a device work queue, most expensive items first.  The
   // row-run length is chosen per class of y half-width (up to 8, 16, 24, 32) by the autotuner.
   std::vector< char > march;              // per image: taken by the row-march path
   std::vector< M2Image > mimg;
   M2Image* d_mimg = nullptr;
   M2Item* d_mitems = nullptr;
   int32_t* d_mcounter = nullptr;
   int m_nitems = 0;
   int m_runlen[ 4 ] = { 384, 384, 384, 384 };
   int m_stall = 0;                        // DIPCU_BATCH_INJECT_STALLED_COPY
};

namespace {

int plan_fail( int code, std::string const& msg ) { return record_error( code, msg.c_str() ); }

// Images the grouped warp-per-tile path takes: both half-widths up to 12, sizes above the bucket,
// x-y boundary conditions with every halo source inside the staged box ("mirror", "zero order",
// "add zeros", "asym mirror") or "periodic" / "asym periodic" (whose edge tiles gather their boxes
// with wrapped indices), 4-byte aligned rows (TMA boxes where the layout allows, per-lane copies
// otherwise).  Their tables and work
// items are uploaded once per plan; `inject` plants one impossible item when the persistent tile
// kernel gets no items of its own.
int plan_groups( dipcu_batch_plan* p, int inject ) {
   p->gbucket.assign( static_cast< size_t >( p->count ), -1 );
   for( int i = 0; i < p->count; ++i ) {
      if( p->march[ static_cast< size_t >( i ) ] ) { p->gbucket[ static_cast< size_t >( i ) ] = 100; }   // row-march path
   }
   bool const no_ws = getenv( "DIPCU_BATCH_NO_WS" ) != nullptr;
   std::vector< G2Image > gimg[ 4 ];
   std::vector< BatchItem > gitems[ 4 ];
   int rest = 0;
   for( int i = 0; i < p->count; ++i ) {
      if( p->march[ static_cast< size_t >( i ) ] ) { continue; }
      BatchImage const& im = p->images[ static_cast< size_t >( i ) ];
      int const hm = std::max( im.h[ 0 ], im.h[ 1 ] );
      int const b = hm <= 4 ? 0 : hm <= 6 ? 1 : hm <= 9 ? 2 : hm <= 12 ? 3 : -1;
      bool ok = !no_ws && b >= 0 && ( reinterpret_cast< uintptr_t >( im.src ) & 3 ) == 0 && im.ss[ 1 ] > 0 && im.ds[ 1 ] > 0 &&
                im.n[ 0 ] < ( 1 << 30 ) && im.n[ 1 ] < ( 1 << 30 );
      for( int d = 0; d < 2 && ok; ++d ) {
         int32_t const bc = im.bc[ d ];
         ok = ( bc == BC_SYMMETRIC_MIRROR || bc == BC_ZERO_ORDER_EXTRAPOLATE || bc == BC_ADD_ZEROS || bc == BC_ASYMMETRIC_MIRROR ||
                bc == BC_PERIODIC || bc == BC_ASYMMETRIC_PERIODIC ) && im.n[ d ] > kG2Buckets[ b ];
      }
      G2Image g{};
      if( !ok ) { ++rest; continue; }
      g.src = im.src;
      g.ss1 = im.ss[ 1 ];
      g.tma = 0;
      if(( reinterpret_cast< uintptr_t >( im.src ) & 15 ) == 0 && ( im.ss[ 1 ] * 4 ) % 16 == 0 && !getenv( "DIPCU_BATCH_NO_TMA" )) {
         cuuint64_t dims[ 4 ] = { static_cast< cuuint64_t >( im.n[ 0 ] ), static_cast< cuuint64_t >( im.n[ 1 ] ), 1, 1 };
         cuuint64_t plane = static_cast< cuuint64_t >( im.ss[ 1 ] * im.n[ 1 ] * 4 );
         plane = ( plane + 15 ) / 16 * 16;
         cuuint64_t strides[ 3 ] = { static_cast< cuuint64_t >( im.ss[ 1 ] * 4 ), plane, plane };
         cuuint32_t box[ 4 ] = { 64, static_cast< cuuint32_t >( g2_box_h( b )), 1, 1 };
         g.tma = encode_source_map( &g.tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, im.src, dims, strides, box ) == CUDA_SUCCESS ? 1 : 0;
      }
      g.pair8 = (( reinterpret_cast< uintptr_t >( im.src ) & 7 ) == 0 && im.ss[ 1 ] % 2 == 0 && im.n[ 0 ] % 2 == 0 ) ? 1 : 0;
      g.dst = im.dst;
      g.ds1 = im.ds[ 1 ];
      g.tma_store = 0;
      if(( reinterpret_cast< uintptr_t >( im.dst ) & 15 ) == 0 && ( im.ds[ 1 ] * 4 ) % 16 == 0 && !getenv( "DIPCU_NO_TMA_STORE" )) {
         cuuint64_t dims[ 4 ] = { static_cast< cuuint64_t >( im.n[ 0 ] ), static_cast< cuuint64_t >( im.n[ 1 ] ), 1, 1 };
         cuuint64_t plane = static_cast< cuuint64_t >( im.ds[ 1 ] * im.n[ 1 ] * 4 );
         plane = ( plane + 15 ) / 16 * 16;
         cuuint64_t strides[ 3 ] = { static_cast< cuuint64_t >( im.ds[ 1 ] * 4 ), plane, plane };
         cuuint32_t box[ 4 ] = { static_cast< cuuint32_t >( g2_tile_x( b )), 32, 1, 1 };
         g.tma_store = encode_source_map( &g.tout, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, im.dst, dims, strides, box ) == CUDA_SUCCESS ? 1 : 0;
      }
      for( int d = 0; d < 2; ++d ) {
         g.n[ d ] = static_cast< int32_t >( im.n[ d ] );
         g.bc[ d ] = im.bc[ d ];
         g.h[ d ] = im.h[ d ];
         g.wofs[ d ] = im.wofs[ d ];
         g.odd[ d ] = im.odd[ d ];
      }
      int const tx = g2_tile_x( b );
      g.tiles_x = static_cast< int32_t >(( im.n[ 0 ] + tx - 1 ) / tx );
      g.tiles_y = static_cast< int32_t >(( im.n[ 1 ] + 31 ) / 32 );
      g.vec_store = (( reinterpret_cast< uintptr_t >( im.dst ) & 7 ) == 0 && im.ds[ 1 ] % 2 == 0 ) ? 1 : 0;
      for( int d = 0; d < 2; ++d ) { g.wrap[ d ] = ( im.bc[ d ] == BC_PERIODIC || im.bc[ d ] == BC_ASYMMETRIC_PERIODIC ) ? 1 : 0; }
      int const gi = static_cast< int >( gimg[ b ].size());
      for( int t = 0; t < g.tiles_x * g.tiles_y; ++t ) { gitems[ b ].push_back( BatchItem{ gi, t } ); }
      gimg[ b ].push_back( g );
      p->gbucket[ static_cast< size_t >( i ) ] = b;
   }
   // The rest: grouped line passes (every batch image qualifies: index-mapping boundary
   // conditions or "add zeros", half-widths up to 32, unit x stride).
   std::vector< BLImage > limg;
   std::vector< BatchItem > lx[ kNBL ], ly[ kNBL ];
   std::vector< int64_t > toff;   // intermediate offset of each image
   int64_t ttot = 0;
   auto bucket = []( int h ) { int b = 0; while( b < kNBL - 1 && h > kBLBuckets[ b ] ) { ++b; } return b; };
   if( !getenv( "DIPCU_BATCH_NO_LINES" )) {
      for( int i = 0; i < p->count; ++i ) {
         if( p->gbucket[ static_cast< size_t >( i ) ] >= 0 ) { continue; }
         BatchImage const& im = p->images[ static_cast< size_t >( i ) ];
         int const hm = std::max( im.h[ 0 ], im.h[ 1 ] );
         if( hm > 32 || ( reinterpret_cast< uintptr_t >( im.src ) & 3 ) || im.n[ 0 ] >= ( 1 << 30 ) || im.n[ 1 ] >= ( 1 << 30 )) { continue; }
         int const lbx = bucket( im.h[ 0 ] ), lby = bucket( im.h[ 1 ] );
         BLImage l{};
         l.src = im.src;
         l.dst = im.dst;
         l.ss1 = im.ss[ 1 ];
         l.ds1 = im.ds[ 1 ];
         l.n0 = static_cast< int32_t >( im.n[ 0 ] );
         l.n1 = static_cast< int32_t >( im.n[ 1 ] );
         for( int d = 0; d < 2; ++d ) {
            l.h[ d ] = im.h[ d ];
            l.odd[ d ] = im.odd[ d ];
            l.bc[ d ] = im.bc[ d ];
            l.wofs[ d ] = im.wofs[ d ];
         }
         l.nseg = ( l.n0 + kBLT - 1 ) / kBLT;
         l.ncb = ( l.n0 + 127 ) / 128;
         int const nrb = ( l.n1 + kBLR - 1 ) / kBLR;
         int const li = static_cast< int >( limg.size());
         for( int t = 0; t < l.n1 * l.nseg; ++t ) { lx[ lbx ].push_back( BatchItem{ li, t } ); }
         for( int t = 0; t < l.ncb * nrb; ++t ) { ly[ lby ].push_back( BatchItem{ li, t } ); }
         toff.push_back( ttot );
         ttot += static_cast< int64_t >( l.n0 ) * l.n1;
         limg.push_back( l );
         p->gbucket[ static_cast< size_t >( i ) ] = 4 + lby;
         --rest;
      }
   }
   if( inject && rest == 0 ) {
      bool done = false;
      for( auto& v : gitems ) {
         if( v.empty()) { continue; }
         if( inject == 1 ) { v[ v.size() / 2 ].image = 1 << 20; } else { v[ v.size() / 2 ].tile = 1 << 30; }
         done = true;
         break;
      }
      for( int b = 0; b < kNBL && !done; ++b ) {
         if( ly[ b ].empty()) { continue; }
         if( inject == 1 ) { ly[ b ][ ly[ b ].size() / 2 ].image = 1 << 20; } else { ly[ b ][ ly[ b ].size() / 2 ].tile = 1 << 30; }
         done = true;
      }
   }
   if( ttot > 0 ) {
      if( cudaMalloc( &p->d_tmp, sizeof( float ) * static_cast< size_t >( ttot )) != cudaSuccess ) {
         return plan_fail( DIPCU_ERR_CUDA, "batch plan: line-pass intermediate" );
      }
      for( size_t k = 0; k < limg.size(); ++k ) { limg[ k ].tmp = p->d_tmp + toff[ k ]; }
   }
   p->l_nimg = static_cast< int >( limg.size());
   if( !limg.empty() && ( cudaMalloc( &p->d_limg, sizeof( BLImage ) * limg.size()) != cudaSuccess ||
                          cudaMemcpy( p->d_limg, limg.data(), sizeof( BLImage ) * limg.size(), cudaMemcpyHostToDevice ) != cudaSuccess )) {
      return plan_fail( DIPCU_ERR_CUDA, "batch plan: line-pass tables" );
   }
   for( int b = 0; b < kNBL; ++b ) {
      p->l_nx[ b ] = static_cast< int >( lx[ b ].size());
      p->l_ny[ b ] = static_cast< int >( ly[ b ].size());
      if(( !lx[ b ].empty() && ( cudaMalloc( &p->d_lxitems[ b ], sizeof( BatchItem ) * lx[ b ].size()) != cudaSuccess ||
                                 cudaMemcpy( p->d_lxitems[ b ], lx[ b ].data(), sizeof( BatchItem ) * lx[ b ].size(), cudaMemcpyHostToDevice ) != cudaSuccess )) ||
         ( !ly[ b ].empty() && ( cudaMalloc( &p->d_lyitems[ b ], sizeof( BatchItem ) * ly[ b ].size()) != cudaSuccess ||
                                 cudaMemcpy( p->d_lyitems[ b ], ly[ b ].data(), sizeof( BatchItem ) * ly[ b ].size(), cudaMemcpyHostToDevice ) != cudaSuccess ))) {
         return plan_fail( DIPCU_ERR_CUDA, "batch plan: line-pass tables" );
      }
   }
   for( int b = 0; b < 4; ++b ) {
      p->g_nimg[ b ] = static_cast< int >( gimg[ b ].size());
      p->g_nitems[ b ] = static_cast< int >( gitems[ b ].size());
      if( gitems[ b ].empty()) { continue; }
      p->g_grid[ b ] = g2_grid( b );
      if( p->g_grid[ b ] < 1 ||
          cudaMalloc( &p->d_gimg[ b ], sizeof( G2Image ) * gimg[ b ].size()) != cudaSuccess ||
          cudaMalloc( &p->d_gitems[ b ], sizeof( BatchItem ) * gitems[ b ].size()) != cudaSuccess ||
          cudaMemcpy( p->d_gimg[ b ], gimg[ b ].data(), sizeof( G2Image ) * gimg[ b ].size(), cudaMemcpyHostToDevice ) != cudaSuccess ||
          cudaMemcpy( p->d_gitems[ b ], gitems[ b ].data(), sizeof( BatchItem ) * gitems[ b ].size(), cudaMemcpyHostToDevice ) != cudaSuccess ) {
         return plan_fail( DIPCU_ERR_CUDA, "batch plan: grouped tables" );
      }
   }
   return DIPCU_OK;
}

// Images the row-march kernel takes (TMA-readable layout, its boundary conditions, half-widths up
// to 32); their tables are uploaded once per plan.
int plan_march( dipcu_batch_plan* p ) {
   p->march.assign( static_cast< size_t >( p->count ), 0 );
   p->mimg.clear();
   if( getenv( "DIPCU_BATCH_NO_MARCH" )) { return DIPCU_OK; }
   for( int i = 0; i < p->count; ++i ) {
      BatchImage const& im = p->images[ static_cast< size_t >( i ) ];
      M2Image m{};
      if( !march2d_image< float >( m, im.src, im.n[ 0 ], im.n[ 1 ], im.ss[ 1 ], 1, 0, im.dst, im.ds[ 1 ], 0, im.bc, im.h, im.odd )) {
         continue;
      }
      m.w[ 0 ] = p->d_bank + im.wofs[ 0 ];
      m.w[ 1 ] = p->d_bank + im.wofs[ 1 ];
      p->march[ static_cast< size_t >( i ) ] = 1;
      p->mimg.push_back( m );
   }
   if( p->mimg.empty()) { return DIPCU_OK; }
   if( cudaMalloc( &p->d_mimg, sizeof( M2Image ) * p->mimg.size()) != cudaSuccess ||
       cudaMalloc( &p->d_mcounter, sizeof( int32_t )) != cudaSuccess ||
       cudaMemcpy( p->d_mimg, p->mimg.data(), sizeof( M2Image ) * p->mimg.size(), cudaMemcpyHostToDevice ) != cudaSuccess ) {
      return plan_fail( DIPCU_ERR_CUDA, "batch plan: row-march tables" );
   }
   return DIPCU_OK;
}

int march_class( int hy ) { return hy <= 8 ? 0 : hy <= 16 ? 1 : hy <= 24 ? 2 : 3; }

// The row-march work items for the current row-run lengths: per image, strips of 128 columns times
// runs of rows (the runs of an image equal in length), sorted by estimated cost (x-phase rows times
// the x window plus output rows times the y tap blocks), most expensive first.  `inject` replaces
// the middle item by an impossible one.
int march_items( dipcu_batch_plan* p, int inject ) {
   struct Costed { double cost; M2Item it; };
   std::vector< Costed > items;
   for( size_t k = 0; k < p->mimg.size(); ++k ) {
      M2Image const& m = p->mimg[ k ];
      int const L0 = p->m_runlen[ march_class( m.h[ 1 ] ) ];
      int const runs = std::max( 1, ( m.ny + L0 - 1 ) / L0 );
      int const L = ( m.ny + runs - 1 ) / runs;
      int const strips = ( m.nx + kM2TX - 1 ) / kM2TX;
      for( int y = 0; y < m.ny; y += L ) {
         int const yb = std::min( m.ny, y + L );
         double const cost = static_cast< double >( yb - y + 2 * m.h[ 1 ] ) * ( 4 + 2 * m.lead ) +
                             static_cast< double >( yb - y ) * 8 * (( 2 * m.h[ 1 ] + 8 ) / 8 ) + 200.0;
         for( int t = 0; t < strips; ++t ) { items.push_back( Costed{ cost, M2Item{ static_cast< int32_t >( k ), t * kM2TX, y, yb } } ); }
      }
   }
   std::stable_sort( items.begin(), items.end(), []( Costed const& a, Costed const& b ) { return a.cost > b.cost; } );
   std::vector< M2Item > list( items.size());
   for( size_t k = 0; k < items.size(); ++k ) { list[ k ] = items[ k ].it; }
   if( inject == 1 && !list.empty()) { list[ list.size() / 2 ].img = 1 << 20; }
   if( inject == 2 && !list.empty()) { list[ list.size() / 2 ].x0 = 1 << 30; }
   cudaFree( p->d_mitems );
   p->d_mitems = nullptr;
   p->m_nitems = static_cast< int >( list.size());
   if( list.empty()) { return DIPCU_OK; }
   if( cudaMalloc( &p->d_mitems, sizeof( M2Item ) * list.size()) != cudaSuccess ||
       cudaMemcpy( p->d_mitems, list.data(), sizeof( M2Item ) * list.size(), cudaMemcpyHostToDevice ) != cudaSuccess ) {
      return plan_fail( DIPCU_ERR_CUDA, "batch plan: row-march items" );
   }
   return DIPCU_OK;
}

cudaError_t march_launch( dipcu_batch_plan* p, cudaStream_t st ) {
   if( p->m_nitems == 0 ) { return cudaSuccess; }
   cudaError_t e = cudaMemsetAsync( p->d_mcounter, 0, sizeof( int32_t ), st );
   if( e != cudaSuccess ) { return e; }
   return launch_march2d_items( p->d_mimg, static_cast< int >( p->mimg.size()), p->d_mitems, p->m_nitems, p->d_mcounter,
                                p->m_stall, st );
}

// Autotuner of the row-march path: per class of y half-width present in the batch, the row-run
// length (96 rows .. whole images) that times fastest on this batch -- a trade between the x phase
// of the 2 hy halo rows every run repeats and the granularity of the work queue -- one class at a
// time (coordinate descent), after the weights are built once.  Remembered per batch signature.
std::mutex g_mtune_mu;
std::map< std::string, std::vector< int >> g_mtune_cache;

int march_tune( dipcu_batch_plan* p, std::string const& sig ) {
   {
      std::lock_guard< std::mutex > lock( g_mtune_mu );
      auto it = g_mtune_cache.find( sig );
      if( it != g_mtune_cache.end() ) {
         for( int c = 0; c < 4; ++c ) { p->m_runlen[ c ] = it->second[ static_cast< size_t >( c ) ]; }
         return DIPCU_OK;
      }
   }
   bool present[ 4 ] = {};
   for( auto const& m : p->mimg ) { present[ march_class( m.h[ 1 ] ) ] = true; }
   if( launch_gauss_weights( p->d_sigmas, p->d_orders, 2 * p->count, p->truncation, p->d_bank, nullptr, nullptr, kBankStride,
                             nullptr ) != cudaSuccess ) {
      return plan_fail( DIPCU_ERR_CUDA, "batch autotune: weights" );
   }
   cudaEvent_t e0, e1;
   cudaEventCreate( &e0 );
   cudaEventCreate( &e1 );
   auto time_it = [ & ]() -> float {
      if( march_items( p, 0 ) != DIPCU_OK ) { return 1e30f; }
      march_launch( p, nullptr );                           // warm-up
      cudaEventRecord( e0, nullptr );
      for( int r = 0; r < 3; ++r ) { march_launch( p, nullptr ); }
      cudaEventRecord( e1, nullptr );
      if( cudaEventSynchronize( e1 ) != cudaSuccess ) { return 1e30f; }
      float ms = 0.0f;
      cudaEventElapsedTime( &ms, e0, e1 );
      return ms;
   };
   int const cand[] = { 96, 192, 384, 768, 1 << 20 };
   for( int c = 0; c < 4; ++c ) {
      if( !present[ c ] ) { continue; }
      int best = p->m_runlen[ c ];
      float best_ms = 1e30f;
      for( int L : cand ) {
         p->m_runlen[ c ] = L;
         float const ms = time_it();
         if( ms < best_ms ) { best_ms = ms; best = L; }
      }
      p->m_runlen[ c ] = best;
   }
   cudaEventDestroy( e0 );
   cudaEventDestroy( e1 );
   std::lock_guard< std::mutex > lock( g_mtune_mu );
   g_mtune_cache[ sig ] = std::vector< int >( p->m_runlen, p->m_runlen + 4 );
   return DIPCU_OK;
}

// Tile the images for shape `s` and upload the work items, most expensive first.
int plan_items( dipcu_batch_plan* p, int s, int inject ) {
   TileShape const ts = kShapes[ s ];
   std::vector< BatchItem > items;
   for( int i = 0; i < p->count; ++i ) {
      BatchImage& im = p->images[ static_cast< size_t >( i ) ];
      if( p->gbucket[ static_cast< size_t >( i ) ] >= 0 ) { continue; }   // grouped warp-per-tile path
      im.tiles_x = static_cast< int32_t >(( im.n[ 0 ] + ts.tx - 1 ) / ts.tx );
      im.tiles_y = static_cast< int32_t >(( im.n[ 1 ] + ts.ty - 1 ) / ts.ty );
      for( int t = 0; t < im.tiles_x * im.tiles_y; ++t ) { items.push_back( BatchItem{ i, t } ); }
   }
   std::stable_sort( items.begin(), items.end(), [ & ]( BatchItem const& a, BatchItem const& b ) {
      return p->images[ static_cast< size_t >( a.image ) ].bucket > p->images[ static_cast< size_t >( b.image ) ].bucket;
   } );
   if( inject == 1 && !items.empty() ) { items[ items.size() / 2 ].image = p->count + 7; }   // impossible item
   if( inject == 2 && !items.empty() ) { items[ items.size() / 2 ].tile = 1 << 30; }
   cudaFree( p->d_items );
   p->d_items = nullptr;
   p->nitems = static_cast< int >( items.size() );
   if( cudaMalloc( &p->d_items, sizeof( BatchItem ) * std::max< size_t >( 1, items.size() )) != cudaSuccess ) {
      return plan_fail( DIPCU_ERR_CUDA, "cudaMalloc (batch items)" );
   }
   if( cudaMemcpy( p->d_items, items.data(), sizeof( BatchItem ) * items.size(), cudaMemcpyHostToDevice ) != cudaSuccess ||
       cudaMemcpy( p->d_images, p->images.data(), sizeof( BatchImage ) * p->images.size(), cudaMemcpyHostToDevice ) != cudaSuccess ) {
      return plan_fail( DIPCU_ERR_CUDA, "cudaMemcpy (batch tables)" );
   }
   p->shape = s;
   p->grid = shape_grid( s );
   if( p->grid < 1 ) { return plan_fail( DIPCU_ERR_CUDA, "batch kernel set-up" ); }
   return DIPCU_OK;
}

int enqueue_run( dipcu_batch_plan* p, cudaStream_t st ) {
   if( cudaMemsetAsync( p->d_counter, 0, sizeof( int32_t ), st ) != cudaSuccess ) {
      return plan_fail( DIPCU_ERR_CUDA, "cudaMemsetAsync (queue)" );
   }
   cudaError_t e = launch_gauss_weights( p->d_sigmas, p->d_orders, 2 * p->count, p->truncation, p->d_bank, nullptr,
                                         nullptr, kBankStride, st );
   if( e != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, "gauss_weights_kernel" ); }
   e = march_launch( p, st );
   if( e != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, std::string( "march2d_kernel: " ) + cudaGetErrorString( e )); }
   if( cudaEventRecord( p->ev_fork, st ) != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, "batch fork" ); }
   if( p->nitems > 0 ) {
      BatchArgs a{};
      a.images = p->d_images;
      a.items = p->d_items;
      a.wbank = p->d_bank;
      a.counter = p->d_counter;
      a.status = device_status_ptr();
      a.nimages = p->count;
      a.nitems = p->nitems;
      e = launch_shape( p->shape, p->grid, a, st );
      if( e != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, std::string( "batch_kernel: " ) + cudaGetErrorString( e )); }
   }
   BLArgs l{};
   l.images = p->d_limg;
   l.wbank = p->d_bank;
   l.status = device_status_ptr();
   l.nimages = p->l_nimg;
   auto line_pass = [ & ]( int b, bool ypass, cudaStream_t sb ) -> cudaError_t {
      l.items = ypass ? p->d_lyitems[ b ] : p->d_lxitems[ b ];
      l.nitems = ypass ? p->l_ny[ b ] : p->l_nx[ b ];
      return l.nitems > 0 ? bl_launch( b, ypass, l, sb ) : cudaSuccess;
   };
   for( int s = 0; s < 4; ++s ) {
      cudaStream_t const sb = p->side[ s ];
      if( cudaStreamWaitEvent( sb, p->ev_fork, 0 ) != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, "batch fork" ); }
      for( int b = s; b < kNBL && e == cudaSuccess; b += 4 ) { e = line_pass( b, false, sb ); }
      if( e != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, std::string( "batch line x pass: " ) + cudaGetErrorString( e )); }
      if( cudaEventRecord( p->ev_x[ s ], sb ) != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, "batch line join" ); }
   }
   for( int s = 0; s < 4; ++s ) {
      cudaStream_t const sb = p->side[ s ];
      for( int t = 0; t < 4; ++t ) {   // the y passes read every image's intermediate
         if( t != s && cudaStreamWaitEvent( sb, p->ev_x[ t ], 0 ) != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, "batch line join" ); }
      }
      for( int b = s; b < kNBL && e == cudaSuccess; b += 4 ) { e = line_pass( b, true, sb ); }
      if( e != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, std::string( "batch line y pass: " ) + cudaGetErrorString( e )); }
      if( p->g_nitems[ s ] > 0 ) {
         G2Args g{};
         g.images = p->d_gimg[ s ];
         g.items = p->d_gitems[ s ];
         g.wbank = p->d_bank;
         g.status = device_status_ptr();
         g.nimages = p->g_nimg[ s ];
         g.nitems = p->g_nitems[ s ];
         e = g2_launch( s, g, std::min( p->g_grid[ s ], std::max( 1, p->g_nitems[ s ] / 4 )), sb );
         if( e != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, std::string( "batch_ws_kernel: " ) + cudaGetErrorString( e )); }
      }
      if( cudaEventRecord( p->ev_join[ s ], sb ) != cudaSuccess || cudaStreamWaitEvent( st, p->ev_join[ s ], 0 ) != cudaSuccess ) {
         return plan_fail( DIPCU_ERR_CUDA, "batch join" );
      }
   }
   return DIPCU_OK;
}

void destroy_graph( dipcu_batch_plan* p ) {
   if( p->exec ) { cudaGraphExecDestroy( p->exec ); p->exec = nullptr; }
   if( p->graph ) { cudaGraphDestroy( p->graph ); p->graph = nullptr; }
}

} // namespace

extern "C" {

int dipcu_batch_plan_create( dipcu_image_desc const* ins, dipcu_image_desc const* outs, int count,
                             double const* sigmas, uint32_t const* orders, int32_t const* bcs, double truncation,
                             int flags, dipcu_batch_plan** plan_out ) {
   if( !plan_out || count < 1 || !ins || !outs || !sigmas || !orders || !bcs ) {
      return plan_fail( DIPCU_ERR_INVALID_ARG, "dipcu_batch_plan_create: bad arguments" );
   }
   *plan_out = nullptr;
   auto* p = new dipcu_batch_plan();
   cudaGetDevice( &p->device );
   p->count = count;
   p->truncation = truncation;
   p->images.resize( static_cast< size_t >( count ));
   p->sig_host.resize( 2 * static_cast< size_t >( count ));
   p->ord_host.resize( 2 * static_cast< size_t >( count ));
   std::string sig;
   for( int i = 0; i < count; ++i ) {
      dipcu_image_desc const& in = ins[ i ];
      dipcu_image_desc const& out = outs[ i ];
      if( in.ndims != 2 || out.ndims != 2 || in.dtype != DT_SFLOAT || out.dtype != DT_SFLOAT || !in.data || !out.data ||
          in.sizes[ 0 ] != out.sizes[ 0 ] || in.sizes[ 1 ] != out.sizes[ 1 ] || in.strides[ 0 ] != 1 || out.strides[ 0 ] != 1 ) {
         delete p;
         return plan_fail( DIPCU_ERR_INVALID_ARG, "batch images must be 2D sfloat with unit x stride and matching sizes (image " +
                                                  std::to_string( i ) + ")" );
      }
      BatchImage& im = p->images[ static_cast< size_t >( i ) ];
      im.src = static_cast< float const* >( in.data );
      im.dst = static_cast< float* >( out.data );
      int hb = 0;
      for( int d = 0; d < 2; ++d ) {
         double s = sigmas[ 2 * i + d ];
         uint32_t o = orders[ 2 * i + d ];
         int32_t bc = bcs[ 2 * i + d ];
         if( o > 3 ) { delete p; return plan_fail( DIPCU_ERR_ORDER_GT_3, "Gaussian FIR filter not implemented for order > 3" ); }
         if( !bc_is_index_map( bc )) {
            delete p;
            return plan_fail( DIPCU_ERR_UNSUPPORTED_BC, "the batched filter supports the index-mapping boundary conditions and \"add zeros\"" );
         }
         im.n[ d ] = in.sizes[ d ];
         im.ss[ d ] = in.strides[ d ];
         im.ds[ d ] = out.strides[ d ];
         im.bc[ d ] = bc;
         bool process = s > 0.0 && in.sizes[ d ] > 1;
         int64_t h = process ? half_gaussian_length( s, o, truncation, false ) - 1 : 0;
         if( h > 32 ) { delete p; return plan_fail( DIPCU_ERR_KERNEL_TOO_LARGE, "the batched filter supports half-widths up to 32" ); }
         im.h[ d ] = static_cast< int32_t >( h );
         im.odd[ d ] = process ? static_cast< int32_t >( o & 1u ) : 0;
         im.wofs[ d ] = ( 2 * i + d ) * kBankStride;
         // Unfiltered axes get the unit kernel (sigma 0 -> a single tap of 1).
         p->sig_host[ 2 * static_cast< size_t >( i ) + d ] = process ? s : 0.0;
         p->ord_host[ 2 * static_cast< size_t >( i ) + d ] = process ? o : 0;
         hb = std::max( hb, static_cast< int >( h ));
      }
      im.bucket = hb <= 4 ? 0 : hb <= 8 ? 1 : hb <= 16 ? 2 : 3;
      sig += std::to_string( im.bucket ) + ":" + std::to_string( im.n[ 0 ] / 64 ) + "x" + std::to_string( im.n[ 1 ] / 64 ) + ";";
   }
   bool ok = cudaMalloc( &p->d_images, sizeof( BatchImage ) * static_cast< size_t >( count )) == cudaSuccess &&
             cudaMalloc( &p->d_sigmas, sizeof( double ) * 2 * static_cast< size_t >( count )) == cudaSuccess &&
             cudaMalloc( &p->d_orders, sizeof( uint32_t ) * 2 * static_cast< size_t >( count )) == cudaSuccess &&
             cudaMalloc( &p->d_bank, sizeof( float ) * kBankStride * 2 * static_cast< size_t >( count )) == cudaSuccess &&
             cudaMalloc( &p->d_counter, sizeof( int32_t )) == cudaSuccess;
   ok = ok && cudaMemcpy( p->d_sigmas, p->sig_host.data(), sizeof( double ) * p->sig_host.size(), cudaMemcpyHostToDevice ) == cudaSuccess &&
        cudaMemcpy( p->d_orders, p->ord_host.data(), sizeof( uint32_t ) * p->ord_host.size(), cudaMemcpyHostToDevice ) == cudaSuccess;
   if( !ok ) {
      dipcu_batch_plan_destroy( p );
      return plan_fail( DIPCU_ERR_CUDA, "batch plan allocation" );
   }
   int const inject = ( flags & DIPCU_BATCH_INJECT_INVALID_IMAGE ) ? 1 : ( flags & DIPCU_BATCH_INJECT_INVALID_TILE ) ? 2 : 0;
   if( !device_status_ptr() ) {   // resolved before any capture
      dipcu_batch_plan_destroy( p );
      return plan_fail( DIPCU_ERR_CUDA, "device status word" );
   }
   if( int st = plan_march( p )) { dipcu_batch_plan_destroy( p ); return st; }
   int const m_inject = p->mimg.empty() ? 0 : inject;       // planted on the row-march path when it has work
   if( int st = plan_groups( p, m_inject ? 0 : inject )) { dipcu_batch_plan_destroy( p ); return st; }
   bool sok = cudaEventCreateWithFlags( &p->ev_fork, cudaEventDisableTiming ) == cudaSuccess;
   for( int b = 0; b < 4 && sok; ++b ) {
      sok = cudaStreamCreateWithFlags( &p->side[ b ], cudaStreamNonBlocking ) == cudaSuccess &&
            cudaEventCreateWithFlags( &p->ev_join[ b ], cudaEventDisableTiming ) == cudaSuccess &&
            cudaEventCreateWithFlags( &p->ev_x[ b ], cudaEventDisableTiming ) == cudaSuccess;
   }
   if( !sok ) { dipcu_batch_plan_destroy( p ); return plan_fail( DIPCU_ERR_CUDA, "batch plan: streams" ); }
   // Tile shape: the autotuner times every candidate on this batch (the filter outputs are
   // overwritten by the final runs), remembering the winner per batch signature.
   int shape = 0;
   if( char const* env = getenv( "DIPCU_BATCH_SHAPE" )) { shape = std::max( 0, std::min( 2, atoi( env ))); }
   p->m_stall = ( flags & DIPCU_BATCH_INJECT_STALLED_COPY ) ? 1 : 0;
   if(( flags & DIPCU_BATCH_AUTOTUNE ) && !p->mimg.empty() && !p->m_stall ) {
      if( int st = march_tune( p, sig )) { dipcu_batch_plan_destroy( p ); return st; }
   }
   if( int st = march_items( p, m_inject )) { dipcu_batch_plan_destroy( p ); return st; }
   bool rest_persistent = false;     // images left for the persistent tile kernel
   for( int i = 0; i < p->count; ++i ) { rest_persistent = rest_persistent || p->gbucket[ static_cast< size_t >( i ) ] < 0; }
   if(( flags & DIPCU_BATCH_AUTOTUNE ) && rest_persistent ) {
      std::lock_guard< std::mutex > lock( g_tune_mu );
      auto it = g_tune_cache.find( sig );
      if( it != g_tune_cache.end() ) {
         shape = it->second;
      } else {
         float best = 1e30f;
         cudaEvent_t e0, e1;
         cudaEventCreate( &e0 );
         cudaEventCreate( &e1 );
         for( int s = 0; s < 3; ++s ) {
            if( plan_items( p, s, 0 ) != DIPCU_OK ) { continue; }
            enqueue_run( p, nullptr );                    // warm-up
            cudaEventRecord( e0, nullptr );
            for( int r = 0; r < 3; ++r ) { enqueue_run( p, nullptr ); }
            cudaEventRecord( e1, nullptr );
            cudaEventSynchronize( e1 );
            float ms = 0.0f;
            cudaEventElapsedTime( &ms, e0, e1 );
            if( ms < best ) { best = ms; shape = s; }
         }
         cudaEventDestroy( e0 );
         cudaEventDestroy( e1 );
         g_tune_cache[ sig ] = shape;
      }
   }
   if( int st = plan_items( p, shape, m_inject ? 0 : inject )) { dipcu_batch_plan_destroy( p ); return st; }
   if( flags & DIPCU_BATCH_GRAPH ) {
      if( cudaStreamCreateWithFlags( &p->cap_stream, cudaStreamNonBlocking ) != cudaSuccess ||
          cudaStreamBeginCapture( p->cap_stream, cudaStreamCaptureModeThreadLocal ) != cudaSuccess ) {
         dipcu_batch_plan_destroy( p );
         return plan_fail( DIPCU_ERR_CUDA, "batch graph capture" );
      }
      int st = enqueue_run( p, p->cap_stream );
      cudaError_t ce = cudaStreamEndCapture( p->cap_stream, &p->graph );
      if( st != DIPCU_OK || ce != cudaSuccess || cudaGraphInstantiate( &p->exec, p->graph, 0 ) != cudaSuccess ) {
         dipcu_batch_plan_destroy( p );
         return plan_fail( DIPCU_ERR_CUDA, "batch graph instantiation" );
      }
   }
   *plan_out = p;
   return DIPCU_OK;
}

int dipcu_batch_plan_run( dipcu_batch_plan* plan, void* stream ) {
   if( !plan ) { return plan_fail( DIPCU_ERR_INVALID_ARG, "null plan" ); }
   cudaStream_t st = static_cast< cudaStream_t >( stream );
   if( plan->exec ) {
      cudaError_t e = cudaGraphLaunch( plan->exec, st );
      if( e != cudaSuccess ) { return plan_fail( DIPCU_ERR_CUDA, std::string( "cudaGraphLaunch: " ) + cudaGetErrorString( e )); }
      return DIPCU_OK;
   }
   return enqueue_run( plan, st );
}

int dipcu_batch_plan_info( dipcu_batch_plan const* plan, int* nitems, int* tile_x, int* tile_y, int* grid ) {
   if( !plan ) { return plan_fail( DIPCU_ERR_INVALID_ARG, "null plan" ); }
   if( nitems ) {
      *nitems = plan->nitems + plan->m_nitems;
      for( int b = 0; b < 4; ++b ) { *nitems += plan->g_nitems[ b ]; }
      for( int b = 0; b < kNBL; ++b ) { *nitems += plan->l_nx[ b ] + plan->l_ny[ b ]; }
   }
   if( tile_x ) { *tile_x = kShapes[ plan->shape ].tx; }
   if( tile_y ) { *tile_y = kShapes[ plan->shape ].ty; }
   if( grid ) { *grid = plan->grid; }
   return DIPCU_OK;
}

int dipcu_batch_plan_launches( dipcu_batch_plan const* plan, int* kernels, int* grouped_items ) {
   if( !plan ) { return plan_fail( DIPCU_ERR_INVALID_ARG, "null plan" ); }
   int k = 1 + ( plan->nitems > 0 ? 1 : 0 ) + ( plan->m_nitems > 0 ? 1 : 0 ), g = plan->m_nitems;
   for( int b = 0; b < 4; ++b ) {
      k += plan->g_nitems[ b ] > 0 ? 1 : 0;
      g += plan->g_nitems[ b ];
   }
   for( int b = 0; b < kNBL; ++b ) {
      k += ( plan->l_nx[ b ] > 0 ? 1 : 0 ) + ( plan->l_ny[ b ] > 0 ? 1 : 0 );
      g += plan->l_nx[ b ] + plan->l_ny[ b ];
   }
   if( kernels ) { *kernels = k; }
   if( grouped_items ) { *grouped_items = g; }
   return DIPCU_OK;
}

double* dipcu_batch_plan_sigmas( dipcu_batch_plan* plan ) {
   return plan ? plan->d_sigmas : nullptr;
}

int dipcu_batch_plan_destroy( dipcu_batch_plan* plan ) {
   if( !plan ) { return DIPCU_OK; }
   destroy_graph( plan );
   if( plan->cap_stream ) { cudaStreamDestroy( plan->cap_stream ); }
   cudaFree( plan->d_images );
   cudaFree( plan->d_items );
   cudaFree( plan->d_sigmas );
   cudaFree( plan->d_orders );
   cudaFree( plan->d_bank );
   cudaFree( plan->d_counter );
   for( int b = 0; b < 4; ++b ) {
      cudaFree( plan->d_gimg[ b ] );
      cudaFree( plan->d_gitems[ b ] );
   }
   cudaFree( plan->d_limg );
   for( int b = 0; b < kNBL; ++b ) {
      cudaFree( plan->d_lxitems[ b ] );
      cudaFree( plan->d_lyitems[ b ] );
   }
   cudaFree( plan->d_tmp );
   cudaFree( plan->d_mimg );
   cudaFree( plan->d_mitems );
   cudaFree( plan->d_mcounter );
   for( int b = 0; b < 4; ++b ) {
      if( plan->side[ b ] ) { cudaStreamDestroy( plan->side[ b ] ); }
      if( plan->ev_join[ b ] ) { cudaEventDestroy( plan->ev_join[ b ] ); }
      if( plan->ev_x[ b ] ) { cudaEventDestroy( plan->ev_x[ b ] ); }
   }
   if( plan->ev_fork ) { cudaEventDestroy( plan->ev_fork ); }
   delete plan;
   return DIPCU_OK;
}

int dipcu_device_status( int* status, int clear ) {
   int32_t* p = device_status_ptr();
   if( !p || !status ) { return plan_fail( DIPCU_ERR_INVALID_ARG, "dipcu_device_status" ); }
   int32_t v = 0;
   if( cudaMemcpy( &v, p, sizeof( v ), cudaMemcpyDeviceToHost ) != cudaSuccess ) {
      return plan_fail( DIPCU_ERR_CUDA, "dipcu_device_status: cudaMemcpy" );
   }
   *status = v;
   if( clear ) {
      int32_t z = 0;
      if( cudaMemcpy( p, &z, sizeof( z ), cudaMemcpyHostToDevice ) != cudaSuccess ) {
         return plan_fail( DIPCU_ERR_CUDA, "dipcu_device_status: cudaMemcpy" );
      }
   }
   return DIPCU_OK;
}

} // extern "C"
