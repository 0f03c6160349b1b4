// K2: the line-pass kernel.  One launch applies the 1D Gaussian FIR along one image axis, for
// every line of the image, exactly like one pass of dip::Framework::Separable
// (src/library/framework_separable.cpp:243-430 in DIPlib) does on the CPU with one thread per
// group of lines.  Each CTA stages a tile of `lines x (outputs + 2h)` samples of the pass
// input into shared memory -- converting the sample type (detail::CopyBuffer) and extending
// the lines at the image border with the boundary condition (detail::ExpandBuffer) -- and then
// evaluates the symmetric/antisymmetric tap sum of SeparableConvolutionLineFilter::Filter
// (src/linear/convolution.cpp:214-241) for its outputs.
//
// This kernel covers every layout a dip::Image can have (any dimensionality and strides, any
// real sample type, every boundary condition, kernels with half-widths up to 2048), and it is
// the path for kernels too long for the fused tile kernels.  Tiles run along the processed
// axis when that axis has the smallest stride; otherwise 32 neighbouring lines along the
// smallest-stride axis share a CTA so that global accesses stay coalesced.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"
#include "tma.cuh"

namespace dipcu {

namespace {

template< typename T, int MAXH1 >
struct LineArgs {
   void const* src;
   void* dst;
   int32_t src_dt, dst_dt;
   int32_t ndims, axis, comp;   // comp: the axis the L lines of a tile run along, or -1
   int32_t L, T_out, W;         // lines per tile, outputs per tile, staged samples per line
   int32_t h, odd, bc, across;  // across: threads run along `comp` when staging
   int32_t general, lo, hi;     // general: taps[0 .. lo + hi] is a full filter over offsets -lo .. hi
   int64_t n, ncomp, nouter;    // line length, size along comp, number of tile rows
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t sst[ DIPCU_MAX_DIMS ], dstst[ DIPCU_MAX_DIMS ];
   T taps[ MAXH1 ];             // centre tap first
};

template< typename T, int MAXH1 >
__global__ void __launch_bounds__( 256 ) line_pass_kernel( LineArgs< T, MAXH1 > const __grid_constant__ a ) {
   extern __shared__ unsigned char smem_raw[];
   T* tile = reinterpret_cast< T* >( smem_raw );
   int const tid = static_cast< int >( threadIdx.x );
   int const nthreads = static_cast< int >( blockDim.x );
   int64_t const a0 = static_cast< int64_t >( blockIdx.x ) * a.T_out;

   for( int64_t u = blockIdx.y; u < a.nouter; u += gridDim.y ) {
      // Decode the tile row u into the coordinates of all axes but `axis` (and the L-block
      // index along `comp`).
      int64_t rem = u;
      int64_t cblock = 0;
      int64_t sbase = 0, dbase = 0;
      if( a.comp >= 0 ) {
         int64_t ncb = ( a.ncomp + a.L - 1 ) / a.L;
         cblock = rem % ncb;
         rem /= ncb;
      }
      for( int d = 0; d < a.ndims; ++d ) {
         if( d == a.axis || d == a.comp ) { continue; }
         int64_t c = rem % a.sizes[ d ];
         rem /= a.sizes[ d ];
         sbase += c * a.sst[ d ];
         dbase += c * a.dstst[ d ];
      }
      int64_t const sa = a.sst[ a.axis ];
      int64_t const sc = a.comp >= 0 ? a.sst[ a.comp ] : 0;

      // Stage: converted, boundary-extended input samples [a0-h, a0+T_out+h) of L lines.
      int const total = a.L * a.W;
      for( int e = tid; e < total; e += nthreads ) {
         int l, w;
         if( a.across ) { l = e % a.L; w = e / a.L; } else { l = e / a.W; w = e % a.W; }
         int64_t line = cblock * a.L + l;
         T v = T( 0 );
         if( line < a.ncomp ) {
            int64_t lbase = sbase + line * sc;
            int64_t j = a0 - a.h + w;
            if( j >= 0 && j < a.n ) {
               v = load_as< T >( a.src, a.src_dt, lbase + j * sa );
            } else if( j >= -static_cast< int64_t >( a.h ) && j < a.n + a.h ) {
               auto ld = [ & ]( int64_t i ) { return load_as< T >( a.src, a.src_dt, lbase + i * sa ); };
               v = bc_extend< T >( j, a.n, a.bc, a.h, ld );
            }
         }
         tile[ l * a.W + w ] = v;
      }
      __syncthreads();

      // Filter: out[i] = f0 x[i] + sum_k f_k ( x[i+k] +- x[i-k] ).
      int const outs = a.L * a.T_out;
      for( int e = tid; e < outs; e += nthreads ) {
         int l, t;
         if( a.across ) { l = e % a.L; t = e / a.L; } else { l = e / a.T_out; t = e % a.T_out; }
         int64_t line = cblock * a.L + l;
         int64_t i = a0 + t;
         if( line >= a.ncomp || i >= a.n ) { continue; }
         T const* c = tile + l * a.W + t + a.h;
         if( a.general ) {
            T sum = T( 0 );
            for( int j = 0; j <= a.lo + a.hi; ++j ) { sum = fma( a.taps[ j ], c[ j - a.lo ], sum ); }
            store_from< T >( a.dst, a.dst_dt, dbase + line * ( a.comp >= 0 ? a.dstst[ a.comp ] : 0 ) + i * a.dstst[ a.axis ], sum );
            continue;
         }
         T sum = a.taps[ 0 ] * c[ 0 ];
         if( a.odd ) {
            for( int k = 1; k <= a.h; ++k ) { sum = fma( a.taps[ k ], c[ k ] - c[ -k ], sum ); }
         } else {
            for( int k = 1; k <= a.h; ++k ) { sum = fma( a.taps[ k ], c[ k ] + c[ -k ], sum ); }
         }
         store_from< T >( a.dst, a.dst_dt, dbase + line * ( a.comp >= 0 ? a.dstst[ a.comp ] : 0 ) + i * a.dstst[ a.axis ], sum );
      }
      __syncthreads();
   }
}

// ---- fast float path ------------------------------------------------------------------------
// Float input and output, half-widths up to 32, the index-mapping boundary conditions and "add
// zeros", and a unit-stride axis in both images: the same pass with the taps unrolled over a
// compile-time bucket HB >= h (zero beyond h) and register windows.
//   * Along the unit-stride axis (line_x_kernel): a CTA stages one line segment of nt R_X outputs
//     plus the halo in shared memory (coalesced loads, boundary extension at the line ends); each
//     thread evaluates R_X consecutive outputs from a float4 window of R_X + 2 HB samples.
//   * Along any other axis (line_y_kernel): threads run along the unit-stride axis (coalesced),
//     each owns one column and evaluates R_Y consecutive outputs along the processed axis from a
//     register window of R_Y + 2 HB samples read straight from global memory (the window overlap
//     of neighbouring blocks is served by L1/L2).
//   * Along any other axis, vectorised (line_y4_kernel), where both images keep 16-byte alignment
//     across the unit-stride axis: each thread owns a group of 4 adjacent columns and marches its
//     z-chunk (the processed axis) in steps of RZ outputs: the step's RZ + 2 HB rows are read as
//     float4 (one 16-byte load per row; the overlap with the previous step hits L1) and scattered
//     into RZ float4 accumulators with the full (unfolded, sign-expanded) kernel taken from the
//     kernel parameters, h exact up to 12 (buckets above).

constexpr int kFastMaxH = 32;
constexpr int kRX = 4;    // outputs per thread, line_x_kernel
constexpr int kRY = 16;   // outputs per thread, line_y_kernel

struct LineFastArgs {
   float const* src;
   float* dst;
   int32_t ndims, axis, comp;   // comp: the unit-stride axis the threads of line_y_kernel run along
   int32_t h, odd, bc;
   int64_t n, ncomp, nouter;    // length along axis, size along comp, lines (x) / column groups (y)
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t sst[ DIPCU_MAX_DIMS ], dstst[ DIPCU_MAX_DIMS ];
   // The other axes of size > 1, fastest first, with axes that nest in both images (stride =
   // the previous axis' stride times its size) merged: a contiguous image has one.
   int32_t nod;
   int64_t osz[ DIPCU_MAX_DIMS ], osst[ DIPCU_MAX_DIMS ], odst[ DIPCU_MAX_DIMS ];
   float taps[ kFastMaxH + 1 ];  // centre first, zero beyond h
};

// Source sample at index j of a line (base offset `base`, stride `st`), extended past [0, n) with
// the boundary condition (index maps; zero for "add zeros").
__device__ __forceinline__ float fast_load( LineFastArgs const& a, int64_t base, int64_t st, int64_t j ) {
   if( j >= 0 && j < a.n ) { return __ldg( a.src + base + j * st ); }
   if( a.bc == BC_ADD_ZEROS ) { return 0.f; }
   bool neg;
   int64_t const i = bc_map_index( j, a.n, a.bc, &neg );
   float const v = __ldg( a.src + base + i * st );
   return neg ? -v : v;
}

// Offsets of the line / column group u over all axes but `axis` (and `comp`).
__device__ __forceinline__ void fast_decode( LineFastArgs const& a, int64_t u, int64_t& sb, int64_t& db ) {
   if( a.nod == 1 ) {   // u < osz[ 0 ]
      sb = u * a.osst[ 0 ];
      db = u * a.odst[ 0 ];
      return;
   }
   sb = 0;
   db = 0;
   for( int d = 0; d < a.nod; ++d ) {
      int64_t const c = u % a.osz[ d ];
      u /= a.osz[ d ];
      sb += c * a.osst[ d ];
      db += c * a.odst[ d ];
   }
}

// Four partial sums (taps k mod 4), so that consecutive FMAs of one output do not wait on each other.
template< int HB, bool ODD >
__device__ __forceinline__ float fast_tap_sum( LineFastArgs const& a, float const* v ) {   // v[0] is the centre
   float s[ 4 ] = { ODD ? 0.f : a.taps[ 0 ] * v[ 0 ], 0.f, 0.f, 0.f };
#pragma unroll
   for( int k = 1; k <= HB; ++k ) {
      float const p = ODD ? v[ k ] - v[ -k ] : v[ k ] + v[ -k ];
      s[ k & 3 ] = fmaf( a.taps[ k ], p, s[ k & 3 ] );
   }
   return ( s[ 0 ] + s[ 1 ] ) + ( s[ 2 ] + s[ 3 ] );
}

// Stages sample j of a line into `dst` (shared memory): an asynchronous 4-byte copy for samples
// inside the line and for boundary sources that keep their sign, zero fill for "add zeros", a
// plain load and store for sources the boundary condition negates.
__device__ __forceinline__ void fast_stage( LineFastArgs const& a, float* dst, int64_t base, int64_t st, int64_t j ) {
   float const* src = a.src + base;
   int32_t bytes = 4;
   if( j >= 0 && j < a.n ) {
      src += j * st;
   } else if( a.bc == BC_ADD_ZEROS ) {
      bytes = 0;
   } else {
      bool neg;
      int64_t const i = bc_map_index( j, a.n, a.bc, &neg );
      src += i * st;
      if( neg ) {
         *dst = -__ldg( src );
         return;
      }
   }
   asm volatile( "cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"( smem_u32( dst )), "l"( src ), "r"( bytes ) : "memory" );
}

template< int HB, bool ODD >
__global__ void __launch_bounds__( 128 ) line_x_kernel( LineFastArgs const __grid_constant__ a ) {
   constexpr int WP = ( 128 * kRX + 2 * HB + 3 ) / 4 * 4;   // tile for the widest CTA (128 threads)
   __shared__ __align__( 16 ) float tile[ 2 ][ WP ];
   int const tid = static_cast< int >( threadIdx.x ), nt = static_cast< int >( blockDim.x );
   int const T = nt * kRX, W = T + 2 * HB;
   int64_t const a0 = static_cast< int64_t >( blockIdx.x ) * T;
   int64_t const sa = a.sst[ a.axis ], da = a.dstst[ a.axis ];
   // Double-buffered: the copies of the next line segment land while this one is filtered.
   // Segments inside the line whose first sample is 16- (8-) byte aligned go as 16- (8-) byte
   // copies (W and a0 - HB are multiples of 4: T = 4 nt, HB a multiple of 4; sa is 1 here).
   auto issue = [ & ]( int64_t u, float* buf ) {
      if( u < a.nouter ) {
         int64_t sb, db;
         fast_decode( a, u, sb, db );
         float const* const g = a.src + sb + ( a0 - HB );
         uintptr_t const ga = reinterpret_cast< uintptr_t >( g );
         if( a0 - HB >= 0 && a0 - HB + W <= a.n && ( ga & 7 ) == 0 ) {
            if(( ga & 15 ) == 0 ) {
               for( int e = 4 * tid; e < W; e += 4 * nt ) {
                  asm volatile( "cp.async.cg.shared.global [%0], [%1], 16;" :: "r"( smem_u32( buf + e )), "l"( g + e ) : "memory" );
               }
            } else {
               for( int e = 2 * tid; e < W; e += 2 * nt ) {
                  asm volatile( "cp.async.ca.shared.global [%0], [%1], 8;" :: "r"( smem_u32( buf + e )), "l"( g + e ) : "memory" );
               }
            }
         } else {
            for( int e = tid; e < W; e += nt ) { fast_stage( a, buf + e, sb, sa, a0 - HB + e ); }
         }
      }
      asm volatile( "cp.async.commit_group;" ::: "memory" );
   };
   issue( blockIdx.y, tile[ 0 ] );
   int k = 0;
   for( int64_t u = blockIdx.y; u < a.nouter; u += gridDim.y, ++k ) {
      issue( u + gridDim.y, tile[ ( k + 1 ) & 1 ] );
      asm volatile( "cp.async.wait_group 1;" ::: "memory" );
      __syncthreads();
      int64_t sb, db;
      fast_decode( a, u, sb, db );
      float v[ kRX + 2 * HB + 4 ];
      float4 const* w4 = reinterpret_cast< float4 const* >( tile[ k & 1 ] + tid * kRX );
#pragma unroll
      for( int q = 0; q < ( kRX + 2 * HB + 3 ) / 4; ++q ) {
         float4 const f = w4[ q ];
         v[ 4 * q ] = f.x; v[ 4 * q + 1 ] = f.y; v[ 4 * q + 2 ] = f.z; v[ 4 * q + 3 ] = f.w;
      }
#pragma unroll
      for( int r = 0; r < kRX; ++r ) {
         int64_t const i = a0 + tid * kRX + r;
         if( i < a.n ) { a.dst[ db + i * da ] = fast_tap_sum< HB, ODD >( a, v + HB + r ); }
      }
      __syncthreads();   // this buffer is refilled two segments later
   }
   asm volatile( "cp.async.wait_group 0;" ::: "memory" );
}

template< int HB, bool ODD >
__global__ void __launch_bounds__( 128 ) line_y_kernel( LineFastArgs const __grid_constant__ a ) {
   int64_t const c = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x;
   if( c >= a.ncomp ) { return; }
   int64_t const sa = a.sst[ a.axis ], da = a.dstst[ a.axis ];
   int64_t const nblk = ( a.n + kRY - 1 ) / kRY;
   for( int64_t u = blockIdx.y; u < a.nouter * nblk; u += gridDim.y ) {
      int64_t const blk = u % nblk;
      int64_t sb, db;
      fast_decode( a, u / nblk, sb, db );
      sb += c * a.sst[ a.comp ];
      db += c * a.dstst[ a.comp ];
      int64_t const i0 = blk * kRY;
      float v[ kRY + 2 * HB ];
      if( i0 - HB >= 0 && i0 + kRY + HB <= a.n ) {
         float const* p = a.src + sb + ( i0 - HB ) * sa;
#pragma unroll
         for( int j = 0; j < kRY + 2 * HB; ++j ) { v[ j ] = __ldg( p + j * sa ); }
      } else {
#pragma unroll
         for( int j = 0; j < kRY + 2 * HB; ++j ) { v[ j ] = fast_load( a, sb, sa, i0 - HB + j ); }
      }
#pragma unroll
      for( int r = 0; r < kRY; ++r ) {
         int64_t const i = i0 + r;
         if( i < a.n ) { a.dst[ db + i * da ] = fast_tap_sum< HB, ODD >( a, v + HB + r ); }
      }
   }
}

struct LineY4Args {
   float const* src;
   float* dst;
   int64_t n;                  // length along the processed axis
   int64_t sa, da;             // strides along it (multiples of 4 samples)
   int64_t ncomp4;             // 4-column groups along the unit-stride axis
   int64_t ncols;              // ncomp4 x outer lines
   int64_t chunk;              // outputs per thread along the axis (a multiple of RZ)
   int32_t bc;
   int32_t nod;
   int64_t osz[ DIPCU_MAX_DIMS ], osst[ DIPCU_MAX_DIMS ], odst[ DIPCU_MAX_DIMS ];
   float w[ 2 * kFastMaxH + 1 ];   // tap j (-h..h) at w[kFastMaxH + j]: sign-expanded, zero beyond h
};

template< int HB, int RZ >
__global__ void __launch_bounds__( 128, HB <= 12 ? 3 : 2 ) line_y4_kernel( LineY4Args const __grid_constant__ a ) {
   int64_t const col = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x;
   if( col >= a.ncols ) { return; }
   int64_t const c4 = col % a.ncomp4;
   int64_t u = col / a.ncomp4, sb = 4 * c4, db = 4 * c4;
   for( int d = 0; d < a.nod; ++d ) {
      int64_t const c = u % a.osz[ d ];
      u /= a.osz[ d ];
      sb += c * a.osst[ d ];
      db += c * a.odst[ d ];
   }
   float const* const src = a.src + sb;
   float* const dst = a.dst + db;
   int64_t const zb = static_cast< int64_t >( blockIdx.y ) * a.chunk;
   int64_t const ze = zb + a.chunk < a.n ? zb + a.chunk : a.n;
   for( int64_t z0 = zb; z0 < ze; z0 += RZ ) {
      float4 acc[ RZ ];
#pragma unroll
      for( int r = 0; r < RZ; ++r ) { acc[ r ] = make_float4( 0.f, 0.f, 0.f, 0.f ); }
      bool const interior = z0 - HB >= 0 && z0 + RZ + HB <= a.n;
      // every row of the step in flight before the arithmetic (windows up to 48 rows; longer
      // kernels read each row as they go, their arithmetic covers the latency)
      constexpr int NW = RZ + 2 * HB <= 48 ? RZ + 2 * HB : 1;
      float4 win[ NW ];
      auto row = [ & ]( int i ) -> float4 {
         int64_t zi = z0 - HB + i;
         if( interior ) { return __ldg( reinterpret_cast< float4 const* >( src + zi * a.sa )); }
         bool neg = false;
         if( zi < 0 || zi >= a.n ) { zi = a.bc == BC_ADD_ZEROS ? -1 : bc_map_index( zi, a.n, a.bc, &neg ); }
         float4 const v = zi < 0 ? make_float4( 0.f, 0.f, 0.f, 0.f ) : __ldg( reinterpret_cast< float4 const* >( src + zi * a.sa ));
         return neg ? make_float4( -v.x, -v.y, -v.z, -v.w ) : v;
      };
      if( NW == 1 ) {
      } else if( interior ) {
         float const* p = src + ( z0 - HB ) * a.sa;
#pragma unroll
         for( int i = 0; i < NW; ++i ) { win[ i ] = __ldg( reinterpret_cast< float4 const* >( p + i * a.sa )); }
      } else {
#pragma unroll
         for( int i = 0; i < NW; ++i ) { win[ i ] = row( i ); }
      }
#pragma unroll
      for( int i = 0; i < RZ + 2 * HB; ++i ) {
         float4 const v = NW == 1 ? row( i ) : win[ i < NW ? i : 0 ];
#pragma unroll
         for( int r = 0; r < RZ; ++r ) {
            int const j = i - HB - r;
            if( j < -HB || j > HB ) { continue; }
            float const w = a.w[ kFastMaxH + j ];
            acc[ r ].x = fmaf( w, v.x, acc[ r ].x );
            acc[ r ].y = fmaf( w, v.y, acc[ r ].y );
            acc[ r ].z = fmaf( w, v.z, acc[ r ].z );
            acc[ r ].w = fmaf( w, v.w, acc[ r ].w );
         }
      }
#pragma unroll
      for( int r = 0; r < RZ; ++r ) {
         if( z0 + r < ze ) { *reinterpret_cast< float4* >( dst + ( z0 + r ) * a.da ) = acc[ r ]; }
      }
   }
}

int sm_count_line() {
   static std::atomic< int > n{ 0 };
   if( n.load() == 0 ) {
      int dev = 0, v = 0;
      cudaGetDevice( &dev );
      cudaDeviceGetAttribute( &v, cudaDevAttrMultiProcessorCount, dev );
      n.store( v > 0 ? v : 148 );
   }
   return n.load();
}

// Ring variant of line_y4_kernel for half-widths up to 10 and the boundary conditions that keep
// the sample's sign: each thread streams its own column group's rows into a private ring of
// kY4Ring shared-memory rows with 16-byte asynchronous copies (zero fill for "add zeros"), kY4Pd
// blocks of RZ4 rows ahead of the block it computes, so every row is read from memory once per
// chunk and the copies in flight need no registers.  A thread reads only its own ring slots, so
// cp.async.wait_group is the only synchronisation.
constexpr int kY4Ring = 32;         // ring rows per thread (16 bytes each)
constexpr int kY4Rz = 4;            // outputs per step
constexpr int kY4Pd = 2;            // blocks in flight beyond the step's window (deeper rings with
                                    // fewer threads per SM measured slower)
constexpr int kY4Threads = 128;     // 64 KB of ring per CTA, 3 CTAs per SM

template< int HB >
__global__ void __launch_bounds__( kY4Threads ) line_y4r_kernel( LineY4Args const __grid_constant__ a ) {
   constexpr int RZ = kY4Rz, NBW = ( 2 * HB + RZ + RZ - 1 ) / RZ;     // blocks a step reads
   static_assert(( NBW + kY4Pd ) * RZ <= kY4Ring, "ring holds the window and the blocks in flight" );
   extern __shared__ __align__( 16 ) float4 y4ring[];    // [kY4Ring][kY4Threads]
   int const tid = static_cast< int >( threadIdx.x );
   int64_t const col = static_cast< int64_t >( blockIdx.x ) * kY4Threads + tid;
   bool const live = col < a.ncols;
   int64_t sb = 0, db = 0;
   if( live ) {
      int64_t const c4 = col % a.ncomp4;
      int64_t u = col / a.ncomp4;
      sb = 4 * c4;
      db = 4 * c4;
      for( int d = 0; d < a.nod; ++d ) {
         int64_t const c = u % a.osz[ d ];
         u /= a.osz[ d ];
         sb += c * a.osst[ d ];
         db += c * a.odst[ d ];
      }
   }
   float const* const src = a.src + sb;
   float* const dst = a.dst + db;
   int64_t const zb = static_cast< int64_t >( blockIdx.y ) * a.chunk;
   int64_t const ze = zb + a.chunk < a.n ? zb + a.chunk : a.n;
   int64_t const nsteps = ( ze - zb + RZ - 1 ) / RZ;
   // block q: rows zb - HB + q RZ .. + RZ - 1, ring slots (q RZ + i) mod kY4Ring
   auto issue = [ & ]( int64_t q ) {
      if( live && q < nsteps + NBW - 1 ) {
#pragma unroll
         for( int i = 0; i < RZ; ++i ) {
            int64_t z = zb - HB + q * RZ + i;
            int bytes = 16;
            if( z < 0 || z >= a.n ) {
               if( a.bc == BC_ADD_ZEROS ) { bytes = 0; z = 0; }
               else { bool neg; z = bc_map_index( z, a.n, a.bc, &neg ); }
            }
            float4* const slot = &y4ring[ (( q * RZ + i ) & ( kY4Ring - 1 )) * kY4Threads + tid ];
            asm volatile( "cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"( smem_u32( slot )),
                          "l"( src + z * a.sa ), "r"( bytes ) : "memory" );
         }
      }
      asm volatile( "cp.async.commit_group;" ::: "memory" );
   };
#pragma unroll
   for( int q = 0; q < NBW + kY4Pd - 1; ++q ) { issue( q ); }
   for( int64_t s = 0; s < nsteps; ++s ) {
      issue( s + NBW + kY4Pd - 1 );
      asm volatile( "cp.async.wait_group %0;" :: "n"( kY4Pd ) : "memory" );
      if( !live ) { continue; }
      float4 acc[ RZ ];
#pragma unroll
      for( int r = 0; r < RZ; ++r ) { acc[ r ] = make_float4( 0.f, 0.f, 0.f, 0.f ); }
      int const base = static_cast< int >(( s * RZ ) & ( kY4Ring - 1 ));
#pragma unroll
      for( int i = 0; i < RZ + 2 * HB; ++i ) {
         float4 const v = y4ring[ (( base + i ) & ( kY4Ring - 1 )) * kY4Threads + tid ];
#pragma unroll
         for( int r = 0; r < RZ; ++r ) {
            int const j = i - HB - r;
            if( j < -HB || j > HB ) { continue; }
            float const w = a.w[ kFastMaxH + j ];
            acc[ r ].x = fmaf( w, v.x, acc[ r ].x );
            acc[ r ].y = fmaf( w, v.y, acc[ r ].y );
            acc[ r ].z = fmaf( w, v.z, acc[ r ].z );
            acc[ r ].w = fmaf( w, v.w, acc[ r ].w );
         }
      }
      int64_t const z0 = zb + s * RZ;
#pragma unroll
      for( int r = 0; r < RZ; ++r ) {
         if( z0 + r < ze ) { *reinterpret_cast< float4* >( dst + ( z0 + r ) * a.da ) = acc[ r ]; }
      }
   }
   asm volatile( "cp.async.wait_group 0;" ::: "memory" );
}

template< int HB >
cudaError_t launch_y4r( LineY4Args& a, cudaStream_t stream ) {
   // chunks along the axis for ~14 resident warps per SM over the column groups
   int64_t const want = static_cast< int64_t >( sm_count_line()) * 14 * 32;
   int64_t nch = ( want + a.ncols - 1 ) / a.ncols;
   int64_t const maxch = ( a.n + kY4Rz - 1 ) / kY4Rz;
   nch = nch < 1 ? 1 : ( nch > maxch ? maxch : nch );
   a.chunk = (( a.n + nch - 1 ) / nch + kY4Rz - 1 ) / kY4Rz * kY4Rz;
   nch = ( a.n + a.chunk - 1 ) / a.chunk;
   int64_t const gx = ( a.ncols + kY4Threads - 1 ) / kY4Threads;
   if( gx > 0x7fffffff || nch > 65535 ) { return cudaErrorNotSupported; }
   constexpr int smem = kY4Ring * kY4Threads * 16;
   {
      // the opt-in above the 48 KB default, once per device
      static std::atomic< uint64_t > done{ 0 };
      int dev = 0;
      cudaGetDevice( &dev );
      uint64_t const bit = 1ull << ( dev & 63 );
      if( !( done.load() & bit )) {
         if( cudaFuncSetAttribute( line_y4r_kernel< HB >, cudaFuncAttributeMaxDynamicSharedMemorySize, smem ) != cudaSuccess ) {
            cudaGetLastError();
            return cudaErrorNotSupported;
         }
         done.fetch_or( bit );
      }
   }
   line_y4r_kernel< HB ><<< dim3( static_cast< unsigned >( gx ), static_cast< unsigned >( nch )), kY4Threads, smem, stream >>>( a );
   count_launch();
   return cudaGetLastError();
}

template< int HB >
cudaError_t launch_y4_bucket( LineY4Args& a, cudaStream_t stream ) {
   if constexpr( HB <= 10 ) {
      if( a.bc == BC_SYMMETRIC_MIRROR || a.bc == BC_PERIODIC || a.bc == BC_ZERO_ORDER_EXTRAPOLATE || a.bc == BC_ADD_ZEROS ) {
         return launch_y4r< HB >( a, stream );
      }
   }
   constexpr int RZ = HB <= 12 ? 8 : 16;
   // enough threads for ~16 warps per SM over the chunks along the axis
   int64_t const want = 148 * 16 * 32;
   int64_t nch = ( want + a.ncols - 1 ) / a.ncols;
   int64_t const maxch = ( a.n + RZ - 1 ) / RZ;
   nch = nch < 1 ? 1 : ( nch > maxch ? maxch : nch );
   a.chunk = (( a.n + nch - 1 ) / nch + RZ - 1 ) / RZ * RZ;
   nch = ( a.n + a.chunk - 1 ) / a.chunk;
   int64_t const gx = ( a.ncols + 127 ) / 128;
   if( gx > 0x7fffffff || nch > 65535 ) { return cudaErrorNotSupported; }
   line_y4_kernel< HB, RZ ><<< dim3( static_cast< unsigned >( gx ), static_cast< unsigned >( nch )), 128, 0, stream >>>( a );
   count_launch();
   return cudaGetLastError();
}

// The vectorised outer-axis pass, or cudaErrorNotSupported when the layout does not keep every
// 4-column group 16-byte aligned in both images.
cudaError_t launch_line_y4( LineFastArgs const& f, cudaStream_t stream ) {
   if( f.comp < 0 || f.ncomp % 4 != 0 || ( reinterpret_cast< uintptr_t >( f.src ) & 15 ) ||
       ( reinterpret_cast< uintptr_t >( f.dst ) & 15 )) {
      return cudaErrorNotSupported;
   }
   LineY4Args a{};
   a.src = f.src;
   a.dst = f.dst;
   a.n = f.n;
   a.sa = f.sst[ f.axis ];
   a.da = f.dstst[ f.axis ];
   if( a.sa % 4 || a.da % 4 || a.sa <= 0 ) { return cudaErrorNotSupported; }
   a.ncomp4 = f.ncomp / 4;
   a.ncols = a.ncomp4 * f.nouter;
   a.bc = f.bc;
   a.nod = f.nod;
   for( int d = 0; d < f.nod; ++d ) {
      if( f.osst[ d ] % 4 || f.odst[ d ] % 4 ) { return cudaErrorNotSupported; }
      a.osz[ d ] = f.osz[ d ];
      a.osst[ d ] = f.osst[ d ];
      a.odst[ d ] = f.odst[ d ];
   }
   for( int j = -kFastMaxH; j <= kFastMaxH; ++j ) {
      int const k = j < 0 ? -j : j;
      float const t = k <= f.h ? f.taps[ k ] : 0.f;
      a.w[ kFastMaxH + j ] = ( f.odd && j < 0 ) ? -t : t;
   }
   switch( f.h ) {
      case 0: case 1: return launch_y4_bucket< 1 >( a, stream );
      case 2: return launch_y4_bucket< 2 >( a, stream );
      case 3: return launch_y4_bucket< 3 >( a, stream );
      case 4: return launch_y4_bucket< 4 >( a, stream );
      case 5: return launch_y4_bucket< 5 >( a, stream );
      case 6: return launch_y4_bucket< 6 >( a, stream );
      case 7: return launch_y4_bucket< 7 >( a, stream );
      case 8: return launch_y4_bucket< 8 >( a, stream );
      case 9: return launch_y4_bucket< 9 >( a, stream );
      case 10: return launch_y4_bucket< 10 >( a, stream );
      case 11: return launch_y4_bucket< 11 >( a, stream );
      case 12: return launch_y4_bucket< 12 >( a, stream );
      default:
         return f.h <= 16 ? launch_y4_bucket< 16 >( a, stream ) : f.h <= 24 ? launch_y4_bucket< 24 >( a, stream )
                                                                 : launch_y4_bucket< 32 >( a, stream );
   }
}

// CTA width (32, 64 or 128 threads) that leaves the fewest idle threads for `n` items of
// `per` outputs per thread; the widest on ties.
int fast_width( int64_t n, int per ) {
   int best = 128;
   int64_t waste = ( n + 128 * per - 1 ) / ( 128 * per ) * ( 128 * per ) - n;
   for( int w : { 64, 32 } ) {
      int64_t const wv = ( n + w * per - 1 ) / ( w * per ) * ( w * per ) - n;
      if( wv < waste ) { waste = wv; best = w; }
   }
   return best;
}

// Short lines along the unit-stride axis (n <= 32 RX): a warp per line, lane l the outputs
// l RX .. l RX + RX - 1 from a window of RX + 2 HB staged samples.  Each warp stages its next line
// (16-byte asynchronous copies, the boundary extension at the line ends sample by sample) three
// lines ahead of the one it filters, in its own buffers: no block barrier, many lines in flight.
constexpr int kXwWarps = 8;
constexpr int kXwBuf = 4;           // line buffers per warp: three lines in flight while one is filtered

template< int HB, int RX, bool ODD >
__global__ void __launch_bounds__( kXwWarps * 32 ) line_xw_kernel( LineFastArgs const __grid_constant__ a ) {
   constexpr int WB = ( 32 * RX + 2 * HB + 3 ) / 4 * 4;     // buffer floats per line
   __shared__ __align__( 16 ) float buf[ kXwWarps ][ kXwBuf ][ WB ];
   int const lane = static_cast< int >( threadIdx.x ) & 31, warp = static_cast< int >( threadIdx.x ) >> 5;
   int64_t const gw = static_cast< int64_t >( blockIdx.x ) * kXwWarps + warp;
   int64_t const nw = static_cast< int64_t >( gridDim.x ) * kXwWarps;
   int64_t const sa = a.sst[ a.axis ], da = a.dstst[ a.axis ];
   int const W = static_cast< int >( a.n ) + 2 * HB;
   static_assert( HB % 4 == 0 && RX % 4 == 0, "16-byte aligned staging and window reads" );
   // The boundary extension is the same for every line: its source samples once per CTA
   // (sample index, -1 for a zero, bit 30 for a negated sample).
   __shared__ int32_t smap[ WB ];
   for( int e = static_cast< int >( threadIdx.x ); e < W; e += kXwWarps * 32 ) {
      int64_t const i = e - HB;
      int32_t m = static_cast< int32_t >( i );
      if( i < 0 || i >= a.n ) {
         if( a.bc == BC_ADD_ZEROS ) { m = -1; }
         else {
            bool neg;
            m = static_cast< int32_t >( bc_map_index( i, a.n, a.bc, &neg ));
            if( neg ) { m |= 1 << 30; }
         }
      }
      smap[ e ] = m;
   }
   __syncthreads();
   auto issue = [ & ]( int64_t u, float* b ) {
      if( u < a.nouter ) {
         int64_t sb, db;
         fast_decode( a, u, sb, db );
         // the line's 4-sample groups by 16-byte copies where its first sample is so aligned; the
         // rest (boundary extension, tail) sample by sample
         int e0 = 0, e1 = 0;                                  // [e0, e1): samples staged by the 16-byte copies
         if( sa == 1 && ( reinterpret_cast< uintptr_t >( a.src + sb ) & 15 ) == 0 ) {
            e1 = static_cast< int >( a.n ) & ~3;
            for( int q = lane; 4 * q < e1; q += 32 ) {
               asm volatile( "cp.async.cg.shared.global [%0], [%1], 16;" :: "r"( smem_u32( b + HB + 4 * q )),
                             "l"( a.src + sb + 4 * q ) : "memory" );
            }
         }
         for( int e = lane; e < W; e += 32 ) {
            int const i = e - HB;
            if( i >= e0 && i < e1 ) { continue; }
            int32_t const m = smap[ e ];
            float const* const src = a.src + sb + static_cast< int64_t >( m & ~( 1 << 30 )) * sa;
            if( m < 0 ) { b[ e ] = 0.f; }
            else if( m & ( 1 << 30 )) { b[ e ] = -__ldg( src ); }
            else { asm volatile( "cp.async.ca.shared.global [%0], [%1], 4;" :: "r"( smem_u32( b + e )), "l"( src ) : "memory" ); }
         }
      }
      asm volatile( "cp.async.commit_group;" ::: "memory" );
   };
#pragma unroll
   for( int j = 0; j < kXwBuf - 1; ++j ) { issue( gw + j * nw, buf[ warp ][ j ] ); }
   int k = 0;
   for( int64_t u = gw; u < a.nouter; u += nw, ++k ) {
      issue( u + ( kXwBuf - 1 ) * nw, buf[ warp ][ ( k + kXwBuf - 1 ) % kXwBuf ] );
      asm volatile( "cp.async.wait_group %0;" :: "n"( kXwBuf - 1 ) : "memory" );
      __syncwarp();
      int64_t sb, db;
      fast_decode( a, u, sb, db );
      float4 const* const w4 = reinterpret_cast< float4 const* >( buf[ warp ][ k % kXwBuf ] + lane * RX );
      float v[ RX + 2 * HB ];
#pragma unroll
      for( int q = 0; q < ( RX + 2 * HB ) / 4; ++q ) {
         float4 const f = w4[ q ];
         v[ 4 * q ] = f.x; v[ 4 * q + 1 ] = f.y; v[ 4 * q + 2 ] = f.z; v[ 4 * q + 3 ] = f.w;
      }
#pragma unroll
      for( int r = 0; r < RX; ++r ) {
         int64_t const i = static_cast< int64_t >( lane ) * RX + r;
         if( i < a.n ) { a.dst[ db + i * da ] = fast_tap_sum< HB, ODD >( a, v + HB + r ); }
      }
      __syncwarp();   // this buffer is refilled kXwBuf lines later
   }
   asm volatile( "cp.async.wait_group 0;" ::: "memory" );
}

template< int HB, int RX >
cudaError_t launch_xw( LineFastArgs const& a, cudaStream_t stream ) {
   int64_t const want = static_cast< int64_t >( sm_count_line()) * 8;
   int64_t const blocks = ( a.nouter + kXwWarps - 1 ) / kXwWarps;
   int64_t const gx = blocks < want ? blocks : want;
   if( a.odd ) { line_xw_kernel< HB, RX, true ><<< static_cast< unsigned >( gx ), kXwWarps * 32, 0, stream >>>( a ); }
   else { line_xw_kernel< HB, RX, false ><<< static_cast< unsigned >( gx ), kXwWarps * 32, 0, stream >>>( a ); }
   count_launch();
   return cudaGetLastError();
}

template< int HB >
cudaError_t launch_fast_bucket( LineFastArgs const& a, bool along, cudaStream_t stream ) {
   if( along && a.n <= 256 && a.nouter >= 1024 ) {
      return a.n <= 128 ? launch_xw< HB, 4 >( a, stream ) : launch_xw< HB, 8 >( a, stream );
   }
   if( along ) {
      int const nt = fast_width( a.n, kRX );
      int64_t const gx = ( a.n + nt * kRX - 1 ) / ( nt * kRX );
      int64_t const gy = a.nouter < 65535 ? a.nouter : 65535;
      if( gx > 0x7fffffff ) { return cudaErrorInvalidValue; }
      dim3 const grid( static_cast< unsigned >( gx ), static_cast< unsigned >( gy ));
      if( a.odd ) { line_x_kernel< HB, true ><<< grid, nt, 0, stream >>>( a ); count_launch(); }
      else { line_x_kernel< HB, false ><<< grid, nt, 0, stream >>>( a ); count_launch(); }
   } else {
      int const nt = fast_width( a.ncomp, 1 );
      int64_t const gx = ( a.ncomp + nt - 1 ) / nt;
      int64_t const work = a.nouter * (( a.n + kRY - 1 ) / kRY );
      int64_t const gy = work < 65535 ? work : 65535;
      if( gx > 0x7fffffff ) { return cudaErrorInvalidValue; }
      dim3 const grid( static_cast< unsigned >( gx ), static_cast< unsigned >( gy ));
      if( a.odd ) { line_y_kernel< HB, true ><<< grid, nt, 0, stream >>>( a ); count_launch(); }
      else { line_y_kernel< HB, false ><<< grid, nt, 0, stream >>>( a ); count_launch(); }
   }
   return cudaGetLastError();
}

// cudaErrorNotSupported when the pass is not one the fast path takes.
cudaError_t launch_line_fast( LinePass const& p, cudaStream_t stream ) {
   if( p.compute_double || p.src_dt != DT_SFLOAT || p.dst_dt != DT_SFLOAT || p.h < 0 || p.h > kFastMaxH ||
       !bc_is_index_map( p.bc ) || getenv( "DIPCU_NO_FAST_LINE" )) {
      return cudaErrorNotSupported;
   }
   LineFastArgs a{};
   a.src = static_cast< float const* >( p.src );
   a.dst = static_cast< float* >( p.dst );
   a.ndims = p.ndims;
   a.axis = p.axis;
   a.h = static_cast< int32_t >( p.h );
   a.odd = p.odd;
   a.bc = p.bc;
   a.n = p.sizes[ p.axis ];
   for( int d = 0; d < p.ndims; ++d ) {
      a.sizes[ d ] = p.sizes[ d ];
      a.sst[ d ] = p.src_strides[ d ];
      a.dstst[ d ] = p.dst_strides[ d ];
   }
   for( int k = 0; k <= kFastMaxH; ++k ) { a.taps[ k ] = k <= p.h ? static_cast< float >( p.taps[ k ] ) : 0.f; }
   bool const along = p.src_strides[ p.axis ] == 1 && p.dst_strides[ p.axis ] == 1;
   a.comp = -1;
   if( !along ) {
      for( int d = 0; d < p.ndims; ++d ) {
         if( d != p.axis && p.sizes[ d ] > 1 && p.src_strides[ d ] == 1 && p.dst_strides[ d ] == 1 ) { a.comp = d; break; }
      }
      if( a.comp < 0 ) { return cudaErrorNotSupported; }
   }
   a.ncomp = along ? 1 : p.sizes[ a.comp ];
   int64_t nouter = 1;
   for( int d = 0; d < p.ndims; ++d ) {
      if( d != a.axis && d != a.comp ) { nouter *= p.sizes[ d ]; }
   }
   a.nouter = nouter;
   a.nod = 0;
   for( int d = 0; d < p.ndims; ++d ) {
      if( d == a.axis || d == a.comp || p.sizes[ d ] <= 1 ) { continue; }
      int const k = a.nod - 1;
      if( k >= 0 && p.src_strides[ d ] == a.osst[ k ] * a.osz[ k ] && p.dst_strides[ d ] == a.odst[ k ] * a.osz[ k ] ) {
         a.osz[ k ] *= p.sizes[ d ];
      } else {
         a.osz[ a.nod ] = p.sizes[ d ];
         a.osst[ a.nod ] = p.src_strides[ d ];
         a.odst[ a.nod ] = p.dst_strides[ d ];
         ++a.nod;
      }
   }
   if( a.nod == 0 ) {   // a single line (or column group)
      a.nod = 1;
      a.osz[ 0 ] = 1;
      a.osst[ 0 ] = 0;
      a.odst[ 0 ] = 0;
   }
   if( !along ) {
      cudaError_t const e = launch_line_y4( a, stream );
      if( e != cudaErrorNotSupported ) { return e; }
   }
   // Buckets at the half-widths of sigma 4 and 8 with order 0 (12, 24) as well as the powers of two.
   int const hb = p.h <= 4 ? 4 : p.h <= 8 ? 8 : p.h <= 12 ? 12 : p.h <= 16 ? 16 : p.h <= 24 ? 24 : 32;
   switch( hb ) {
      case 4: return launch_fast_bucket< 4 >( a, along, stream );
      case 8: return launch_fast_bucket< 8 >( a, along, stream );
      case 12: return launch_fast_bucket< 12 >( a, along, stream );
      case 16: return launch_fast_bucket< 16 >( a, along, stream );
      case 24: return launch_fast_bucket< 24 >( a, along, stream );
      default: return launch_fast_bucket< 32 >( a, along, stream );
   }
}

// Sample-type conversion of a whole image (dip::Image::Copy with clamp_cast), used when no
// axis is filtered (framework_separable.cpp:155-159).
template< typename T >
__global__ void __launch_bounds__( 256 ) convert_kernel( ConvertArgs const __grid_constant__ a ) {
   for( int64_t e = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; e < a.total;
        e += static_cast< int64_t >( gridDim.x ) * blockDim.x ) {
      int64_t rem = e, so = 0, doff = 0;
      for( int d = 0; d < a.ndims; ++d ) {
         int64_t c = rem % a.sizes[ d ];
         rem /= a.sizes[ d ];
         so += c * a.sst[ d ];
         doff += c * a.dstst[ d ];
      }
      store_from< T >( a.dst, a.dst_dt, doff, load_as< T >( a.src, a.src_dt, so ));
   }
}

template< typename T, int MAXH1 >
cudaError_t launch_line( LinePass const& p, cudaStream_t stream ) {
   LineArgs< T, MAXH1 > a{};
   a.src = p.src;
   a.dst = p.dst;
   a.src_dt = p.src_dt;
   a.dst_dt = p.dst_dt;
   a.ndims = p.ndims;
   a.axis = p.axis;
   a.h = static_cast< int32_t >( p.h );
   a.odd = p.odd;
   a.bc = p.bc;
   a.n = p.sizes[ p.axis ];
   for( int d = 0; d < p.ndims; ++d ) {
      a.sizes[ d ] = p.sizes[ d ];
      a.sst[ d ] = p.src_strides[ d ];
      a.dstst[ d ] = p.dst_strides[ d ];
   }
   if( p.mode == 1 ) {
      a.general = 1;
      a.lo = static_cast< int32_t >( p.lo );
      a.hi = static_cast< int32_t >( p.hi );
      for( int64_t k = 0; k <= p.lo + p.hi; ++k ) { a.taps[ k ] = static_cast< T >( p.full[ k ] ); }
   } else {
      for( int k = 0; k <= p.h; ++k ) { a.taps[ k ] = static_cast< T >( p.taps[ k ] ); }
   }

   // Companion axis: the smallest source stride among the other axes of size > 1.
   int comp = -1;
   for( int d = 0; d < p.ndims; ++d ) {
      if( d == p.axis || p.sizes[ d ] <= 1 ) { continue; }
      if( comp < 0 || llabs( p.src_strides[ d ] ) < llabs( p.src_strides[ comp ] )) { comp = d; }
   }
   bool along = ( comp < 0 ) || ( llabs( p.src_strides[ p.axis ] ) <= llabs( p.src_strides[ comp ] ));
   int64_t const smem_budget = 48 * 1024;
   int64_t const esz = sizeof( T );
   if( along ) {
      // Tiles run along the axis; one line per tile.
      a.comp = -1;
      a.L = 1;
      a.across = 0;
      int64_t t = 2048;
      if( t > a.n ) { t = a.n; }
      while( t > 32 && ( t + 2 * a.h ) * esz > smem_budget ) { t /= 2; }
      a.T_out = static_cast< int32_t >( t );
   } else {
      a.comp = comp;
      a.across = 1;
      a.L = 32;
      int64_t t = 128;
      while( a.L > 1 && ( 32 + 2 * a.h ) * esz * a.L > smem_budget ) { a.L /= 2; }
      while( t > 32 && ( t + 2 * a.h ) * esz * a.L > smem_budget ) { t /= 2; }
      if( t > a.n ) { t = a.n; }
      a.T_out = static_cast< int32_t >( t );
   }
   a.W = a.T_out + 2 * a.h;
   if( a.across && ( a.W % 2 ) == 0 ) { a.W += 1; } // odd pitch: conflict-free staging
   int64_t smem = static_cast< int64_t >( a.L ) * a.W * esz;
   if( smem > smem_budget ) { return cudaErrorInvalidValue; }
   a.ncomp = a.comp >= 0 ? p.sizes[ a.comp ] : 1;
   int64_t nouter = 1;
   for( int d = 0; d < p.ndims; ++d ) {
      if( d != a.axis && d != a.comp ) { nouter *= p.sizes[ d ]; }
   }
   if( a.comp >= 0 ) { nouter *= ( a.ncomp + a.L - 1 ) / a.L; }
   a.nouter = nouter;
   int64_t gx = ( a.n + a.T_out - 1 ) / a.T_out;
   int64_t gy = nouter < 65535 ? nouter : 65535;
   if( gx > 0x7fffffff ) { return cudaErrorInvalidValue; }
   line_pass_kernel< T, MAXH1 ><<< dim3( static_cast< unsigned >( gx ), static_cast< unsigned >( gy )), 256,
                                   static_cast< size_t >( smem ), stream >>>( a ); count_launch();
   return cudaGetLastError();
}

} // namespace

// The rectangular uniform filter along one axis: one thread per line keeps the running sum of
// RectangularUniformLineFilter::Filter (src/linear/uniform.cpp:41-62 in DIPlib) in the same
// operation order, over the line extended by `border` samples with the boundary condition.
struct UniformArgs {
   void const* src;
   void* dst;
   int32_t src_dt, dst_dt, ndims, axis, bc;
   int64_t n, nlines, usize, border;
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t sst[ DIPCU_MAX_DIMS ], dstst[ DIPCU_MAX_DIMS ];
};

// Additions and the product in the reference's order, never contracted into FMAs.
__device__ __forceinline__ float uadd( float a, float b ) { return __fadd_rn( a, b ); }
__device__ __forceinline__ double uadd( double a, double b ) { return __dadd_rn( a, b ); }
__device__ __forceinline__ float usub( float a, float b ) { return __fsub_rn( a, b ); }
__device__ __forceinline__ double usub( double a, double b ) { return __dsub_rn( a, b ); }
__device__ __forceinline__ float umul( float a, float b ) { return __fmul_rn( a, b ); }
__device__ __forceinline__ double umul( double a, double b ) { return __dmul_rn( a, b ); }

template< typename T >
__global__ void __launch_bounds__( 128 ) uniform_line_kernel( UniformArgs const __grid_constant__ a ) {
   int64_t const line = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x;
   if( line >= a.nlines ) { return; }
   int64_t rem = line, sbase = 0, dbase = 0;
   for( int d = 0; d < a.ndims; ++d ) {
      if( d == a.axis ) { continue; }
      int64_t const c = rem % a.sizes[ d ];
      rem /= a.sizes[ d ];
      sbase += c * a.sst[ d ];
      dbase += c * a.dstst[ d ];
   }
   int64_t const sa = a.sst[ a.axis ], da = a.dstst[ a.axis ], n = a.n;
   auto ld = [ & ]( int64_t i ) { return load_as< T >( a.src, a.src_dt, sbase + i * sa ); };
   auto x = [ & ]( int64_t j ) { return ( j >= 0 && j < n ) ? ld( j ) : bc_extend< T >( j, n, a.bc, a.border, ld ); };
   T const norm = T( 1 ) / static_cast< T >( a.usize );
   int64_t left = -( a.usize / 2 ), right = ( a.usize + 1 ) / 2;
   T sum = T( 0 );
   for( int64_t j = left; j < right; ++j ) { sum = uadd( sum, x( j )); }
   store_from< T >( a.dst, a.dst_dt, dbase, umul( sum, norm ));
   for( int64_t ii = 1; ii < n; ++ii ) {
      sum = usub( sum, x( left ));
      sum = uadd( sum, x( right ));
      ++left;
      ++right;
      store_from< T >( a.dst, a.dst_dt, dbase + ii * da, umul( sum, norm ));
   }
}

template< typename T >
cudaError_t launch_uniform( LinePass const& p, cudaStream_t stream ) {
   UniformArgs a{};
   a.src = p.src;
   a.dst = p.dst;
   a.src_dt = p.src_dt;
   a.dst_dt = p.dst_dt;
   a.ndims = p.ndims;
   a.axis = p.axis;
   a.bc = p.bc;
   a.n = p.sizes[ p.axis ];
   a.usize = p.usize;
   a.border = p.h;
   int64_t total = 1;
   for( int d = 0; d < p.ndims; ++d ) {
      a.sizes[ d ] = p.sizes[ d ];
      a.sst[ d ] = p.src_strides[ d ];
      a.dstst[ d ] = p.dst_strides[ d ];
      total *= p.sizes[ d ];
   }
   a.nlines = total / a.n;
   int64_t const blocks = ( a.nlines + 127 ) / 128;
   if( blocks > 0x7fffffff ) { return cudaErrorInvalidValue; }
   uniform_line_kernel< T ><<< static_cast< unsigned >( blocks ), 128, 0, stream >>>( a ); count_launch();
   return cudaGetLastError();
}

cudaError_t launch_line_pass( LinePass const& p, cudaStream_t stream ) {
   if( p.h < 0 || p.h > kLineMaxHalf ) { return cudaErrorInvalidValue; }
   if( p.mode == 2 ) {
      return p.compute_double ? launch_uniform< double >( p, stream ) : launch_uniform< float >( p, stream );
   }
   if( p.mode == 1 ) {
      if( p.lo < 0 || p.hi < 0 || p.lo + p.hi + 1 > kGeneralMaxTaps ) { return cudaErrorInvalidValue; }
      return p.compute_double ? launch_line< double, kGeneralMaxTaps >( p, stream ) : launch_line< float, kGeneralMaxTaps >( p, stream );
   }
   {
      cudaError_t const e = launch_line_fast( p, stream );
      if( e != cudaErrorNotSupported ) { return e; }
   }
   if( p.compute_double ) {
      return p.h < 64 ? launch_line< double, 64 >( p, stream ) : launch_line< double, kLineMaxHalf + 1 >( p, stream );
   }
   return p.h < 64 ? launch_line< float, 64 >( p, stream ) : launch_line< float, kLineMaxHalf + 1 >( p, stream );
}

cudaError_t launch_convert( ConvertArgs const& a, bool compute_double, cudaStream_t stream ) {
   int64_t blocks = ( a.total + 255 ) / 256;
   if( blocks > 148 * 16 ) { blocks = 148 * 16; }
   if( blocks < 1 ) { blocks = 1; }
   if( compute_double ) {
      convert_kernel< double ><<< static_cast< unsigned >( blocks ), 256, 0, stream >>>( a ); count_launch();
   } else {
      convert_kernel< float ><<< static_cast< unsigned >( blocks ), 256, 0, stream >>>( a ); count_launch();
   }
   return cudaGetLastError();
}

} // namespace dipcu
