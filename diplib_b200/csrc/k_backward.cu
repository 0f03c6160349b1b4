// K3 pieces of the adjoint (backward) of the Gaussian FIR.
//
// Along one axis the forward pass is y = C E x: E extends each line by h samples with the
// boundary condition (detail::ExpandBuffer, src/library/copy_buffer.cpp:751-813 in DIPlib) and C
// is the tap sum of SeparableConvolutionLineFilter::Filter (src/linear/convolution.cpp:214-241).
// Its adjoint is x_bar = E^T C^T y_bar.  C^T y_bar restricted to the line is a zero-padded
// correlation with the flipped kernel (run by the line kernel with "add zeros" and mirrored taps);
// the part of C^T y_bar that falls on the 2h halo positions is folded back onto the samples each
// halo sample was made from, with the coefficients of E (host-computed from the same boundary code
// the forward uses).  fold_kernel does that fold, one thread per line, or two (one per halo
// side) when the two sides fold onto disjoint samples; fold_fast_kernel, for float images whose
// halo positions each take one sample (the index mappings on lines longer than twice the
// half-width), keeps a side's samples and the taps in registers.
//
// dot_kernel reduces <a, b> over an image in double: the sigma gradient of axis a is
// <y_bar, G_a'(x)>, with G_a' the forward filter whose axis-a taps are d(taps)/d(sigma).
#include <cuda_runtime.h>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

namespace {

template< typename T >
struct FoldArgs {
   T const* g;               // gradient w.r.t. the pass output (input of this adjoint pass)
   T* xb;                    // gradient w.r.t. the pass input, holding the correlation part already
   int32_t ndims, axis;
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t gst[ DIPCU_MAX_DIMS ], xst[ DIPCU_MAX_DIMS ];
   int64_t n, nlines;
   int32_t h, odd, nentries;
   int32_t split;            // > 0: entries [0, split) and [split, nentries) by two threads per line
   T w[ kFoldMaxHalf + 1 ];  // forward taps, centre first
   FoldEntry e[ kFoldMaxEntries ];
};

template< typename T >
__global__ void fold_kernel( FoldArgs< T > const __grid_constant__ a ) {
   int64_t const tid = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x;
   bool const two = a.split > 0;
   int64_t const line = two ? tid >> 1 : tid;
   if( line >= a.nlines ) { return; }
   int const k0 = ( two && ( tid & 1 )) ? a.split : 0;
   int const k1 = ( two && !( tid & 1 )) ? a.split : a.nentries;
   int64_t rem = line, gb = 0, xbb = 0;
   for( int d = 0; d < a.ndims; ++d ) {
      if( d == a.axis ) { continue; }
      int64_t c = rem % a.sizes[ d ];
      rem /= a.sizes[ d ];
      gb += c * a.gst[ d ];
      xbb += c * a.xst[ d ];
   }
   int64_t const gs = a.gst[ a.axis ], xs = a.xst[ a.axis ];
   int32_t jprev = 0x7fffffff;
   double zj = 0.0;
   for( int k = k0; k < k1; ++k ) {
      FoldEntry const en = a.e[ k ];
      if( en.j != jprev ) {
         // Halo gradient: z_bar_j = sum_t g_t w_{j-t} over in-range t with |j - t| <= h.
         jprev = en.j;
         zj = 0.0;
         int64_t t0 = en.j - a.h, t1 = en.j + a.h;
         if( t0 < 0 ) { t0 = 0; }
         if( t1 > a.n - 1 ) { t1 = a.n - 1; }
#pragma unroll 4
         for( int64_t t = t0; t <= t1; ++t ) {
            int64_t kk = en.j - t;
            int64_t ak = kk < 0 ? -kk : kk;
            double wk = static_cast< double >( a.w[ ak ] );
            if( a.odd && kk < 0 ) { wk = -wk; }
            zj += wk * static_cast< double >( a.g[ gb + t * gs ] );
         }
      }
      T* p = a.xb + xbb + static_cast< int64_t >( en.i ) * xs;
      *p = static_cast< T >( static_cast< double >( *p ) + en.c * zj );
   }
}

template< typename T >
__global__ void __launch_bounds__( 256 ) dot_kernel( ConvertArgs const __grid_constant__ a, double* out ) {
   // <src, dst> over all samples; src/dst reuse ConvertArgs' layout fields (both of type T).
   double acc = 0.0;
   for( int64_t e = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; e < a.total;
        e += static_cast< int64_t >( gridDim.x ) * blockDim.x ) {
      int64_t rem = e, so = 0, doff = 0;
      for( int d = 0; d < a.ndims; ++d ) {
         int64_t c = rem % a.sizes[ d ];
         rem /= a.sizes[ d ];
         so += c * a.sst[ d ];
         doff += c * a.dstst[ d ];
      }
      acc += static_cast< double >( static_cast< T const* >( a.src )[ so ] ) *
             static_cast< double >( static_cast< T const* >( a.dst )[ doff ] );
   }
   for( int off = 16; off > 0; off >>= 1 ) { acc += __shfl_down_sync( 0xffffffffu, acc, off ); }
   __shared__ double part[ 8 ];
   int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if( lane == 0 ) { part[ warp ] = acc; }
   __syncthreads();
   if( warp == 0 ) {
      acc = lane < static_cast< int >( blockDim.x >> 5 ) ? part[ lane ] : 0.0;
      for( int off = 4; off > 0; off >>= 1 ) { acc += __shfl_down_sync( 0xffffffffu, acc, off ); }
      if( lane == 0 ) { atomicAdd( out, acc ); }
   }
}

// Fast fold for single-source boundary conditions (every halo position takes one sample, as the
// index mappings do when the line is longer than the half-width) and float images: a thread per
// line side keeps the side's HB samples of g and the taps in registers; halo position k (k = 1..h
// beyond the end) gathers z_k = sum_m w(k + m) g_m over the side's samples m = 0..h - k (m counted
// from the end inwards) and adds c_k z_k to its source sample.  The same sums and targets as
// fold_kernel, in float.
template< int HB >
struct FoldFastArgs {
   float const* g;
   float* xb;
   int32_t ndims, axis;
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t gst[ DIPCU_MAX_DIMS ], xst[ DIPCU_MAX_DIMS ];
   int64_t n, nlines;
   int32_t h, odd;
   float w[ HB + 1 ];                 // forward taps, centre first, zero beyond h
   int32_t src[ 2 ][ HB ];            // [side][k - 1]: source sample of halo position k
   float c[ 2 ][ HB ];                // its coefficient (0 beyond h)
};

template< int HB >
__global__ void __launch_bounds__( 128 ) fold_fast_kernel( FoldFastArgs< HB > const __grid_constant__ a ) {
   int64_t const tid = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x;
   int64_t const line = tid >> 1;
   int const side = static_cast< int >( tid & 1 );     // 0: before sample 0, 1: after sample n - 1
   if( line >= a.nlines ) { return; }
   int64_t rem = line, gb = 0, xbb = 0;
   for( int d = 0; d < a.ndims; ++d ) {
      if( d == a.axis ) { continue; }
      int64_t const c = rem % a.sizes[ d ];
      rem /= a.sizes[ d ];
      gb += c * a.gst[ d ];
      xbb += c * a.xst[ d ];
   }
   int64_t const gs = a.gst[ a.axis ], xs = a.xst[ a.axis ];
   // side samples, counted from the end inwards: m -> line sample m (side 0) or n - 1 - m (side 1)
   int64_t const g0 = side ? gb + ( a.n - 1 ) * gs : gb;
   int64_t const gstep = side ? -gs : gs;
   float gv[ HB ];
#pragma unroll
   for( int m = 0; m < HB; ++m ) { gv[ m ] = m < a.h ? a.g[ g0 + m * gstep ] : 0.f; }
   // the tap between halo position k (k beyond the end) and side sample m is at distance k + m; an
   // odd kernel's tap w(j - t) has the sign of j - t: negative before the line, positive after it
   float const sg = ( a.odd && !side ) ? -1.f : 1.f;
#pragma unroll
   for( int k = 1; k <= HB; ++k ) {
      if( k > a.h ) { break; }
      float z = 0.f;
#pragma unroll
      for( int m = 0; m + k <= HB; ++m ) { z = fmaf( a.w[ k + m ], gv[ m ], z ); }
      float* const p = a.xb + xbb + static_cast< int64_t >( a.src[ side ][ k - 1 ] ) * xs;
      *p += a.c[ side ][ k - 1 ] * sg * z;
   }
}

// The fast fold when its conditions hold; cudaErrorNotSupported otherwise.
template< int HB >
cudaError_t run_fold_fast( FoldPass const& p, cudaStream_t s ) {
   FoldFastArgs< HB > a{};
   int64_t const n = p.sizes[ p.axis ];
   if( p.compute_double || p.h < 1 || p.h > HB || n <= 2 * p.h || p.nentries != 2 * p.h ) { return cudaErrorNotSupported; }
   for( int k = 0; k < p.nentries; ++k ) {
      FoldEntry const& e = p.entries[ k ];
      int side, kk;
      if( e.j < 0 ) { side = 0; kk = -e.j; } else { side = 1; kk = static_cast< int >( e.j - ( n - 1 )); }
      if( kk < 1 || kk > p.h || a.c[ side ][ kk - 1 ] != 0.f || e.c == 0.0 ) { return cudaErrorNotSupported; }   // one source per position
      a.src[ side ][ kk - 1 ] = static_cast< int32_t >( e.i );
      a.c[ side ][ kk - 1 ] = static_cast< float >( e.c );
   }
   for( int side = 0; side < 2; ++side ) {
      for( int k = 0; k < p.h; ++k ) { if( a.c[ side ][ k ] == 0.f ) { return cudaErrorNotSupported; } }
   }
   // the two sides must fold onto disjoint samples (the two threads of a line write without atomics;
   // within a side one thread does every read-modify-write in order)
   for( int k = 0; k < p.h; ++k ) {
      for( int m = 0; m < p.h; ++m ) {
         if( a.src[ 0 ][ k ] == a.src[ 1 ][ m ] ) { return cudaErrorNotSupported; }
      }
   }
   a.g = static_cast< float const* >( p.g );
   a.xb = static_cast< float* >( p.xb );
   a.ndims = p.ndims;
   a.axis = p.axis;
   a.n = n;
   a.nlines = 1;
   for( int d = 0; d < p.ndims; ++d ) {
      a.sizes[ d ] = p.sizes[ d ];
      a.gst[ d ] = p.gst[ d ];
      a.xst[ d ] = p.xst[ d ];
      if( d != p.axis ) { a.nlines *= p.sizes[ d ]; }
   }
   a.h = static_cast< int32_t >( p.h );
   a.odd = p.odd;
   for( int k = 0; k <= HB; ++k ) { a.w[ k ] = k <= p.h ? static_cast< float >( p.taps[ k ] ) : 0.f; }
   int64_t const blocks = ( 2 * a.nlines + 127 ) / 128;
   if( blocks > 0x7fffffff ) { return cudaErrorInvalidValue; }
   fold_fast_kernel< HB ><<< static_cast< unsigned >( blocks ), 128, 0, s >>>( a ); count_launch();
   return cudaGetLastError();
}

template< typename T >
cudaError_t run_fold( FoldPass const& p, cudaStream_t s ) {
   FoldArgs< T > a{};
   a.g = static_cast< T const* >( p.g );
   a.xb = static_cast< T* >( p.xb );
   a.ndims = p.ndims;
   a.axis = p.axis;
   a.n = p.sizes[ p.axis ];
   a.nlines = 1;
   for( int d = 0; d < p.ndims; ++d ) {
      a.sizes[ d ] = p.sizes[ d ];
      a.gst[ d ] = p.gst[ d ];
      a.xst[ d ] = p.xst[ d ];
      if( d != p.axis ) { a.nlines *= p.sizes[ d ]; }
   }
   a.h = static_cast< int32_t >( p.h );
   a.odd = p.odd;
   a.nentries = p.nentries;
   for( int k = 0; k <= p.h; ++k ) { a.w[ k ] = static_cast< T >( p.taps[ k ] ); }
   for( int k = 0; k < p.nentries; ++k ) { a.e[ k ] = p.entries[ k ]; }
   if( a.nentries == 0 || a.nlines == 0 ) { return cudaSuccess; }
   // The entries come left halo first (j < 0), then right (j >= n); two threads per line when no
   // sample receives from both sides.
   a.split = 0;
   int split = 0;
   while( split < p.nentries && p.entries[ split ].j < 0 ) { ++split; }
   if( split > 0 && split < p.nentries ) {
      bool disjoint = true;
      for( int k = 0; k < split && disjoint; ++k ) {
         for( int m = split; m < p.nentries; ++m ) { disjoint &= p.entries[ k ].i != p.entries[ m ].i; }
      }
      if( disjoint ) { a.split = split; }
   }
   int64_t const threads = a.nlines * ( a.split > 0 ? 2 : 1 );
   int64_t blocks = ( threads + 127 ) / 128;
   if( blocks > 0x7fffffff ) { return cudaErrorInvalidValue; }
   fold_kernel< T ><<< static_cast< unsigned >( blocks ), 128, 0, s >>>( a ); count_launch();
   return cudaGetLastError();
}

} // namespace

cudaError_t launch_fold( FoldPass const& p, cudaStream_t stream ) {
   if( p.h < 0 || p.h > kFoldMaxHalf || p.nentries > kFoldMaxEntries ) { return cudaErrorInvalidValue; }
   if( !p.compute_double && p.h >= 1 && p.h <= 16 ) {
      cudaError_t const e = p.h <= 4 ? run_fold_fast< 4 >( p, stream ) : p.h <= 8 ? run_fold_fast< 8 >( p, stream )
                                                                          : run_fold_fast< 16 >( p, stream );
      if( e != cudaErrorNotSupported ) { return e; }
   }
   return p.compute_double ? run_fold< double >( p, stream ) : run_fold< float >( p, stream );
}

cudaError_t launch_dot( ConvertArgs const& a, bool compute_double, double* out, cudaStream_t stream ) {
   int64_t blocks = ( a.total + 255 ) / 256;
   if( blocks > 148 * 8 ) { blocks = 148 * 8; }
   if( blocks < 1 ) { blocks = 1; }
   if( compute_double ) {
      dot_kernel< double ><<< static_cast< unsigned >( blocks ), 256, 0, stream >>>( a, out ); count_launch();
   } else {
      dot_kernel< float ><<< static_cast< unsigned >( blocks ), 256, 0, stream >>>( a, out ); count_launch();
   }
   return cudaGetLastError();
}

} // namespace dipcu
