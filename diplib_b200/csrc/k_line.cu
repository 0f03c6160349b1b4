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

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

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
   for( int k = 0; k <= p.h; ++k ) { a.taps[ k ] = static_cast< T >( p.taps[ k ] ); }

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
                                   static_cast< size_t >( smem ), stream >>>( a );
   return cudaGetLastError();
}

} // namespace

cudaError_t launch_line_pass( LinePass const& p, cudaStream_t stream ) {
   if( p.h < 0 || p.h > kLineMaxHalf ) { return cudaErrorInvalidValue; }
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
      convert_kernel< double ><<< static_cast< unsigned >( blocks ), 256, 0, stream >>>( a );
   } else {
      convert_kernel< float ><<< static_cast< unsigned >( blocks ), 256, 0, stream >>>( a );
   }
   return cudaGetLastError();
}

} // namespace dipcu
