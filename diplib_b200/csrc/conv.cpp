// The C-ABI of the two other separable filters on the same pass machinery as the Gaussian:
// dip::SeparableConvolution with real filters of any symmetry (src/linear/convolution.cpp:67-162,
// 319-421 in DIPlib) and dip::Uniform with a rectangular kernel (src/linear/uniform.cpp:68-86,
// 147-163).  Validation, filter interning and the per-axis border follow the reference; the
// passes run on the line kernel (general-filter mode, and the uniform filter's running sum).
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

namespace {

// InternOneDimensionalFilter (convolution.cpp:67-162) for a real filter, expanded to the full
// tap list of LinePass mode 1: out[i] = sum_j full[j + lo] x[i + j], j in [-lo, hi].  Returns a
// status; `meaningless` reports IsMeaninglessFilter (convolution.cpp:304-314).
int intern( dipcu_filter_1d const& fin, bool dbl, AxisFilter& af, bool& meaningless ) {
   int64_t const ds = fin.size;
   if( ds < 0 || ( ds > 0 && !fin.weights )) { return record_error( DIPCU_ERR_INVALID_ARG, "filter: bad weights" ); }
   int64_t size = ds;
   switch( fin.symmetry ) {
      case DIPCU_SYM_GENERAL: break;
      case DIPCU_SYM_EVEN: case DIPCU_SYM_ODD: size = ds > 0 ? 2 * ds - 1 : 0; break;
      case DIPCU_SYM_D_EVEN: case DIPCU_SYM_D_ODD: size = 2 * ds; break;
      default: return record_error( DIPCU_ERR_INVALID_ARG, "Symmetry string not recognized" );
   }
   meaningless = false;
   if( size == 0 ) { meaningless = true; return DIPCU_OK; }
   int64_t const o_in = fin.origin < 0 ? size / 2 : fin.origin;
   if( o_in >= size ) { return record_error( DIPCU_ERR_INVALID_ARG, "Origin outside of filter" ); }
   int64_t const origin = size - o_in - 1;                  // the reversed origin
   if( size > kGeneralMaxTaps ) {
      return record_error( DIPCU_ERR_KERNEL_TOO_LARGE, "filter longer than 256 taps" );
   }
   std::vector< double > f( static_cast< size_t >( ds ));   // CopyReverseData, in the compute precision
   for( int64_t k = 0; k < ds; ++k ) {
      double const v = fin.weights[ ds - 1 - k ];
      f[ static_cast< size_t >( k ) ] = dbl ? v : static_cast< double >( static_cast< float >( v ));
   }
   if( size == 1 && f[ 0 ] == 1.0 ) { meaningless = true; }
   af.mode = 1;
   // Tap span relative to the output sample: [-origin, size-1-origin], except for the two
   // even-sized symmetric kinds, whose loop (convolution.cpp:256-283) pairs in[r+k] with in[r-1-k],
   // r = i - origin + ds - 1, and so reads from i - origin - 1 to i - origin + size - 2.
   bool const dsym = fin.symmetry == DIPCU_SYM_D_EVEN || fin.symmetry == DIPCU_SYM_D_ODD;
   af.lo = dsym ? origin + 1 : origin;
   af.hi = dsym ? size - 2 - origin : size - 1 - origin;
   af.h = std::max( af.lo, af.hi );                          // covers the border of convolution.cpp:364-379
   af.full.assign( static_cast< size_t >( size ), 0.0 );
   auto at = [ & ]( int64_t j ) -> double& { return af.full[ static_cast< size_t >( j + af.lo ) ]; };
   switch( fin.symmetry ) {
      case DIPCU_SYM_GENERAL:          // sum_k f[k] x[i - origin + k]
         for( int64_t k = 0; k < ds; ++k ) { at( k - origin ) = f[ static_cast< size_t >( k ) ]; }
         break;
      case DIPCU_SYM_EVEN: case DIPCU_SYM_ODD: {   // centre at i - origin + ds - 1
         double const s = fin.symmetry == DIPCU_SYM_ODD ? -1.0 : 1.0;
         int64_t const m = ds - 1 - origin;
         at( m ) = f[ 0 ];
         for( int64_t k = 1; k < ds; ++k ) {
            at( m + k ) = f[ static_cast< size_t >( k ) ];
            at( m - k ) = s * f[ static_cast< size_t >( k ) ];
         }
         break;
      }
      default: {                       // D_EVEN / D_ODD: taps at r + k and r - 1 - k, r = i - origin + ds - 1
         double const s = fin.symmetry == DIPCU_SYM_D_ODD ? -1.0 : 1.0;
         int64_t const r = ds - 1 - origin;
         for( int64_t k = 0; k < ds; ++k ) {
            at( r + k ) = f[ static_cast< size_t >( k ) ];
            at( r - 1 - k ) = s * f[ static_cast< size_t >( k ) ];
         }
         break;
      }
   }
   if( af.hi < 0 ) {                   // the span ends left of the output sample: pad with zero taps
      af.full.resize( af.full.size() + static_cast< size_t >( -af.hi ), 0.0 );
      af.hi = 0;
      af.h = std::max( af.lo, af.hi );
      if( static_cast< int64_t >( af.full.size() ) > kGeneralMaxTaps ) {
         return record_error( DIPCU_ERR_KERNEL_TOO_LARGE, "filter longer than 256 taps" );
      }
   }
   return DIPCU_OK;
}

// The pass chain over `f` with stream-ordered intermediates (as the Gaussian's line-kernel path).
int run_chain( dipcu_image_desc const* in, dipcu_image_desc const* out, std::vector< AxisFilter > const& f,
               cudaStream_t stream ) {
   bool const compute_double = suggest_flex( in->dtype ) == DT_DFLOAT;
   std::vector< int > order = pass_order( in, f );
   if( order.empty() ) { return run_convert( in, out, stream ); }
   int32_t const buf_dt = compute_double ? DT_DFLOAT : DT_SFLOAT;
   int const nscratch = line_pass_scratch_images( static_cast< int >( order.size() ), out->dtype == buf_dt );
   int64_t n = 1;
   for( int d = 0; d < in->ndims; ++d ) { n *= in->sizes[ d ]; }
   size_t const bytes = static_cast< size_t >( n ) * ( compute_double ? 8 : 4 );
   void* scratch[ 2 ] = { nullptr, nullptr };
   for( int i = 0; i < nscratch; ++i ) {
      cudaError_t e = cudaMallocAsync( &scratch[ i ], bytes, stream );
      if( e != cudaSuccess ) {
         for( int j = 0; j < i; ++j ) { cudaFreeAsync( scratch[ j ], stream ); }
         std::string msg = std::string( "cudaMallocAsync (pass intermediate): " ) + cudaGetErrorString( e );
         return record_error( DIPCU_ERR_CUDA, msg.c_str() );
      }
   }
   int status = run_line_passes( in, out, f, order, compute_double, scratch, stream );
   for( int i = 0; i < nscratch; ++i ) { cudaFreeAsync( scratch[ i ], stream ); }
   return status;
}

bool bc_ok( int32_t bc ) { return bc >= 0 && bc <= BC_THIRD_ORDER_EXTRAPOLATE; }

} // namespace

} // namespace dipcu

using namespace dipcu;

extern "C" {

int dipcu_separable_convolution( dipcu_image_desc const* in, dipcu_image_desc const* out, dipcu_filter_1d const* filters,
                                 int nfilters, int32_t const* bcs, uint8_t const* process, void* stream ) {
   if( int st = check_pair( in, out )) { return st; }
   int const nd = in->ndims;
   if( !filters || !bcs || ( nfilters != 1 && nfilters != nd )) {
      return record_error( DIPCU_ERR_INVALID_ARG, "Array parameter has the wrong number of elements" );
   }
   bool const dbl = suggest_flex( in->dtype ) == DT_DFLOAT;
   std::vector< AxisFilter > interned( static_cast< size_t >( nfilters ));
   std::vector< char > meaningless( static_cast< size_t >( nfilters ), 0 );
   for( int i = 0; i < nfilters; ++i ) {
      bool m = false;
      if( int st = intern( filters[ i ], dbl, interned[ static_cast< size_t >( i ) ], m )) { return st; }
      meaningless[ static_cast< size_t >( i ) ] = m ? 1 : 0;
   }
   std::vector< AxisFilter > f( static_cast< size_t >( nd ));
   for( int d = 0; d < nd; ++d ) {
      int const i = nfilters == 1 ? 0 : d;
      bool proc = process ? process[ d ] != 0 : true;
      if( meaningless[ static_cast< size_t >( i ) ] || in->sizes[ d ] <= 1 ) { proc = false; }
      if( !proc ) { continue; }
      if( !bc_ok( bcs[ d ] )) {
         return record_error( DIPCU_ERR_UNSUPPORTED_BC, bcs[ d ] == BC_ALREADY_EXPANDED
                                                       ? "Boundary condition \"already expanded\" is not supported"
                                                       : "Boundary condition not recognized" );
      }
      f[ static_cast< size_t >( d ) ] = interned[ static_cast< size_t >( i ) ];
      f[ static_cast< size_t >( d ) ].process = true;
      f[ static_cast< size_t >( d ) ].bc = bcs[ d ];
   }
   return run_chain( in, out, f, static_cast< cudaStream_t >( stream ));
}

int dipcu_uniform( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sizes, int32_t const* bcs,
                   void* stream ) {
   if( int st = check_pair( in, out )) { return st; }
   if( !sizes || !bcs ) { return record_error( DIPCU_ERR_INVALID_ARG, "null parameter array" ); }
   int const nd = in->ndims;
   std::vector< AxisFilter > f( static_cast< size_t >( nd ));
   for( int d = 0; d < nd; ++d ) {
      // Kernel::Sizes for a rectangle (include/diplib/kernel.h:178-181): floor of sizes > 1, else 1.
      int64_t const sz = sizes[ d ] > 1.0 ? static_cast< int64_t >( sizes[ d ] ) : 1;
      if( sz <= 1 || in->sizes[ d ] <= 1 ) { continue; }
      if( !bc_ok( bcs[ d ] )) {
         return record_error( DIPCU_ERR_UNSUPPORTED_BC, bcs[ d ] == BC_ALREADY_EXPANDED
                                                       ? "Boundary condition \"already expanded\" is not supported"
                                                       : "Boundary condition not recognized" );
      }
      if( sz / 2 > kLineMaxHalf ) { return record_error( DIPCU_ERR_KERNEL_TOO_LARGE, "uniform filter too large" ); }
      AxisFilter& a = f[ static_cast< size_t >( d ) ];
      a.process = true;
      a.mode = 2;
      a.usize = sz;
      a.h = sz / 2;
      a.bc = bcs[ d ];
   }
   return run_chain( in, out, f, static_cast< cudaStream_t >( stream ));
}

} // extern "C"
