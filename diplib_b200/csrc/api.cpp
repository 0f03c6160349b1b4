// The C-ABI of libdipcu.so (include/dipcu.h): parameter validation with DIPlib's rules, the
// per-axis filter set-up of dip::GaussFIR, the pass planning of dip::Framework::Separable, and
// dispatch to the fused tile kernels (K1) or the line kernel (K2).
#include <atomic>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

cudaError_t launch_gauss_weights( double const* sigmas, uint32_t const* orders, int count, double truncation,
                                  float* weights, float* dweights, int32_t* lengths, int stride, cudaStream_t stream );

namespace {

thread_local std::string g_last_error;

int fail( int code, std::string const& msg ) {
   g_last_error = msg;
   return code;
}

int cuda_fail( cudaError_t e, char const* where ) {
   return fail( DIPCU_ERR_CUDA, std::string( where ) + ": " + cudaGetErrorString( e ));
}

bool valid_dtype( int32_t dt ) { return dt >= DT_BIN && dt <= DT_DFLOAT; }

int check_desc( dipcu_image_desc const* d, char const* name ) {
   if( !d ) { return fail( DIPCU_ERR_INVALID_ARG, std::string( name ) + ": null descriptor" ); }
   if( !d->data ) { return fail( DIPCU_ERR_INVALID_ARG, std::string( "Image is not forged" )); }
   if( d->ndims < 1 || d->ndims > DIPCU_MAX_DIMS ) {
      return fail( DIPCU_ERR_INVALID_ARG, std::string( name ) + ": dimensionality not supported" );
   }
   if( !valid_dtype( d->dtype )) { return fail( DIPCU_ERR_UNSUPPORTED_DTYPE, "Data type not supported" ); }
   for( int k = 0; k < d->ndims; ++k ) {
      if( d->sizes[ k ] < 1 ) { return fail( DIPCU_ERR_INVALID_ARG, std::string( name ) + ": sizes must be positive" ); }
   }
   return DIPCU_OK;
}

int64_t numel( dipcu_image_desc const* d ) {
   int64_t n = 1;
   for( int k = 0; k < d->ndims; ++k ) { n *= d->sizes[ k ]; }
   return n;
}

// Byte range touched by an image, for the overlap test.
void byte_range( dipcu_image_desc const* d, uintptr_t& lo, uintptr_t& hi ) {
   int64_t mn = 0, mx = 0;
   for( int k = 0; k < d->ndims; ++k ) {
      int64_t e = ( d->sizes[ k ] - 1 ) * d->strides[ k ];
      if( e < 0 ) { mn += e; } else { mx += e; }
   }
   int64_t es = dtype_size( d->dtype );
   lo = reinterpret_cast< uintptr_t >( d->data ) + static_cast< uintptr_t >( mn * es );
   hi = reinterpret_cast< uintptr_t >( d->data ) + static_cast< uintptr_t >(( mx + 1 ) * es );
}

// Try the fused tile kernels.  Returns true (with *err set) when it launched.
bool try_fused( dipcu_image_desc const* in, dipcu_image_desc const* out, std::vector< AxisFilter > const& f,
                std::vector< int > const& order, bool compute_double, cudaStream_t stream, cudaError_t* err ) {
   int const nd = in->ndims;
   int const np = static_cast< int >( order.size() );
   if( compute_double || out->dtype != DT_SFLOAT || getenv( "DIPCU_NO_FUSED" )) { return false; }   // switch for A/B timing
   if( !( in->dtype == DT_SFLOAT || in->dtype == DT_UINT16 || in->dtype == DT_UINT8 || in->dtype == DT_SINT16 )) { return false; }
   if( np != 2 && np != 3 ) { return false; }
   for( int d : order ) {
      if( !bc_is_index_map( f[ d ].bc ) || f[ d ].h >= kFusedMaxTaps ) { return false; }
   }
   // x: the processed axis with unit stride in both images; y, z: the others by input stride.
   int ax = -1;
   for( int d : order ) {
      if( in->strides[ d ] == 1 && out->strides[ d ] == 1 ) { ax = d; break; }
   }
   if( ax < 0 ) { return false; }
   std::vector< int > rest;
   for( int d : order ) { if( d != ax ) { rest.push_back( d ); } }
   if( rest.size() == 2 && std::llabs( in->strides[ rest[ 1 ] ] ) < std::llabs( in->strides[ rest[ 0 ] ] )) {
      std::swap( rest[ 0 ], rest[ 1 ] );
   }
   // At most one unfiltered axis of size > 1 (the batch axis).
   int batch = -1;
   for( int d = 0; d < nd; ++d ) {
      if( d == ax || ( rest.size() > 0 && d == rest[ 0 ] ) || ( rest.size() > 1 && d == rest[ 1 ] )) { continue; }
      if( in->sizes[ d ] > 1 ) {
         if( batch >= 0 ) { return false; }
         batch = d;
      }
   }
   int axes[ 3 ] = { ax, rest[ 0 ], np == 3 ? rest[ 1 ] : -1 };
   FusedKey key{};
   key.ndims = np;
   key.in_dt = in->dtype;
   for( int i = 0; i < np; ++i ) {
      key.h[ i ] = static_cast< int32_t >( f[ axes[ i ] ].h );
      key.odd[ i ] = f[ axes[ i ] ].odd;
   }
   FusedArgs a{};
   a.src = in->data;
   a.dst = static_cast< float* >( out->data );
   for( int i = 0; i < 3; ++i ) {
      if( i < np ) {
         int d = axes[ i ];
         a.n[ i ] = in->sizes[ d ];
         a.ss[ i ] = in->strides[ d ];
         a.ds[ i ] = out->strides[ d ];
         a.bc[ i ] = f[ d ].bc;
         for( int k = 0; k <= f[ d ].h; ++k ) { a.w[ i ][ k ] = static_cast< float >( f[ d ].taps[ k ] ); }
      } else {
         a.n[ i ] = 1;
         a.ss[ i ] = 0;
         a.ds[ i ] = 0;
         a.bc[ i ] = 0;
      }
   }
   if( batch >= 0 ) {
      a.nb = in->sizes[ batch ];
      a.sb = in->strides[ batch ];
      a.db = out->strides[ batch ];
   } else {
      a.nb = 1;
      a.sb = 0;
      a.db = 0;
   }
   if( np == 2 ) {
      // Half-widths up to 12: the warp-per-tile kernel (packed FMAs, no block barrier) is the
      // faster one; beyond, and for the layouts and conditions it hands back, the row march.
      *err = launch_fused2d_ws( key, a, stream );
      if( *err != cudaErrorNotSupported ) { return true; }
      *err = launch_march2d( key, a, stream );
      if( *err != cudaErrorNotSupported ) { return true; }
   }
   if( !fused_available( key )) { return false; }
   *err = launch_fused( key, a, stream );
   return *err != cudaErrorNotSupported;
}

} // namespace

int record_error( int code, char const* msg ) {
   return fail( code, msg );
}

int check_pair( dipcu_image_desc const* in, dipcu_image_desc const* out ) {
   if( int st = check_desc( in, "in" )) { return st; }
   if( int st = check_desc( out, "out" )) { return st; }
   int const nd = in->ndims;
   if( out->ndims != nd ) { return fail( DIPCU_ERR_SIZES_DONT_MATCH, "Sizes don't match" ); }
   for( int d = 0; d < nd; ++d ) {
      if( out->sizes[ d ] != in->sizes[ d ] ) { return fail( DIPCU_ERR_SIZES_DONT_MATCH, "Sizes don't match" ); }
      if( out->strides[ d ] == 0 && out->sizes[ d ] > 1 ) {
         return fail( DIPCU_ERR_INVALID_ARG, "out: zero stride along an axis of size > 1" );
      }
   }
   uintptr_t ilo, ihi, olo, ohi;
   byte_range( in, ilo, ihi );
   byte_range( out, olo, ohi );
   if( ilo < ohi && olo < ihi ) {
      return fail( DIPCU_ERR_INVALID_ARG, "out overlaps in (strip the output image first)" );
   }
   return DIPCU_OK;
}

int build_filters( dipcu_image_desc const* in, double const* sigmas, uint32_t const* orders, int32_t const* bcs,
                   double truncation, std::vector< AxisFilter >& f, std::vector< std::vector< double >>* dtaps ) {
   // dip::GaussFIR: weight precision follows the input (gauss.cpp:254); the line buffers and
   // the output use dip::DataType::SuggestFlex (convolution.cpp:341-343).
   int const nd = in->ndims;
   bool const weights_double = in->dtype == DT_DFLOAT;
   bool const compute_double = suggest_flex( in->dtype ) == DT_DFLOAT;
   f.assign( static_cast< size_t >( nd ), AxisFilter{} );
   if( dtaps ) { dtaps->assign( static_cast< size_t >( nd ), {} ); }
   for( int d = 0; d < nd; ++d ) {
      if( !( sigmas[ d ] > 0.0 ) || in->sizes[ d ] <= 1 ) { continue; }
      if( orders[ d ] > 3 ) {
         return fail( DIPCU_ERR_ORDER_GT_3, "Gaussian FIR filter not implemented for order > 3" );
      }
      if( bcs[ d ] < 0 || bcs[ d ] > BC_THIRD_ORDER_EXTRAPOLATE ) {
         return fail( DIPCU_ERR_UNSUPPORTED_BC, bcs[ d ] == BC_ALREADY_EXPANDED
                                                ? "Boundary condition \"already expanded\" is not supported"
                                                : "Boundary condition not recognized" );
      }
      AxisFilter& a = f[ static_cast< size_t >( d ) ];
      int64_t len = half_gaussian_length( sigmas[ d ], orders[ d ], truncation, weights_double );
      if( len - 1 > kLineMaxHalf ) {
         return fail( DIPCU_ERR_KERNEL_TOO_LARGE, "Gaussian kernel half-width exceeds 2048 samples" );
      }
      a.process = true;
      a.h = len - 1;
      a.odd = static_cast< int32_t >( orders[ d ] & 1u );
      a.bc = bcs[ d ];
      a.taps.resize( static_cast< size_t >( len ));
      std::vector< double >* dt = dtaps ? &( *dtaps )[ static_cast< size_t >( d ) ] : nullptr;
      if( dt ) { dt->resize( static_cast< size_t >( len )); }
      make_half_gaussian< double >( sigmas[ d ], orders[ d ], len, a.taps.data(), dt ? dt->data() : nullptr );
      if( !compute_double ) {
         for( auto& t : a.taps ) { t = static_cast< double >( static_cast< float >( t )); }
         if( dt ) { for( auto& t : *dt ) { t = static_cast< double >( static_cast< float >( t )); } }
      }
      // IsMeaninglessFilter (convolution.cpp:304-314): a single unit tap.
      if( len == 1 && a.taps[ 0 ] == 1.0 ) { a.process = false; }
   }
   return DIPCU_OK;
}

std::vector< int > pass_order( dipcu_image_desc const* in, std::vector< AxisFilter > const& f ) {
   // Framework::Separable: by input stride, stable (framework_separable.cpp:146-165).
   std::vector< int > order;
   for( int d = 0; d < in->ndims; ++d ) {
      if( f[ static_cast< size_t >( d ) ].process ) { order.push_back( d ); }
   }
   for( size_t i = 1; i < order.size(); ++i ) {
      int e = order[ i ];
      size_t j = i;
      while( j > 0 && in->strides[ order[ j - 1 ] ] > in->strides[ e ] ) { order[ j ] = order[ j - 1 ]; --j; }
      order[ j ] = e;
   }
   return order;
}

int run_convert( dipcu_image_desc const* in, dipcu_image_desc const* out, cudaStream_t stream ) {
   int const nd = in->ndims;
   ConvertArgs c{};
      c.src = in->data;
      c.dst = out->data;
      c.src_dt = in->dtype;
      c.dst_dt = out->dtype;
      c.ndims = nd;
      c.total = numel( in );
      for( int d = 0; d < nd; ++d ) {
         c.sizes[ d ] = in->sizes[ d ];
         c.sst[ d ] = in->strides[ d ];
         c.dstst[ d ] = out->strides[ d ];
      }
   cudaError_t e = launch_convert( c, true, stream );
   if( e != cudaSuccess ) { return cuda_fail( e, "convert_kernel" ); }
   return DIPCU_OK;
}

int line_pass_scratch_images( int passes, bool out_is_buf ) {
   if( passes <= 1 ) { return 0; }
   return ( out_is_buf || passes == 2 ) ? 1 : 2;
}

int run_line_passes( dipcu_image_desc const* in, dipcu_image_desc const* out, std::vector< AxisFilter > const& f,
                     std::vector< int > const& order, bool compute_double, void* const scratch[ 2 ], cudaStream_t stream ) {
   // No pass reads and writes the same buffer: the last pass writes `out`, earlier ones alternate
   // between `out` (when it has the buffer type) and the scratch images (normal strides).
   int const nd = in->ndims;
   int32_t const buf_dt = compute_double ? DT_DFLOAT : DT_SFLOAT;
   int const P = static_cast< int >( order.size() );
   bool const out_is_buf = out->dtype == buf_dt;
   int64_t normal[ DIPCU_MAX_DIMS ];
   {
      int64_t s = 1;
      for( int d = 0; d < nd; ++d ) { normal[ d ] = s; s *= in->sizes[ d ]; }
   }
   void const* src = in->data;
   int32_t src_dt = in->dtype;
   int64_t const* src_st = in->strides;
   int status = DIPCU_OK;
   for( int p = 0; p < P; ++p ) {
      int const back = P - 1 - p;   // passes after this one
      void* dst;
      int32_t dst_dt;
      int64_t const* dst_st;
      if( back == 0 ) {
         dst = out->data; dst_dt = out->dtype; dst_st = out->strides;
      } else if( out_is_buf ) {
         if( back % 2 == 0 ) { dst = out->data; dst_st = out->strides; } else { dst = scratch[ 0 ]; dst_st = normal; }
         dst_dt = buf_dt;
      } else {
         dst = scratch[ ( back - 1 ) % 2 ]; dst_dt = buf_dt; dst_st = normal;
      }
      AxisFilter const& af = f[ static_cast< size_t >( order[ p ] ) ];
      LinePass lp{};
      lp.src = src;
      lp.dst = dst;
      lp.src_dt = src_dt;
      lp.dst_dt = dst_dt;
      lp.ndims = nd;
      lp.axis = order[ p ];
      for( int d = 0; d < nd; ++d ) {
         lp.sizes[ d ] = in->sizes[ d ];
         lp.src_strides[ d ] = src_st[ d ];
         lp.dst_strides[ d ] = dst_st[ d ];
      }
      lp.h = af.h;
      lp.odd = af.odd;
      lp.bc = af.bc;
      lp.compute_double = compute_double;
      lp.taps = af.taps.data();
      lp.mode = af.mode;
      lp.lo = af.lo;
      lp.hi = af.hi;
      lp.usize = af.usize;
      lp.full = af.full.data();
      cudaError_t e = launch_line_pass( lp, stream );
      if( e != cudaSuccess ) { status = cuda_fail( e, "line_pass_kernel" ); break; }
      src = dst;
      src_dt = dst_dt;
      src_st = dst_st;
   }
   return status;
}

int run_filters( dipcu_image_desc const* in, dipcu_image_desc const* out, std::vector< AxisFilter > const& f,
                 bool compute_double, cudaStream_t stream ) {
   std::vector< int > order = pass_order( in, f );
   if( order.empty() ) { return run_convert( in, out, stream ); }

   cudaError_t ferr = cudaSuccess;
   if( try_fused( in, out, f, order, compute_double, stream, &ferr )) {
      if( ferr != cudaSuccess ) { return cuda_fail( ferr, "fused tile kernel" ); }
      return DIPCU_OK;
   }

   // Line kernel passes with their intermediates from the stream-ordered allocator.
   int32_t const buf_dt = compute_double ? DT_DFLOAT : DT_SFLOAT;
   int const nscratch = line_pass_scratch_images( static_cast< int >( order.size() ), out->dtype == buf_dt );
   size_t const bytes = static_cast< size_t >( numel( in )) * ( compute_double ? 8 : 4 );
   void* scratch[ 2 ] = { nullptr, nullptr };
   for( int i = 0; i < nscratch; ++i ) {
      cudaError_t e = cudaMallocAsync( &scratch[ i ], bytes, stream );
      if( e != cudaSuccess ) {
         for( int j = 0; j < i; ++j ) { cudaFreeAsync( scratch[ j ], stream ); }
         return cuda_fail( e, "cudaMallocAsync (pass intermediate)" );
      }
   }
   int status = run_line_passes( in, out, f, order, compute_double, scratch, stream );
   for( int i = 0; i < nscratch; ++i ) { cudaFreeAsync( scratch[ i ], stream ); }
   return status;
}

namespace {
std::atomic< uint64_t > g_launches{ 0 };
} // namespace

void count_launch() { g_launches.fetch_add( 1, std::memory_order_relaxed ); }
uint64_t launches_so_far() { return g_launches.load( std::memory_order_relaxed ); }

} // namespace dipcu

using namespace dipcu;

extern "C" {

char const* dipcu_last_error_message( void ) {
   return g_last_error.c_str();
}

char const* dipcu_version( void ) {
   return "dipcu 0.1 (sm_100a)";
}

uint64_t dipcu_launch_count( void ) {
   return dipcu::launches_so_far();
}

int dipcu_bc_from_string( char const* bc ) {
   // dip::StringToBoundaryCondition, include/diplib/boundary.h:87-103.
   static char const* const names[] = {
      "mirror", "asym mirror", "antisym reflect", "periodic", "asym periodic", "add zeros", "add max",
      "add min", "zero order", "first order", "second order", "third order", "already expanded" };
   if( !bc || bc[ 0 ] == 0 || std::strcmp( bc, "default" ) == 0 ) { return BC_SYMMETRIC_MIRROR; }
   for( int i = 0; i < 13; ++i ) {
      if( std::strcmp( bc, names[ i ] ) == 0 ) { return i; }
   }
   g_last_error = std::string( "Boundary condition not recognized: " ) + bc;
   return -1;
}

int dipcu_half_gaussian_length( double sigma, uint32_t order, double truncation, int dt_double ) {
   if( order > 3 ) { return -1; }
   return static_cast< int >( half_gaussian_length( sigma, order, truncation, dt_double != 0 ));
}

int dipcu_make_gauss_weights( double const* sigmas, uint32_t const* orders, int count, double truncation,
                              float* weights, float* dweights, int32_t* lengths, int stride, void* stream ) {
   if( count < 0 || stride < 1 || ( count > 0 && ( !sigmas || !orders || !weights ))) {
      return fail( DIPCU_ERR_INVALID_ARG, "dipcu_make_gauss_weights: bad arguments" );
   }
   cudaError_t e = launch_gauss_weights( sigmas, orders, count, truncation, weights, dweights, lengths, stride,
                                         static_cast< cudaStream_t >( stream ));
   if( e != cudaSuccess ) { return cuda_fail( e, "gauss_weights_kernel" ); }
   return DIPCU_OK;
}

int dipcu_gauss_fir( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sigmas,
                     uint32_t const* orders, int32_t const* bcs, double truncation, void* stream_ ) {
   cudaStream_t stream = static_cast< cudaStream_t >( stream_ );
   if( int st = check_pair( in, out )) { return st; }
   if( !sigmas || !orders || !bcs ) { return fail( DIPCU_ERR_INVALID_ARG, "null parameter array" ); }
   std::vector< AxisFilter > f;
   if( int st = build_filters( in, sigmas, orders, bcs, truncation, f, nullptr )) { return st; }
   return run_filters( in, out, f, suggest_flex( in->dtype ) == DT_DFLOAT, stream );
}

} // extern "C"
