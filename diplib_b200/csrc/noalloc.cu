// dipcu_gauss_fir_noalloc: the Gaussian FIR with the pass intermediates in a fixed, statically
// allocated device array instead of memory obtained from cudaMallocAsync.
//
// Who needs it: code that runs the filter where device memory must not be requested at call
// time -- a process whose GPU memory is entirely handed out by another allocator (a framework's
// caching allocator, or a pool reserved at start-up) and must not grow its footprint behind that
// allocator's back, or a long-running pipeline that must not fail for lack of memory once it has
// started.  Such callers still pass their own input and output images; everything else the
// filter needs is in the static array below.
//
// The array is part of this library's device code: every GPU on which the library is used holds
// it (kNoAllocScratchBytes) until the process exits.  It holds two intermediate images of up to
// kNoAllocScratchBytes / 2 bytes each, which limits images to 4 Mi samples when the filter
// computes in float (input up to 16 bits or sfloat) and 2 Mi samples when it computes in double
// (32/64-bit integer or dfloat input).  Larger images are rejected with DIPCU_ERR_INVALID_ARG.
//
// All calls share the array and it keeps whatever the last call left in it.  Nothing in it has to
// start at zero: every pass writes each intermediate sample before the next pass reads it.  Calls
// whose work overlaps on the GPU (on different streams, or from different host threads without
// ordering) race on the array and give wrong results; order them on one stream.
//
// The first call on a device looks up the array's device address (cudaGetSymbolAddress) with that
// device current; make that first call before any stream capture on the device.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

namespace {

constexpr size_t kNoAllocScratchBytes = size_t( 32 ) << 20;

// The scratch.  In host code `g_noalloc_scratch` is only a stand-in symbol, never a device
// address: its address on a device comes from cudaGetSymbolAddress (noalloc_scratch_ptr).
static __device__ __align__( 256 ) unsigned char g_noalloc_scratch[ kNoAllocScratchBytes ];

// Device address of the scratch on the current device, looked up once per device.
unsigned char* noalloc_scratch_ptr( cudaError_t* err ) {
   static std::mutex mu;
   static unsigned char* ptrs[ 64 ] = {};
   int dev = 0;
   *err = cudaGetDevice( &dev );
   if( *err != cudaSuccess ) { return nullptr; }
   if( dev < 0 || dev >= 64 ) { *err = cudaErrorInvalidDevice; return nullptr; }
   std::lock_guard< std::mutex > lock( mu );
   if( !ptrs[ dev ] ) {
      void* p = nullptr;
      *err = cudaGetSymbolAddress( &p, g_noalloc_scratch );
      if( *err != cudaSuccess ) { return nullptr; }
      ptrs[ dev ] = static_cast< unsigned char* >( p );
   }
   return ptrs[ dev ];
}

} // namespace

} // namespace dipcu

using namespace dipcu;

extern "C" int dipcu_gauss_fir_noalloc( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sigmas,
                                         uint32_t const* orders, int32_t const* bcs, double truncation, void* stream_ ) {
   cudaStream_t stream = static_cast< cudaStream_t >( stream_ );
   if( !in || !out || !in->data || !out->data || !sigmas || !orders || !bcs ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "dipcu_gauss_fir_noalloc: null argument" );
   }
   int const nd = in->ndims;
   if( nd < 1 || nd > DIPCU_MAX_DIMS || out->ndims != nd ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "dipcu_gauss_fir_noalloc: bad dimensionality" );
   }
   if( in->dtype < DT_BIN || in->dtype > DT_DFLOAT || out->dtype < DT_BIN || out->dtype > DT_DFLOAT ) {
      return record_error( DIPCU_ERR_UNSUPPORTED_DTYPE, "Data type not supported" );
   }
   int64_t n = 1;
   for( int d = 0; d < nd; ++d ) {
      if( in->sizes[ d ] < 1 || out->sizes[ d ] != in->sizes[ d ] ) {
         return record_error( DIPCU_ERR_SIZES_DONT_MATCH, "Sizes don't match" );
      }
      if( out->strides[ d ] == 0 && out->sizes[ d ] > 1 ) {
         return record_error( DIPCU_ERR_INVALID_ARG, "out: zero stride along an axis of size > 1" );
      }
      n *= in->sizes[ d ];
   }
   {
      // The input and output must not overlap (DIPlib strips an overlapping output first).
      auto range = []( dipcu_image_desc const* d, uintptr_t& lo, uintptr_t& hi ) {
         int64_t mn = 0, mx = 0;
         for( int k = 0; k < d->ndims; ++k ) {
            int64_t ext = ( d->sizes[ k ] - 1 ) * d->strides[ k ];
            if( ext < 0 ) { mn += ext; } else { mx += ext; }
         }
         int64_t es = dtype_size( d->dtype );
         lo = reinterpret_cast< uintptr_t >( d->data ) + static_cast< uintptr_t >( mn * es );
         hi = reinterpret_cast< uintptr_t >( d->data ) + static_cast< uintptr_t >(( mx + 1 ) * es );
      };
      uintptr_t ilo, ihi, olo, ohi;
      range( in, ilo, ihi );
      range( out, olo, ohi );
      if( ilo < ohi && olo < ihi ) {
         return record_error( DIPCU_ERR_INVALID_ARG, "out overlaps in (strip the output image first)" );
      }
   }
   cudaError_t e = cudaSuccess;
   unsigned char* scratch = noalloc_scratch_ptr( &e );
   if( !scratch ) {
      std::string msg = std::string( "dipcu_gauss_fir_noalloc: cudaGetSymbolAddress: " ) + cudaGetErrorString( e );
      return record_error( DIPCU_ERR_CUDA, msg.c_str() );
   }
   bool const weights_double = in->dtype == DT_DFLOAT;
   int32_t const buf_dt = suggest_flex( in->dtype );
   bool const compute_double = buf_dt == DT_DFLOAT;
   size_t const esz = compute_double ? 8 : 4;
   size_t const max_samples = ( kNoAllocScratchBytes / 2 ) / esz;
   if( static_cast< size_t >( n ) > max_samples ) {
      std::string msg = "dipcu_gauss_fir_noalloc: the image has " + std::to_string( n ) +
                        " samples; the static scratch holds images of at most " + std::to_string( max_samples ) +
                        " samples for this input type";
      return record_error( DIPCU_ERR_INVALID_ARG, msg.c_str() );
   }

   // Filter set-up as dip::GaussFIR (src/linear/gauss.cpp:255-284).
   struct Axis { bool process = false; int64_t h = 0; int32_t odd = 0, bc = 0; std::vector< double > taps; };
   std::vector< Axis > f( static_cast< size_t >( nd ));
   for( int d = 0; d < nd; ++d ) {
      if( !( sigmas[ d ] > 0.0 ) || in->sizes[ d ] <= 1 ) { continue; }
      if( orders[ d ] > 3 ) {
         return record_error( DIPCU_ERR_ORDER_GT_3, "Gaussian FIR filter not implemented for order > 3" );
      }
      if( bcs[ d ] < 0 || bcs[ d ] > BC_THIRD_ORDER_EXTRAPOLATE ) {
         return record_error( DIPCU_ERR_UNSUPPORTED_BC, "Boundary condition not recognized" );
      }
      Axis& a = f[ static_cast< size_t >( d ) ];
      int64_t len = half_gaussian_length( sigmas[ d ], orders[ d ], truncation, weights_double );
      if( len - 1 > kLineMaxHalf ) {
         return record_error( DIPCU_ERR_KERNEL_TOO_LARGE, "Gaussian kernel half-width exceeds 2048 samples" );
      }
      a.process = true;
      a.h = len - 1;
      a.odd = static_cast< int32_t >( orders[ d ] & 1u );
      a.bc = bcs[ d ];
      a.taps.resize( static_cast< size_t >( len ));
      make_half_gaussian< double >( sigmas[ d ], orders[ d ], len, a.taps.data(), nullptr );
      if( !compute_double ) {
         for( auto& t : a.taps ) { t = static_cast< double >( static_cast< float >( t )); }
      }
      if( len == 1 && a.taps[ 0 ] == 1.0 ) { a.process = false; }
   }
   std::vector< int > order;
   for( int d = 0; d < nd; ++d ) {
      if( f[ static_cast< size_t >( d ) ].process ) { order.push_back( d ); }
   }
   for( size_t i = 1; i < order.size(); ++i ) {     // by input stride, stable
      int e = order[ i ];
      size_t j = i;
      while( j > 0 && in->strides[ order[ j - 1 ] ] > in->strides[ e ] ) { order[ j ] = order[ j - 1 ]; --j; }
      order[ j ] = e;
   }
   if( order.empty() ) {
      ConvertArgs c{};
      c.src = in->data;
      c.dst = out->data;
      c.src_dt = in->dtype;
      c.dst_dt = out->dtype;
      c.ndims = nd;
      c.total = n;
      for( int d = 0; d < nd; ++d ) {
         c.sizes[ d ] = in->sizes[ d ];
         c.sst[ d ] = in->strides[ d ];
         c.dstst[ d ] = out->strides[ d ];
      }
      e = launch_convert( c, true, stream );
      if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
      return DIPCU_OK;
   }

   void* half[ 2 ] = { scratch, scratch + kNoAllocScratchBytes / 2 };
   // Line-kernel passes; no pass reads and writes the same buffer (as the allocating path).
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
   for( int p = 0; p < P; ++p ) {
      int const back = P - 1 - p;
      void* dst;
      int32_t dst_dt;
      int64_t const* dst_st;
      if( back == 0 ) {
         dst = out->data; dst_dt = out->dtype; dst_st = out->strides;
      } else if( out_is_buf ) {
         if( back % 2 == 0 ) { dst = out->data; dst_st = out->strides; } else { dst = half[ 0 ]; dst_st = normal; }
         dst_dt = buf_dt;
      } else {
         dst = half[ ( back - 1 ) % 2 ]; dst_dt = buf_dt; dst_st = normal;
      }
      Axis const& af = f[ static_cast< size_t >( order[ p ] ) ];
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
      e = launch_line_pass( lp, stream );
      if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
      src = dst;
      src_dt = dst_dt;
      src_st = dst_st;
   }
   return DIPCU_OK;
}
