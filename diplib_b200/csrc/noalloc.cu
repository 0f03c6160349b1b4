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
// Every call outside stream capture looks up the array's device address (cudaGetSymbolAddress)
// with the call's device current; a call under stream capture reuses the address found by the
// device's last call outside capture, so make one call on a device (after any device reset)
// before capturing one.  Arguments, checks, filter set-up and pass order are those of
// dipcu_gauss_fir (check_pair, build_filters, pass_order); the passes are its line-kernel chain.
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

// Device address of the scratch on the current device.  Looked up afresh on every call that is not
// being captured into a CUDA graph (a device reset or a new primary context can load the array at
// another address); a call under stream capture reuses the address of the device's last call
// outside capture.
unsigned char* noalloc_scratch_ptr( cudaStream_t stream, cudaError_t* err ) {
   static std::mutex mu;
   static unsigned char* ptrs[ 64 ] = {};
   int dev = 0;
   *err = cudaGetDevice( &dev );
   if( *err != cudaSuccess ) { return nullptr; }
   if( dev < 0 || dev >= 64 ) { *err = cudaErrorInvalidDevice; return nullptr; }
   cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
   *err = cudaStreamIsCapturing( stream, &cs );
   if( *err != cudaSuccess ) { return nullptr; }
   std::lock_guard< std::mutex > lock( mu );
   if( cs == cudaStreamCaptureStatusNone ) {
      void* p = nullptr;
      *err = cudaGetSymbolAddress( &p, g_noalloc_scratch );
      if( *err != cudaSuccess ) { return nullptr; }
      ptrs[ dev ] = static_cast< unsigned char* >( p );
   } else if( !ptrs[ dev ] ) {
      *err = cudaErrorStreamCaptureUnsupported;
      return nullptr;
   }
   return ptrs[ dev ];
}

} // namespace

} // namespace dipcu

using namespace dipcu;

extern "C" int dipcu_gauss_fir_noalloc( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sigmas,
                                         uint32_t const* orders, int32_t const* bcs, double truncation, void* stream_ ) {
   cudaStream_t stream = static_cast< cudaStream_t >( stream_ );
   // Arguments, filter set-up and pass order exactly as dipcu_gauss_fir.
   if( int st = check_pair( in, out )) { return st; }
   if( !sigmas || !orders || !bcs ) { return record_error( DIPCU_ERR_INVALID_ARG, "null parameter array" ); }
   std::vector< AxisFilter > f;
   if( int st = build_filters( in, sigmas, orders, bcs, truncation, f, nullptr )) { return st; }
   int64_t n = 1;
   for( int d = 0; d < in->ndims; ++d ) { n *= in->sizes[ d ]; }
   bool const compute_double = suggest_flex( in->dtype ) == DT_DFLOAT;
   size_t const max_samples = ( kNoAllocScratchBytes / 2 ) / ( compute_double ? 8 : 4 );
   if( static_cast< size_t >( n ) > max_samples ) {
      std::string msg = "dipcu_gauss_fir_noalloc: the image has " + std::to_string( n ) +
                        " samples; the static scratch holds images of at most " + std::to_string( max_samples ) +
                        " samples for this input type";
      return record_error( DIPCU_ERR_INVALID_ARG, msg.c_str() );
   }
   std::vector< int > order = pass_order( in, f );
   if( order.empty() ) { return run_convert( in, out, stream ); }
   cudaError_t e = cudaSuccess;
   unsigned char* scratch = noalloc_scratch_ptr( stream, &e );
   if( !scratch ) {
      std::string msg = std::string( "dipcu_gauss_fir_noalloc: address of the static scratch: " ) + cudaGetErrorString( e );
      return record_error( DIPCU_ERR_CUDA, msg.c_str() );
   }
   // The line-kernel pass chain with its intermediates in the two halves of the static array.
   void* const half[ 2 ] = { scratch, scratch + kNoAllocScratchBytes / 2 };
   return run_line_passes( in, out, f, order, compute_double, half, stream );
}
