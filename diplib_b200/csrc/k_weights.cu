// K0: on-device construction of Gaussian kernel weights (and their sigma derivatives) for a
// table of (sigma, order) pairs held in device memory.  This is what lets a batch plan or an
// autograd graph change sigmas without a host round trip: the tables are rebuilt inside the
// captured work.  The arithmetic is dipcu_common.cuh's restatement of DIPlib's
// MakeHalfGaussian (src/linear/gauss.cpp:53-165), evaluated in double and stored as float.
#include <cuda_runtime.h>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

namespace {

__global__ void gauss_weights_kernel( double const* __restrict__ sigmas, uint32_t const* __restrict__ orders, int count,
                                      double truncation, float* weights, float* dweights, int32_t* lengths, int stride ) {
   int i = static_cast< int >( blockIdx.x * blockDim.x + threadIdx.x );
   if( i >= count ) { return; }
   double sigma = sigmas[ i ];
   uint32_t order = orders[ i ];
   if( order > 3 ) {
      if( lengths ) { lengths[ i ] = -1; }
      return;
   }
   int64_t len = half_gaussian_length( sigma, order, truncation, false );
   bool fits = len <= stride;
   if( lengths ) { lengths[ i ] = fits ? static_cast< int32_t >( len ) : -static_cast< int32_t >( len ); }
   if( !fits ) { return; }
   float* w = weights + static_cast< int64_t >( i ) * stride;
   float* dw = dweights ? dweights + static_cast< int64_t >( i ) * stride : nullptr;
   make_half_gaussian< float >( sigma, order, len, w, dw );
   for( int64_t k = len; k < stride; ++k ) {
      w[ k ] = 0.0f;
      if( dw ) { dw[ k ] = 0.0f; }
   }
}

} // namespace

cudaError_t launch_gauss_weights( double const* sigmas, uint32_t const* orders, int count, double truncation,
                                  float* weights, float* dweights, int32_t* lengths, int stride, cudaStream_t stream ) {
   if( count <= 0 ) { return cudaSuccess; }
   int threads = 64;
   int blocks = ( count + threads - 1 ) / threads;
   gauss_weights_kernel<<< blocks, threads, 0, stream >>>( sigmas, orders, count, truncation, weights, dweights, lengths, stride ); count_launch();
   return cudaGetLastError();
}

} // namespace dipcu
