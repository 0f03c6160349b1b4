// dip::GaussFT on the device (src/linear/gauss.cpp:397-487 in DIPlib): the Gaussian (derivative)
// filter applied in the Fourier domain, spatial input and output.
//
// Pipeline, one stream:
//   1. gather: the input, extended by the boundary condition to the transform sizes (dip::Gauss's
//      ExpandInput, gauss.cpp:380-393: each size grown by twice the half Gaussian size, then to
//      the next 5-smooth length, the image centred as ExtendImageToSize places it), written as a
//      complex array with the spatial origin (index n/2 of the centred convention) at index 0;
//   2. forward complex transform (cuFFT, all axes);
//   3. spectrum: the reference's real-to-complex transform (src/transform/fourier.cpp:247-282,
//      387-441) runs along one axis r and, for an odd length along r, leaves the outermost
//      frequency of its half line unconjugated, so the spectrum it hands on has the planes
//      k_r = +M and k_r = -M swapped (M = (n_r - 1) / 2); that swap is reproduced, the spectrum
//      multiplied by every axis' look-up table (GaussFTLineFilter, gauss.cpp:290-360), and, as
//      the reference's complex-to-real inverse uses only the half k_r <= 0, the half k_r > 0 is
//      replaced by the Hermitian completion of the other half;
//   4. inverse complex transform (cuFFT);
//   5. scatter: the real part scaled by 1 / (number of samples), shifted back to the centred
//      origin, cropped to the input's sizes and written in the output's type.
// The computation type is DataType::SuggestComplex of the input (double for 32/64-bit integers
// and dfloat, else float), as in the reference.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <complex>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

namespace {

constexpr int kFtMaxDims = 3;   // cuFFT transforms of rank 1..3

struct FtGeom {
   int32_t nd;
   int32_t r;                         // the axis of the reference's real-to-complex transform
   int32_t swap;                      // 1: swap the planes k_r = M and k_r = n_r - M
   int64_t n[ kFtMaxDims ];           // transform sizes, DIPlib order (x first)
   int64_t sz[ kFtMaxDims ];          // input / output sizes
   int64_t origin[ kFtMaxDims ];      // input origin inside the transform array
   int32_t bc[ kFtMaxDims ];
   int64_t total;
};

template< typename T > struct Cplx;
template<> struct Cplx< float > { using type = float2; };
template<> struct Cplx< double > { using type = double2; };

// Transform element m (x fastest) -> the extended input sample at the centred position.
template< typename T >
__global__ void ft_gather_kernel( FtGeom g, void const* __restrict__ src, int32_t src_dt, int64_t s0, int64_t s1, int64_t s2,
                                  typename Cplx< T >::type* __restrict__ x ) {
   int64_t const st[ 3 ] = { s0, s1, s2 };
   for( int64_t m = blockIdx.x * static_cast< int64_t >( blockDim.x ) + threadIdx.x; m < g.total;
        m += static_cast< int64_t >( gridDim.x ) * blockDim.x ) {
      int64_t rem = m, off = 0;
      bool zero = false, neg = false;
      for( int d = 0; d < g.nd; ++d ) {
         int64_t const k = rem % g.n[ d ];
         rem /= g.n[ d ];
         int64_t j = k + g.n[ d ] / 2;                // the spatial origin sits at index n/2
         if( j >= g.n[ d ] ) { j -= g.n[ d ]; }
         int64_t s = j - g.origin[ d ];
         if( s < 0 || s >= g.sz[ d ] ) {
            if( g.bc[ d ] == BC_ADD_ZEROS ) {
               zero = true;
               s = 0;
            } else {
               bool ng = false;
               s = bc_map_index( s, g.sz[ d ], g.bc[ d ], &ng );
               neg = neg != ng;
            }
         }
         off += s * st[ d ];
      }
      T v = zero ? T( 0 ) : load_as< T >( src, src_dt, off );
      if( neg ) { v = -v; }
      typename Cplx< T >::type c;
      c.x = v;
      c.y = T( 0 );
      x[ m ] = c;
   }
}

// Spectrum k: swapped, filtered, and the half k_r > 0 replaced by the Hermitian completion of
// the half k_r < 0.  `lut` holds every axis' table in unshifted frequency order, axis after axis.
template< typename T >
__global__ void ft_spectrum_kernel( FtGeom g, typename Cplx< T >::type const* __restrict__ x,
                                    typename Cplx< T >::type const* __restrict__ lut, typename Cplx< T >::type* __restrict__ y ) {
   using C = typename Cplx< T >::type;
   for( int64_t m = blockIdx.x * static_cast< int64_t >( blockDim.x ) + threadIdx.x; m < g.total;
        m += static_cast< int64_t >( gridDim.x ) * blockDim.x ) {
      int64_t k[ kFtMaxDims ] = { 0, 0, 0 };
      int64_t rem = m;
      for( int d = 0; d < g.nd; ++d ) {
         k[ d ] = rem % g.n[ d ];
         rem /= g.n[ d ];
      }
      int64_t const nr = g.n[ g.r ];
      bool const mirror = k[ g.r ] >= 1 && k[ g.r ] <= ( nr + 1 ) / 2 - 1;
      if( mirror ) {
         for( int d = 0; d < g.nd; ++d ) { k[ d ] = k[ d ] == 0 ? 0 : g.n[ d ] - k[ d ]; }
      }
      // the filtered spectrum at k (after the reference's swap along r)
      int64_t const m_r = ( nr - 1 ) / 2;
      int64_t kr = k[ g.r ];
      if( g.swap ) {
         if( kr == m_r ) { kr = nr - m_r; } else if( kr == nr - m_r ) { kr = m_r; }
      }
      int64_t idx = 0, stride = 1, loff = 0;
      T fr = T( 1 ), fi = T( 0 );
      for( int d = 0; d < g.nd; ++d ) {
         idx += ( d == g.r ? kr : k[ d ] ) * stride;
         stride *= g.n[ d ];
         C const l = lut[ loff + k[ d ]];
         T const nr_ = fr * l.x - fi * l.y;
         fi = fr * l.y + fi * l.x;
         fr = nr_;
         loff += g.n[ d ];
      }
      C const v = x[ idx ];
      C o;
      o.x = v.x * fr - v.y * fi;
      o.y = v.x * fi + v.y * fr;
      if( mirror ) { o.y = -o.y; }
      y[ m ] = o;
   }
}

// Output sample i: the real part of transform element (i + origin - n/2) mod n, scaled.
template< typename T >
__global__ void ft_scatter_kernel( FtGeom g, typename Cplx< T >::type const* __restrict__ y, T scale, void* __restrict__ dst,
                                   int32_t dst_dt, int64_t d0, int64_t d1, int64_t d2, int64_t count ) {
   int64_t const ds[ 3 ] = { d0, d1, d2 };
   for( int64_t i = blockIdx.x * static_cast< int64_t >( blockDim.x ) + threadIdx.x; i < count;
        i += static_cast< int64_t >( gridDim.x ) * blockDim.x ) {
      int64_t rem = i, idx = 0, stride = 1, off = 0;
      for( int d = 0; d < g.nd; ++d ) {
         int64_t const c = rem % g.sz[ d ];
         rem /= g.sz[ d ];
         int64_t j = c + g.origin[ d ] - g.n[ d ] / 2;
         if( j < 0 ) { j += g.n[ d ]; }
         idx += j * stride;
         stride *= g.n[ d ];
         off += c * ds[ d ];
      }
      store_from< T >( dst, dst_dt, off, y[ idx ].x * scale );
   }
}

// GetOptimalDFTSize( n, larger = true, maxFactor = 5 ) (src/transform/dft_optimal_size.cpp:168-184):
// the smallest 2^a 3^b 5^c >= n.
int64_t next_5_smooth( int64_t n ) {
   for( int64_t m = n < 1 ? 1 : n;; ++m ) {
      int64_t v = m;
      for( int64_t f : { 2, 3, 5 } ) {
         while( v % f == 0 ) { v /= f; }
      }
      if( v == 1 ) { return m; }
   }
}

// GaussFTLineFilter's table for one axis (src/linear/gauss.cpp:290-350): centred coordinates
// (origin n / 2), computed in the transform's precision T on the host, then returned in
// unshifted frequency order (element k holds the centred coordinate (k + n/2) mod n).
template< typename T >
void gauss_ft_lut( int64_t n, double sigma, uint32_t order, double truncation, std::vector< std::complex< T >>& out ) {
   using C = std::complex< T >;
   std::vector< C > lut( static_cast< size_t >( n ), C( 0, 0 ));
   int64_t const origin = n / 2;
   T b = static_cast< T >( 2.0 * M_PI * sigma ) / static_cast< T >( n );
   b = -T( 0.5 ) * b * b;
   int64_t const hn = ( b == 0 ) ? n
                                 : half_gaussian_size( static_cast< double >( n ) / ( 2.0 * M_PI * sigma ), order, truncation,
                                                       std::is_same< T, double >::value );
   int64_t const begin = origin - hn > 0 ? origin - hn : 0;
   int64_t const end = origin + hn + 1 < n ? origin + hn + 1 : n;
   if( order > 0 ) {
      T const o = static_cast< T >( order );
      C a( 0, static_cast< T >( 2.0 * M_PI ) / static_cast< T >( n ));
      a = std::pow( a, o );
      for( int64_t j = begin; j < end; ++j ) {
         T const x = static_cast< T >( j - origin );
         lut[ static_cast< size_t >( j ) ] = ( b != 0 ) ? a * std::pow( x, o ) * std::exp( b * x * x ) : a * std::pow( x, o );
      }
   } else if( b != 0 ) {
      for( int64_t j = begin; j < end; ++j ) {
         T const x = static_cast< T >( j - origin );
         lut[ static_cast< size_t >( j ) ] = C( std::exp( b * x * x ), 0 );
      }
   } else {
      std::fill( lut.begin(), lut.end(), C( 1, 0 ));
   }
   size_t const base = out.size();
   out.resize( base + static_cast< size_t >( n ));
   for( int64_t k = 0; k < n; ++k ) { out[ base + static_cast< size_t >( k ) ] = lut[ static_cast< size_t >(( k + origin ) % n ) ]; }
}

// One cuFFT plan per (device, stream, sizes, precision): a plan's work area serves one
// execution at a time, and executions on one stream are ordered.
std::mutex g_plan_mu;
std::map< std::tuple< int, void*, int, int64_t, int64_t, int64_t, bool >, cufftHandle > g_plans;

int get_plan( FtGeom const& g, bool dbl, cudaStream_t stream, cufftHandle* plan ) {
   int dev = 0;
   cudaGetDevice( &dev );
   auto key = std::make_tuple( dev, static_cast< void* >( stream ), g.nd, g.n[ 0 ], g.nd > 1 ? g.n[ 1 ] : 1,
                               g.nd > 2 ? g.n[ 2 ] : 1, dbl );
   std::lock_guard< std::mutex > lock( g_plan_mu );
   auto it = g_plans.find( key );
   if( it != g_plans.end() ) {
      *plan = it->second;
      return DIPCU_OK;
   }
   int nrev[ kFtMaxDims ];
   for( int i = 0; i < g.nd; ++i ) { nrev[ i ] = static_cast< int >( g.n[ g.nd - 1 - i ] ); }   // slowest axis first
   cufftHandle h = 0;
   cufftResult r = cufftPlanMany( &h, g.nd, nrev, nullptr, 1, 0, nullptr, 1, 0, dbl ? CUFFT_Z2Z : CUFFT_C2C, 1 );
   if( r != CUFFT_SUCCESS ) {
      return record_error( DIPCU_ERR_CUDA, ( "cufftPlanMany failed: " + std::to_string( static_cast< int >( r ))).c_str() );
   }
   g_plans[ key ] = h;
   *plan = h;
   return DIPCU_OK;
}

int exec_fft( cufftHandle plan, bool dbl, void* data, int direction, cudaStream_t stream ) {
   std::lock_guard< std::mutex > lock( g_plan_mu );
   cufftResult r = cufftSetStream( plan, stream );
   if( r == CUFFT_SUCCESS ) {
      r = dbl ? cufftExecZ2Z( plan, static_cast< cufftDoubleComplex* >( data ), static_cast< cufftDoubleComplex* >( data ), direction )
              : cufftExecC2C( plan, static_cast< cufftComplex* >( data ), static_cast< cufftComplex* >( data ), direction );
   }
   if( r != CUFFT_SUCCESS ) {
      return record_error( DIPCU_ERR_CUDA, ( "cuFFT execution failed: " + std::to_string( static_cast< int >( r ))).c_str() );
   }
   return DIPCU_OK;
}

int grid_for( int64_t n ) {
   int64_t g = ( n + 255 ) / 256;
   return static_cast< int >( g < 148 * 16 ? ( g < 1 ? 1 : g ) : 148 * 16 );
}

template< typename T >
int run_gauss_ft( dipcu_image_desc const* in, dipcu_image_desc const* out, FtGeom const& g, std::vector< double > const& sig,
                  std::vector< uint32_t > const& ord, double truncation, cudaStream_t stream ) {
   using C = typename Cplx< T >::type;
   std::vector< std::complex< T >> lut;
   for( int d = 0; d < g.nd; ++d ) { gauss_ft_lut< T >( g.n[ d ], sig[ static_cast< size_t >( d ) ], ord[ static_cast< size_t >( d ) ], truncation, lut ); }
   cufftHandle plan = 0;
   bool const dbl = std::is_same< T, double >::value;
   if( int st = get_plan( g, dbl, stream, &plan )) { return st; }
   size_t const bytes = static_cast< size_t >( g.total ) * sizeof( C );
   void* x = nullptr;
   void* y = nullptr;
   void* dl = nullptr;
   cudaError_t e = cudaMallocAsync( &x, bytes, stream );
   if( e == cudaSuccess ) { e = cudaMallocAsync( &y, bytes, stream ); }
   if( e == cudaSuccess ) { e = cudaMallocAsync( &dl, lut.size() * sizeof( C ), stream ); }
   if( e == cudaSuccess ) { e = cudaMemcpyAsync( dl, lut.data(), lut.size() * sizeof( C ), cudaMemcpyHostToDevice, stream ); }
   int status = DIPCU_OK;
   if( e != cudaSuccess ) {
      status = record_error( DIPCU_ERR_CUDA, ( std::string( "GaussFT buffers: " ) + cudaGetErrorString( e )).c_str() );
   }
   if( status == DIPCU_OK ) {
      ft_gather_kernel< T ><<< grid_for( g.total ), 256, 0, stream >>>( g, in->data, in->dtype, in->strides[ 0 ],
                                                                          g.nd > 1 ? in->strides[ 1 ] : 0, g.nd > 2 ? in->strides[ 2 ] : 0,
                                                                          static_cast< C* >( x )); count_launch();
      status = exec_fft( plan, dbl, x, CUFFT_FORWARD, stream );
   }
   if( status == DIPCU_OK ) {
      ft_spectrum_kernel< T ><<< grid_for( g.total ), 256, 0, stream >>>( g, static_cast< C const* >( x ), static_cast< C const* >( dl ),
                                                                            static_cast< C* >( y )); count_launch();
      status = exec_fft( plan, dbl, y, CUFFT_INVERSE, stream );
   }
   if( status == DIPCU_OK ) {
      int64_t count = 1;
      for( int d = 0; d < g.nd; ++d ) { count *= g.sz[ d ]; }
      T const scale = static_cast< T >( 1.0 / static_cast< double >( g.total ));
      ft_scatter_kernel< T ><<< grid_for( count ), 256, 0, stream >>>( g, static_cast< C const* >( y ), scale, out->data, out->dtype,
                                                                         out->strides[ 0 ], g.nd > 1 ? out->strides[ 1 ] : 0,
                                                                         g.nd > 2 ? out->strides[ 2 ] : 0, count ); count_launch();
      e = cudaGetLastError();
      if( e != cudaSuccess ) { status = record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
   }
   if( x ) { cudaFreeAsync( x, stream ); }
   if( y ) { cudaFreeAsync( y, stream ); }
   if( dl ) { cudaFreeAsync( dl, stream ); }
   return status;
}

} // namespace

} // namespace dipcu

using namespace dipcu;

extern "C" {

int dipcu_gauss_ft( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sigmas, uint32_t const* orders,
                    double truncation, int32_t const* bcs, int nbcs, void* stream ) {
   if( int st = check_pair( in, out )) { return st; }
   if( !sigmas || !orders || nbcs < 0 || ( nbcs > 0 && !bcs )) { return record_error( DIPCU_ERR_INVALID_ARG, "null parameter array" ); }
   int const nd = in->ndims;
   if( nd > kFtMaxDims ) { return record_error( DIPCU_ERR_INVALID_ARG, "GaussFT: images of up to 3 dimensions" ); }
   if( nbcs != 0 && nbcs != nd ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "Array parameter has the wrong number of elements" );
   }
   // Parameters as GaussFT sets them up (gauss.cpp:416-432): an axis of size 1 is not filtered,
   // a negative sigma means no smoothing.
   std::vector< double > sig( static_cast< size_t >( nd ));
   std::vector< uint32_t > ord( static_cast< size_t >( nd ));
   bool any = false;
   for( int d = 0; d < nd; ++d ) {
      size_t const i = static_cast< size_t >( d );
      sig[ i ] = sigmas[ d ] < 0 ? 0.0 : sigmas[ d ];
      ord[ i ] = orders[ d ];
      if( in->sizes[ d ] == 1 ) {
         sig[ i ] = 0.0;
         ord[ i ] = 0;
      }
      any = any || sig[ i ] != 0.0 || ord[ i ] != 0;
   }
   cudaStream_t const s = static_cast< cudaStream_t >( stream );
   if( !any ) { return run_convert( in, out, s ); }
   bool const dbl = suggest_flex( in->dtype ) == DT_DFLOAT;
   FtGeom g{};
   g.nd = nd;
   g.total = 1;
   bool const expand = nbcs > 0;
   for( int d = 0; d < nd; ++d ) {
      size_t const i = static_cast< size_t >( d );
      g.sz[ d ] = in->sizes[ d ];
      if( expand ) {
         int32_t const bc = bcs[ d ];
         if( !bc_is_index_map( bc )) {
            return record_error( DIPCU_ERR_UNSUPPORTED_BC,
                                 "GaussFT: the boundary extension supports mirror, periodic (and their asymmetric forms), "
                                 "zero order and add zeros" );
         }
         g.bc[ d ] = bc;
         int64_t const h = half_gaussian_size( sig[ i ], ord[ i ], truncation, in->dtype == DT_DFLOAT );
         g.n[ d ] = next_5_smooth( in->sizes[ d ] + 2 * h );
         // GetWindowOrigin for CENTER (src/library/image_manip.cpp:557-566)
         g.origin[ d ] = ( g.n[ d ] - g.sz[ d ] ) / 2 + ((( g.n[ d ] & 1 ) == 0 && ( g.sz[ d ] & 1 ) == 1 ) ? 1 : 0 );
      } else {
         g.bc[ d ] = BC_ADD_ZEROS;   // never consulted: the transform covers exactly the input
         g.n[ d ] = in->sizes[ d ];
         g.origin[ d ] = 0;
      }
      if( g.n[ d ] > 0x7fffffff ) { return record_error( DIPCU_ERR_INVALID_ARG, "GaussFT: transform too large" ); }
      g.total *= g.n[ d ];
   }
   // The axis of the reference's real-to-complex transform (src/transform/fourier.cpp:532-559):
   // the first axis, replaced by a later one longer than 2 when the current one has at most 2
   // samples or a larger stride (strides of the transformed image: the fresh extended image, or
   // the input itself without extension).
   int64_t st[ kFtMaxDims ];
   int64_t acc = 1;
   for( int d = 0; d < nd; ++d ) {
      st[ d ] = expand ? acc : ( in->strides[ d ] < 0 ? -in->strides[ d ] : in->strides[ d ] );
      acc *= g.n[ d ];
   }
   g.r = 0;
   for( int d = 1; d < nd; ++d ) {
      if( g.n[ d ] > 2 && ( g.n[ g.r ] <= 2 || st[ d ] < st[ g.r ] )) { g.r = d; }
   }
   g.swap = ( g.n[ g.r ] > 2 && ( g.n[ g.r ] & 1 ) == 1 ) ? 1 : 0;
   return dbl ? run_gauss_ft< double >( in, out, g, sig, ord, truncation, s ) : run_gauss_ft< float >( in, out, g, sig, ord, truncation, s );
}

} // extern "C"
