// Structure tensor on the Gaussian FIR path, forward and backward.
//
// Forward, as dip::StructureTensor (src/analysis/structure_tensor.cpp:33-59 in DIPlib) with a
// Gaussian method and no mask: the gradient g_k = GaussFIR(in, sigma_g, order e_k) along each
// axis of size > 1 (dip::Gradient, src/linear/derivative.cpp:142-172), the symmetric products
// g_i g_j in DIPlib's symmetric-matrix order (diagonal first, then the upper triangle column by
// column, include/diplib/library/tensor.h:100-110, which for the m <= 3 axes here is also row by
// row; dip::Multiply( g, Transpose( g ))), and each product smoothed by GaussFIR(sigma_t).  The
// products are formed together and smoothed by one call over the component axis; when that much
// scratch is not available, per component (at most one product image at a time).
//
// Backward (no DIPlib counterpart): for L = sum_c <W_c, T_c>,
//   Q_c = S^T W_c (the smoothing's adjoint),
//   g_bar_k = sum over components (i, j) containing k of Q_c times the other factor,
//   in_bar  = sum_k D_k^T g_bar_k (the gradient filters' adjoints).
// The gradient images g_k are recomputed from the input here; the forward stores nothing.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

extern "C" int dipcu_gauss_fir_backward( dipcu_image_desc const* grad_out, dipcu_image_desc const* in,
                                          dipcu_image_desc const* grad_in, double* grad_sigma,
                                          double const* sigmas, uint32_t const* orders, int32_t const* bcs,
                                          double truncation, void* stream );

namespace dipcu {

namespace {

// dst[i] = a[i] * b[i] * s        (mode 0)
// dst[i] += a[i] * b[i] * s       (mode 1)
// dst[i] += a[i]                  (mode 2)
template< typename T >
__global__ void elementwise_kernel( T* dst, T const* a, T const* b, T s, int64_t n, int mode ) {
   for( int64_t i = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; i < n;
        i += static_cast< int64_t >( gridDim.x ) * blockDim.x ) {
      if( mode == 0 ) { dst[ i ] = a[ i ] * b[ i ] * s; }
      else if( mode == 1 ) { dst[ i ] = fma( a[ i ] * b[ i ], s, dst[ i ] ); }
      else { dst[ i ] += a[ i ]; }
   }
}

cudaError_t elementwise( bool dbl, void* dst, void const* a, void const* b, double s, int64_t n, int mode, cudaStream_t st ) {
   int64_t blocks = ( n + 255 ) / 256;
   if( blocks > 148 * 16 ) { blocks = 148 * 16; }
   if( blocks < 1 ) { blocks = 1; }
   if( dbl ) {
      elementwise_kernel< double ><<< static_cast< unsigned >( blocks ), 256, 0, st >>>(
            static_cast< double* >( dst ), static_cast< double const* >( a ), static_cast< double const* >( b ), s, n, mode ); count_launch();
   } else {
      elementwise_kernel< float ><<< static_cast< unsigned >( blocks ), 256, 0, st >>>(
            static_cast< float* >( dst ), static_cast< float const* >( a ), static_cast< float const* >( b ),
            static_cast< float >( s ), n, mode ); count_launch();
   }
   return cudaGetLastError();
}

// All products of the structure tensor in one pass: dst[c n + i] = g_{pi[c]}[i] g_{pj[c]}[i] for
// the nc <= 6 component pairs of m <= 3 gradient images (each gradient sample read once).
template< typename T >
struct ProdArgs {
   T const* g[ 3 ];
   T* dst;
   int64_t n;
   int32_t m, nc;
   int32_t pi[ 6 ], pj[ 6 ];
};

template< typename T >
__device__ __forceinline__ T pick3( T const* v, int k ) { return k == 0 ? v[ 0 ] : k == 1 ? v[ 1 ] : v[ 2 ]; }

template< typename T >
__global__ void __launch_bounds__( 256 ) products_kernel( ProdArgs< T > const __grid_constant__ a ) {
   for( int64_t i = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; i < a.n;
        i += static_cast< int64_t >( gridDim.x ) * blockDim.x ) {
      T v[ 3 ] = { T( 0 ), T( 0 ), T( 0 ) };
#pragma unroll
      for( int k = 0; k < 3; ++k ) { if( k < a.m ) { v[ k ] = a.g[ k ][ i ]; } }
#pragma unroll
      for( int c = 0; c < 6; ++c ) {
         if( c < a.nc ) { a.dst[ c * a.n + i ] = pick3( v, a.pi[ c ] ) * pick3( v, a.pj[ c ] ); }
      }
   }
}

// The gradient images' adjoints in one pass: for every component c = (i, j) in order,
// gb_i += 2 q_c g_i (i == j), else gb_i += q_c g_j and gb_j += q_c g_i -- the same operations, in
// the same order, as one accumulation launch per term; gb starts at zero.
template< typename T >
struct GbarArgs {
   T const* q;       // nc components, stride n
   T const* g[ 3 ];
   T* gb[ 3 ];
   int64_t n;
   int32_t m, nc;
   int32_t pi[ 6 ], pj[ 6 ];
};

template< typename T >
__global__ void __launch_bounds__( 256 ) gbar_kernel( GbarArgs< T > const __grid_constant__ a ) {
   for( int64_t i = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; i < a.n;
        i += static_cast< int64_t >( gridDim.x ) * blockDim.x ) {
      T v[ 3 ] = { T( 0 ), T( 0 ), T( 0 ) }, acc[ 3 ] = { T( 0 ), T( 0 ), T( 0 ) };
#pragma unroll
      for( int k = 0; k < 3; ++k ) { if( k < a.m ) { v[ k ] = a.g[ k ][ i ]; } }
#pragma unroll
      for( int c = 0; c < 6; ++c ) {
         if( c >= a.nc ) { continue; }
         T const qc = a.q[ c * a.n + i ];
         int const ci = a.pi[ c ], cj = a.pj[ c ];
#pragma unroll
         for( int k = 0; k < 3; ++k ) {
            if( ci == cj ) {
               if( k == ci ) { acc[ k ] = fma( qc * v[ k ], T( 2 ), acc[ k ] ); }
            } else if( k == ci ) {
               acc[ k ] = fma( qc * pick3( v, cj ), T( 1 ), acc[ k ] );
            } else if( k == cj ) {
               acc[ k ] = fma( qc * pick3( v, ci ), T( 1 ), acc[ k ] );
            }
         }
      }
#pragma unroll
      for( int k = 0; k < 3; ++k ) { if( k < a.m ) { a.gb[ k ][ i ] = acc[ k ]; } }
   }
}

template< typename Args, typename Kern >
cudaError_t launch_flat( Kern kern, Args const& a, int64_t n, cudaStream_t st ) {
   int64_t blocks = ( n + 255 ) / 256;
   if( blocks > 148 * 16 ) { blocks = 148 * 16; }
   if( blocks < 1 ) { blocks = 1; }
   kern<<< static_cast< unsigned >( blocks ), 256, 0, st >>>( a ); count_launch();
   return cudaGetLastError();
}

using Pairs = std::vector< std::pair< int, int >>;

template< typename T >
cudaError_t products( int64_t n, Pairs const& comps, std::vector< void* > const& g, void* dst, cudaStream_t st ) {
   ProdArgs< T > a{};
   for( size_t k = 0; k < g.size() && k < 3; ++k ) { a.g[ k ] = static_cast< T const* >( g[ k ] ); }
   a.dst = static_cast< T* >( dst );
   a.n = n;
   a.m = static_cast< int32_t >( g.size());
   a.nc = static_cast< int32_t >( comps.size());
   for( size_t c = 0; c < comps.size(); ++c ) { a.pi[ c ] = comps[ c ].first; a.pj[ c ] = comps[ c ].second; }
   return launch_flat( products_kernel< T >, a, n, st );
}

template< typename T >
cudaError_t gradient_adjoints( int64_t n, Pairs const& comps, void const* q_all, std::vector< void* > const& g,
                               std::vector< void* > const& gb, cudaStream_t st ) {
   GbarArgs< T > a{};
   a.q = static_cast< T const* >( q_all );
   for( size_t k = 0; k < g.size() && k < 3; ++k ) {
      a.g[ k ] = static_cast< T const* >( g[ k ] );
      a.gb[ k ] = static_cast< T* >( gb[ k ] );
   }
   a.n = n;
   a.m = static_cast< int32_t >( g.size());
   a.nc = static_cast< int32_t >( comps.size());
   for( size_t c = 0; c < comps.size(); ++c ) { a.pi[ c ] = comps[ c ].first; a.pj[ c ] = comps[ c ].second; }
   return launch_flat( gbar_kernel< T >, a, n, st );
}

struct Scratch {
   std::vector< void* > bufs;
   cudaStream_t st;
   ~Scratch() { for( void* p : bufs ) { cudaFreeAsync( p, st ); } }
   void* get( size_t bytes ) {
      void* p = nullptr;
      if( cudaMallocAsync( &p, bytes, st ) != cudaSuccess ) { return nullptr; }
      bufs.push_back( p );
      return p;
   }
};

// Common set-up of the forward and backward: gradient axes, component list, image geometry.
struct StSetup {
   int nd = 0;
   std::vector< int > dims;                 // axes of the gradient (size > 1, sigma > 0)
   std::vector< std::pair< int, int >> comps;
   int64_t n = 0;
   int32_t cdt = DT_SFLOAT;
   bool cdouble = false;
   dipcu_image_desc plain{};                // a normal-stride image of the compute type (data unset)
};

int st_setup( dipcu_image_desc const* in, double const* grad_sigmas, double const* tensor_sigmas, int32_t const* bcs,
              StSetup& s ) {
   if( !in || !in->data || in->ndims < 1 || in->ndims > 3 ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "structure tensor: the input must be a forged 1D-3D image" );
   }
   if( !grad_sigmas || !tensor_sigmas || !bcs ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "structure tensor: null parameter array" );
   }
   if( in->dtype <= DT_BIN || in->dtype > DT_DFLOAT ) {
      return record_error( DIPCU_ERR_UNSUPPORTED_DTYPE, "Data type not supported" );
   }
   s.nd = in->ndims;
   s.n = 1;
   for( int d = 0; d < s.nd; ++d ) {
      s.n *= in->sizes[ d ];
      if( in->sizes[ d ] > 1 && grad_sigmas[ d ] > 0.0 ) { s.dims.push_back( d ); }
   }
   if( s.dims.empty() ) { return record_error( DIPCU_ERR_INVALID_ARG, "Dimensionality not supported" ); }
   int const m = static_cast< int >( s.dims.size() );
   for( int i = 0; i < m; ++i ) { s.comps.push_back( { i, i } ); }
   for( int i = 0; i < m; ++i ) {
      for( int j = i + 1; j < m; ++j ) { s.comps.push_back( { i, j } ); }
   }
   s.cdt = suggest_flex( in->dtype );
   s.cdouble = s.cdt == DT_DFLOAT;
   s.plain.dtype = s.cdt;
   s.plain.ndims = s.nd;
   int64_t st = 1;
   for( int d = 0; d < s.nd; ++d ) {
      s.plain.sizes[ d ] = in->sizes[ d ];
      s.plain.strides[ d ] = st;
      st *= in->sizes[ d ];
   }
   return DIPCU_OK;
}

int check_tensor_image( dipcu_image_desc const* t, StSetup const& s, char const* name ) {
   if( !t || !t->data || t->ndims != s.nd + 1 || t->dtype != s.cdt ||
       t->sizes[ s.nd ] != static_cast< int64_t >( s.comps.size() )) {
      std::string msg = std::string( "structure tensor: `" ) + name + "` must have the input's sizes plus a last axis of " +
                        std::to_string( s.comps.size() ) + " components, of the computation type";
      return record_error( DIPCU_ERR_INVALID_ARG, msg.c_str() );
   }
   for( int d = 0; d < s.nd; ++d ) {
      if( t->sizes[ d ] != s.plain.sizes[ d ] ) { return record_error( DIPCU_ERR_SIZES_DONT_MATCH, "Sizes don't match" ); }
   }
   return DIPCU_OK;
}

dipcu_image_desc component( dipcu_image_desc const* t, int c, int nd ) {
   dipcu_image_desc d = *t;
   d.ndims = nd;
   d.data = static_cast< char* >( t->data ) + static_cast< int64_t >( c ) * t->strides[ nd ] * dtype_size( t->dtype );
   return d;
}

// g_k for every gradient axis, into `g[k]` (normal strides).
int gradients( dipcu_image_desc const* in, StSetup const& s, double const* grad_sigmas, int32_t const* bcs, double trunc,
               std::vector< void* > const& g, cudaStream_t stream ) {
   for( size_t k = 0; k < s.dims.size(); ++k ) {
      std::vector< uint32_t > ord( static_cast< size_t >( s.nd ), 0u );
      ord[ static_cast< size_t >( s.dims[ k ] ) ] = 1u;
      std::vector< AxisFilter > f;
      if( int st = build_filters( in, grad_sigmas, ord.data(), bcs, trunc, f, nullptr )) { return st; }
      dipcu_image_desc out = s.plain;
      out.data = g[ k ];
      if( int st = run_filters( in, &out, f, s.cdouble, stream )) { return st; }
   }
   return DIPCU_OK;
}

} // namespace

} // namespace dipcu

using namespace dipcu;

extern "C" {

int dipcu_structure_tensor( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* grad_sigmas,
                            double const* tensor_sigmas, int32_t const* bcs, double truncation, void* stream_ ) {
   cudaStream_t stream = static_cast< cudaStream_t >( stream_ );
   StSetup s;
   if( int st = st_setup( in, grad_sigmas, tensor_sigmas, bcs, s )) { return st; }
   if( int st = check_tensor_image( out, s, "out" )) { return st; }
   size_t const bytes = static_cast< size_t >( s.n ) * ( s.cdouble ? 8 : 4 );
   Scratch sc{ {}, stream };
   std::vector< void* > g;
   for( size_t k = 0; k < s.dims.size(); ++k ) {
      g.push_back( sc.get( bytes ));
      if( !g.back() ) { return record_error( DIPCU_ERR_CUDA, "cudaMallocAsync (gradient)" ); }
   }
   // All products at once, smoothed by one call with the components as an unfiltered batch axis
   // (one launch of the tile kernel instead of one per component); where that buffer does not
   // fit, one product at a time.
   size_t const nc = s.comps.size();
   void* prod_all = nc > 1 ? sc.get( bytes * nc ) : nullptr;
   if( !prod_all ) { cudaGetLastError(); }   // a failed allocation is not a launch error
   void* prod = prod_all ? nullptr : sc.get( bytes );
   if( !prod_all && !prod ) { return record_error( DIPCU_ERR_CUDA, "cudaMallocAsync (product)" ); }
   if( int st = gradients( in, s, grad_sigmas, bcs, truncation, g, stream )) { return st; }
   if( prod_all ) {
      cudaError_t const e = s.cdouble ? products< double >( s.n, s.comps, g, prod_all, stream )
                                      : products< float >( s.n, s.comps, g, prod_all, stream );
      if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
      dipcu_image_desc pall = s.plain;
      pall.ndims = s.nd + 1;
      pall.data = prod_all;
      pall.sizes[ s.nd ] = static_cast< int64_t >( nc );
      pall.strides[ s.nd ] = s.n;
      std::vector< double > sig( tensor_sigmas, tensor_sigmas + s.nd );
      sig.push_back( 0.0 );
      std::vector< uint32_t > ord0( static_cast< size_t >( s.nd + 1 ), 0u );
      std::vector< int32_t > bc( bcs, bcs + s.nd );
      bc.push_back( bcs[ 0 ] );
      std::vector< AxisFilter > f4;
      if( int st = build_filters( &pall, sig.data(), ord0.data(), bc.data(), truncation, f4, nullptr )) { return st; }
      return run_filters( &pall, out, f4, s.cdouble, stream );
   }
   std::vector< uint32_t > ord( static_cast< size_t >( s.nd ), 0u );
   dipcu_image_desc pimg = s.plain;
   pimg.data = prod;
   std::vector< AxisFilter > f;
   if( int st = build_filters( &pimg, tensor_sigmas, ord.data(), bcs, truncation, f, nullptr )) { return st; }
   for( size_t c = 0; c < s.comps.size(); ++c ) {
      cudaError_t e = elementwise( s.cdouble, prod, g[ static_cast< size_t >( s.comps[ c ].first ) ],
                                   g[ static_cast< size_t >( s.comps[ c ].second ) ], 1.0, s.n, 0, stream );
      if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
      dipcu_image_desc oc = component( out, static_cast< int >( c ), s.nd );
      if( int st = run_filters( &pimg, &oc, f, s.cdouble, stream )) { return st; }
   }
   return DIPCU_OK;
}

int dipcu_structure_tensor_backward( dipcu_image_desc const* grad_out, dipcu_image_desc const* in,
                                     dipcu_image_desc const* grad_in, double const* grad_sigmas,
                                     double const* tensor_sigmas, int32_t const* bcs, double truncation,
                                     void* stream_ ) {
   cudaStream_t stream = static_cast< cudaStream_t >( stream_ );
   StSetup s;
   if( int st = st_setup( in, grad_sigmas, tensor_sigmas, bcs, s )) { return st; }
   if( int st = check_tensor_image( grad_out, s, "grad_out" )) { return st; }
   if( !grad_in || grad_in->ndims != s.nd || grad_in->dtype != s.cdt ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "structure tensor: grad_in must be an image of the input's sizes and the computation type" );
   }
   size_t const bytes = static_cast< size_t >( s.n ) * ( s.cdouble ? 8 : 4 );
   Scratch sc{ {}, stream };
   size_t const m = s.dims.size();
   std::vector< void* > g, gb;
   for( size_t k = 0; k < m; ++k ) {
      g.push_back( sc.get( bytes ));
      gb.push_back( sc.get( bytes ));
      if( !g.back() || !gb.back() ) { return record_error( DIPCU_ERR_CUDA, "cudaMallocAsync (gradients)" ); }
      if( cudaMemsetAsync( gb.back(), 0, bytes, stream ) != cudaSuccess ) {
         return record_error( DIPCU_ERR_CUDA, "cudaMemsetAsync (gradients)" );
      }
   }
   void* q = sc.get( bytes );
   void* acc = sc.get( bytes );
   if( !q || !acc ) { return record_error( DIPCU_ERR_CUDA, "cudaMallocAsync (backward)" ); }
   // Recompute the gradient images.
   if( int st = gradients( in, s, grad_sigmas, bcs, truncation, g, stream )) { return st; }
   std::vector< uint32_t > zero( static_cast< size_t >( s.nd ), 0u );
   dipcu_image_desc qimg = s.plain;
   qimg.data = q;
   // Q_c of all components by one adjoint call over the component axis (unfiltered batch axis)
   // where the scratch fits, else per component.
   size_t const nc = s.comps.size();
   void* q_all = nc > 1 ? sc.get( bytes * nc ) : nullptr;
   if( !q_all ) { cudaGetLastError(); }   // a failed allocation is not a launch error
   if( q_all ) {
      dipcu_image_desc qa = s.plain;
      qa.ndims = s.nd + 1;
      qa.data = q_all;
      qa.sizes[ s.nd ] = static_cast< int64_t >( nc );
      qa.strides[ s.nd ] = s.n;
      std::vector< double > sig( tensor_sigmas, tensor_sigmas + s.nd );
      sig.push_back( 0.0 );
      std::vector< uint32_t > zero4( static_cast< size_t >( s.nd + 1 ), 0u );
      std::vector< int32_t > bc( bcs, bcs + s.nd );
      bc.push_back( bcs[ 0 ] );
      if( int st = dipcu_gauss_fir_backward( grad_out, nullptr, &qa, nullptr, sig.data(), zero4.data(), bc.data(), truncation,
                                             stream )) {
         return st;
      }
   }
   if( q_all ) {   // all components' adjoints at hand: one pass over the images
      cudaError_t const e = s.cdouble ? gradient_adjoints< double >( s.n, s.comps, q_all, g, gb, stream )
                                      : gradient_adjoints< float >( s.n, s.comps, q_all, g, gb, stream );
      if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
   }
   for( size_t c = 0; c < nc && !q_all; ++c ) {
      void* qc = q;
      {
         dipcu_image_desc wc = component( grad_out, static_cast< int >( c ), s.nd );
         if( int st = dipcu_gauss_fir_backward( &wc, nullptr, &qimg, nullptr, tensor_sigmas, zero.data(), bcs, truncation,
                                                stream )) {
            return st;
         }
      }
      size_t const i = static_cast< size_t >( s.comps[ c ].first ), j = static_cast< size_t >( s.comps[ c ].second );
      cudaError_t e;
      if( i == j ) {
         e = elementwise( s.cdouble, gb[ i ], qc, g[ i ], 2.0, s.n, 1, stream );
      } else {
         e = elementwise( s.cdouble, gb[ i ], qc, g[ j ], 1.0, s.n, 1, stream );
         if( e == cudaSuccess ) { e = elementwise( s.cdouble, gb[ j ], qc, g[ i ], 1.0, s.n, 1, stream ); }
      }
      if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
   }
   // in_bar = sum_k D_k^T g_bar_k, accumulated in `acc`, then converted into grad_in.
   dipcu_image_desc aimg = s.plain;
   aimg.data = acc;
   for( size_t k = 0; k < m; ++k ) {
      std::vector< uint32_t > ord( static_cast< size_t >( s.nd ), 0u );
      ord[ static_cast< size_t >( s.dims[ k ] ) ] = 1u;
      dipcu_image_desc gk = s.plain;
      gk.data = gb[ k ];
      dipcu_image_desc target = aimg;
      if( k > 0 ) { target.data = q; }
      if( int st = dipcu_gauss_fir_backward( &gk, nullptr, &target, nullptr, grad_sigmas, ord.data(), bcs, truncation,
                                             stream )) {
         return st;
      }
      if( k > 0 ) {
         cudaError_t e = elementwise( s.cdouble, acc, q, nullptr, 1.0, s.n, 2, stream );
         if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
      }
   }
   ConvertArgs cv{};
   cv.src = acc;
   cv.dst = grad_in->data;
   cv.src_dt = s.cdt;
   cv.dst_dt = grad_in->dtype;
   cv.ndims = s.nd;
   cv.total = s.n;
   for( int d = 0; d < s.nd; ++d ) {
      cv.sizes[ d ] = s.plain.sizes[ d ];
      cv.sst[ d ] = s.plain.strides[ d ];
      cv.dstst[ d ] = grad_in->strides[ d ];
   }
   cudaError_t e = launch_convert( cv, true, stream );
   if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
   return DIPCU_OK;
}

} // extern "C"
