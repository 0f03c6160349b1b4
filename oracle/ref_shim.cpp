// Test infrastructure only (linked into oracle/_ref/libdipref.so, never into the product).
//
// A thin extern "C" layer over the unmodified DIPlib sources so that Python tests and the bench's
// CPU leg can call the reference's own Gaussian FIR path on raw host buffers:
//   dip::Gauss               src/linear/derivative.cpp:62-86
//   dip::StructureTensor     src/analysis/structure_tensor.cpp:33-59
//   dip::Gradient, GradientMagnitude, Hessian, Laplace  src/linear/derivative.cpp:142-418
//   dip::MakeHalfGaussian    src/linear/gauss.cpp:151-165
//   dip::detail::ExpandBuffer src/library/copy_buffer.cpp:751-813
//   dip::ReadPixelWithBoundaryCondition src/library/boundary.cpp:47-128
//   dip::SeparableConvolution src/linear/convolution.cpp:319-421, dip::Uniform src/linear/uniform.cpp:147-163
//   dip::GaussIIR            src/linear/gaussiir.cpp:725-790
//
// Sizes and strides are given in DIPlib order (x first), in samples.  Data type codes are the
// ones of include/dipcu.h (DIPCU_BIN .. DIPCU_DFLOAT).  Every entry point returns 0 on success
// and 1 on a dip::Error, whose message is copied into `err`.

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "diplib.h"
#include "diplib/analysis.h"
#include "diplib/boundary.h"
#include "diplib/generation.h"
#include "diplib/kernel.h"
#include "diplib/library/copy_buffer.h"
#include "diplib/linear.h"
#include "diplib/transform.h"
#include "diplib/multithreading.h"

namespace {

dip::DataType CodeToType( int code ) {
   switch( code ) {
      case 0: return dip::DT_BIN;
      case 1: return dip::DT_UINT8;
      case 2: return dip::DT_UINT16;
      case 3: return dip::DT_UINT32;
      case 4: return dip::DT_UINT64;
      case 5: return dip::DT_SINT8;
      case 6: return dip::DT_SINT16;
      case 7: return dip::DT_SINT32;
      case 8: return dip::DT_SINT64;
      case 9: return dip::DT_SFLOAT;
      case 10: return dip::DT_DFLOAT;
      default: DIP_THROW( "bad dtype code" );
   }
}

int TypeToCode( dip::DataType dt ) {
   for( int c = 0; c <= 10; ++c ) {
      if( CodeToType( c ) == dt ) { return c; }
   }
   return -1;
}

void SetErr( char* err, int errlen, std::string const& msg ) {
   if( err && errlen > 0 ) {
      std::strncpy( err, msg.c_str(), static_cast< std::size_t >( errlen - 1 ));
      err[ errlen - 1 ] = 0;
   }
}

dip::StringArray SplitList( char const* s, bool present ) {
   dip::StringArray out;
   if( !present ) { return out; }
   std::string str( s ? s : "" );
   std::size_t start = 0;
   while( true ) {
      std::size_t pos = str.find( '\n', start );
      out.push_back( str.substr( start, pos == std::string::npos ? std::string::npos : pos - start ));
      if( pos == std::string::npos ) { break; }
      start = pos + 1;
   }
   return out;
}

dip::Image Wrap( void const* data, int dtype, int ndims, int64_t const* sizes, int64_t const* strides ) {
   dip::UnsignedArray sz( static_cast< dip::uint >( ndims ));
   dip::IntegerArray st;
   for( int ii = 0; ii < ndims; ++ii ) { sz[ ii ] = static_cast< dip::uint >( sizes[ ii ] ); }
   if( strides ) {
      st.resize( static_cast< dip::uint >( ndims ));
      for( int ii = 0; ii < ndims; ++ii ) { st[ ii ] = strides[ ii ]; }
   }
   void* p = const_cast< void* >( data );
   return dip::Image( dip::NonOwnedRefToDataSegment( p ), p, CodeToType( dtype ), sz, st );
}

void CopyOut( dip::Image const& img, void* out ) {
   // Normal strides (contiguous, x fastest, tensor interleaved); a result with other strides (e.g. a
   // cropped view) is copied into such an image first.
   if( !img.HasNormalStrides() ) {
      dip::Image tmp;
      tmp.ReForge( img.Sizes(), img.TensorElements(), img.DataType() );
      DIP_THROW_IF( !tmp.HasNormalStrides(), "unexpected strides" );
      tmp.Copy( img );
      std::memcpy( out, tmp.Origin(), tmp.NumberOfSamples() * tmp.DataType().SizeOf() );
      return;
   }
   std::memcpy( out, img.Origin(), img.NumberOfSamples() * img.DataType().SizeOf() );
}

} // namespace

extern "C" {

// dip::SeparableConvolution with real filters: `nfilters` filters, filter i = lens[i] values of
// `data[i]`, origin origins[i], symmetry string syms (newline-separated); `bcs` as in dipref_gauss;
// `process` (nullptr: all axes).  The output (the reference's own, normal strides) goes to `out`;
// its type to *out_dtype.
int dipref_separable_convolution(
      void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* strides, int nfilters,
      double const* const* data, int const* lens, long const* origins, char const* syms,
      char const* bcs, int has_bcs, int const* process, void* out, int* out_dtype, char* err, int errlen ) {
   try {
      dip::Image img = Wrap( in, in_dtype, ndims, sizes, strides );
      dip::StringArray sy = SplitList( syms, true );
      dip::OneDimensionalFilterArray fa( static_cast< dip::uint >( nfilters ));
      for( int ii = 0; ii < nfilters; ++ii ) {
         fa[ ii ].filter.assign( data[ ii ], data[ ii ] + lens[ ii ] );
         fa[ ii ].origin = origins[ ii ];
         fa[ ii ].symmetry = sy[ static_cast< dip::uint >( ii ) ];
      }
      dip::BooleanArray pr;
      if( process ) {
         pr.resize( static_cast< dip::uint >( ndims ));
         for( int ii = 0; ii < ndims; ++ii ) { pr[ ii ] = process[ ii ] != 0; }
      }
      dip::Image res;
      dip::SeparableConvolution( img, res, fa, SplitList( bcs, has_bcs != 0 ), pr );
      *out_dtype = TypeToCode( res.DataType() );
      CopyOut( res, out );
      return 0;
   } catch( dip::Error const& e ) {
      SetErr( err, errlen, e.what() );
      return 1;
   }
}

// dip::Uniform with a rectangular kernel of per-axis sizes `fsizes` (ndims values).
int dipref_uniform(
      void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* strides, double const* fsizes,
      char const* bcs, int has_bcs, void* out, int* out_dtype, char* err, int errlen ) {
   try {
      dip::Image img = Wrap( in, in_dtype, ndims, sizes, strides );
      dip::FloatArray fs( static_cast< dip::uint >( ndims ));
      for( int ii = 0; ii < ndims; ++ii ) { fs[ ii ] = fsizes[ ii ]; }
      dip::Image res;
      dip::Uniform( img, res, dip::Kernel( fs, dip::S::RECTANGULAR ), SplitList( bcs, has_bcs != 0 ));
      *out_dtype = TypeToCode( res.DataType() );
      CopyOut( res, out );
      return 0;
   } catch( dip::Error const& e ) {
      SetErr( err, errlen, e.what() );
      return 1;
   }
}

// dip::FourierTransform of a real sfloat image into an scomplex one (interleaved re, im; normal
// strides), options newline-separated ("" for the forward transform).
int dipref_fourier_transform( float const* in, int ndims, int64_t const* sizes, char const* options, float* out,
                              char* err, int errlen ) {
   try {
      dip::Image img = Wrap( in, 9, ndims, sizes, nullptr );
      dip::StringArray opts = SplitList( options, options && options[ 0 ] );
      dip::StringSet os( opts.begin(), opts.end() );
      dip::Image res;
      dip::FourierTransform( img, res, os );
      res.Convert( dip::DT_SCOMPLEX );
      CopyOut( res, out );
      return 0;
   } catch( dip::Error const& e ) {
      SetErr( err, errlen, e.what() );
      return 1;
   }
}

int dipref_set_threads( int n ) {
   dip::SetNumberOfThreads( static_cast< dip::uint >( n < 0 ? 0 : n ));
   return static_cast< int >( dip::GetNumberOfThreads() );
}

// out_dtype: in/out.  If `protect_out` is 0, the reference allocates its own output (whose type
// is returned in *out_dtype) and the samples are copied into `out` with normal strides.  If
// `protect_out` is 1, `out` is wrapped as a protected image of type *out_dtype with normal
// strides, and the reference writes into it directly (its protected-output path).
int dipref_gauss(
      void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* strides,
      double const* sigmas, int nsigmas, uint32_t const* orders, int norders,
      char const* bcs, int has_bcs, double truncation, char const* method,
      void* out, int* out_dtype, int protect_out, char* err, int errlen ) {
   try {
      dip::Image img = Wrap( in, in_dtype, ndims, sizes, strides );
      dip::FloatArray s( static_cast< dip::uint >( nsigmas ));
      for( int ii = 0; ii < nsigmas; ++ii ) { s[ ii ] = sigmas[ ii ]; }
      dip::UnsignedArray o( static_cast< dip::uint >( norders ));
      for( int ii = 0; ii < norders; ++ii ) { o[ ii ] = orders[ ii ]; }
      dip::StringArray bc = SplitList( bcs, has_bcs != 0 );
      if( protect_out ) {
         dip::Image res = Wrap( out, *out_dtype, ndims, sizes, nullptr );
         res.Protect();
         dip::Gauss( img, res, s, o, method, bc, truncation );
      } else {
         dip::Image res;
         dip::Gauss( img, res, s, o, method, bc, truncation );
         *out_dtype = TypeToCode( res.DataType() );
         CopyOut( res, out );
      }
      return 0;
   } catch( dip::Error const& e ) {
      SetErr( err, errlen, e.what() );
      return 1;
   }
}

// dip::GaussIIR: per-axis sigmas / orders (nsigmas / norders values, broadcast by the reference),
// `forders` (nforders values, 0: the reference's defaults), `design` the design-method string.
// The output (the reference's own, normal strides) goes to `out`, its type to *out_dtype.
int dipref_gauss_iir(
      void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* strides,
      double const* sigmas, int nsigmas, uint32_t const* orders, int norders, char const* bcs, int has_bcs,
      uint32_t const* forders, int nforders, char const* design, double truncation,
      void* out, int* out_dtype, char* err, int errlen ) {
   try {
      dip::Image img = Wrap( in, in_dtype, ndims, sizes, strides );
      dip::FloatArray s( static_cast< dip::uint >( nsigmas ));
      for( int ii = 0; ii < nsigmas; ++ii ) { s[ ii ] = sigmas[ ii ]; }
      dip::UnsignedArray o( static_cast< dip::uint >( norders ));
      for( int ii = 0; ii < norders; ++ii ) { o[ ii ] = orders[ ii ]; }
      dip::UnsignedArray fo( static_cast< dip::uint >( nforders ));
      for( int ii = 0; ii < nforders; ++ii ) { fo[ ii ] = forders[ ii ]; }
      dip::Image res;
      dip::GaussIIR( img, res, s, o, SplitList( bcs, has_bcs != 0 ), fo, design, truncation );
      *out_dtype = TypeToCode( res.DataType() );
      CopyOut( res, out );
      return 0;
   } catch( dip::Error const& e ) {
      SetErr( err, errlen, e.what() );
      return 1;
   }
}

// Output: the tensor components per pixel, interleaved (normal strides), in the reference's
// symmetric-matrix order (diagonal first); `out` has room for ndims*(ndims+1)/2 of them.  Returns the
// output data type in *out_dtype and the number of components in *ncomp.
int dipref_structure_tensor(
      void const* in, int in_dtype, int ndims, int64_t const* sizes,
      double grad_sigma, double tensor_sigma, char const* method, char const* bc, double truncation,
      void* out, int* out_dtype, int* ncomp, char* err, int errlen ) {
   try {
      dip::Image img = Wrap( in, in_dtype, ndims, sizes, nullptr );
      dip::Image res;
      dip::StructureTensor( img, {}, res, { grad_sigma }, { tensor_sigma }, method, { bc }, truncation );
      *out_dtype = TypeToCode( res.DataType() );
      *ncomp = static_cast< int >( res.TensorElements() );
      if( *ncomp > ndims * ( ndims + 1 ) / 2 ) { return 1; }
      CopyOut( res, out );
      return 0;
   } catch( dip::Error const& e ) {
      SetErr( err, errlen, e.what() );
      return 1;
   }
}

// which: 0 dip::Gradient, 1 dip::GradientMagnitude, 2 dip::Hessian, 3 dip::Laplace, with the
// given method; `bcs` as in dipref_gauss.  Output: the tensor components per pixel, interleaved
// (normal strides), at most `maxcomp` of them; the data type in *out_dtype, the count in *ncomp.
int dipref_derivative_op(
      int which, void const* in, int in_dtype, int ndims, int64_t const* sizes,
      double const* sigmas, int nsigmas, char const* bcs, int has_bcs, double truncation, char const* method,
      void* out, int maxcomp, int* out_dtype, int* ncomp, char* err, int errlen ) {
   try {
      dip::Image img = Wrap( in, in_dtype, ndims, sizes, nullptr );
      dip::FloatArray s( static_cast< dip::uint >( nsigmas ));
      for( int ii = 0; ii < nsigmas; ++ii ) { s[ ii ] = sigmas[ ii ]; }
      dip::StringArray bc = SplitList( bcs, has_bcs != 0 );
      dip::Image res;
      switch( which ) {
         case 0: dip::Gradient( img, res, s, method, bc, {}, truncation ); break;
         case 1: dip::GradientMagnitude( img, res, s, method, bc, {}, truncation ); break;
         case 2: dip::Hessian( img, res, s, method, bc, {}, truncation ); break;
         default: dip::Laplace( img, res, s, method, bc, {}, truncation ); break;
      }
      *out_dtype = TypeToCode( res.DataType() );
      *ncomp = static_cast< int >( res.TensorElements() );
      if( *ncomp > maxcomp ) { return 1; }
      CopyOut( res, out );
      return 0;
   } catch( dip::Error const& e ) {
      SetErr( err, errlen, e.what() );
      return 1;
   }
}

int dipref_half_gaussian( double sigma, uint32_t order, double truncation, int dt_double, double* out, int cap ) {
   try {
      std::vector< dip::dfloat > h = dip::MakeHalfGaussian( sigma, order, truncation, dt_double ? dip::DT_DFLOAT : dip::DT_SFLOAT );
      int n = static_cast< int >( h.size() );
      for( int ii = 0; ii < n && ii < cap; ++ii ) { out[ ii ] = h[ static_cast< dip::uint >( ii ) ]; }
      return n;
   } catch( dip::Error const& ) {
      return -1;
   }
}

// `buffer` points at the first of `pixels` samples; `left` samples before it and `right` after
// it are written.  `bc` is a dip::BoundaryCondition enumerator value.
int dipref_expand_buffer( void* buffer, int dtype, int64_t stride, uint64_t pixels, uint64_t left, uint64_t right, int bc ) {
   try {
      dip::detail::ExpandBuffer( buffer, CodeToType( dtype ), stride, 1, pixels, 1, left, right,
                                 static_cast< dip::BoundaryCondition >( bc ));
      return 0;
   } catch( dip::Error const& ) {
      return 1;
   }
}

int dipref_string_to_bc( char const* s ) {
   try {
      return static_cast< int >( dip::StringToBoundaryCondition( s ));
   } catch( dip::Error const& ) {
      return -1;
   }
}

double dipref_max_gauss_truncation( int dt_double ) {
   return dt_double ? dip::maximum_gauss_truncation< dip::dfloat >() : dip::maximum_gauss_truncation< dip::sfloat >();
}

// Reads one sample of a scalar sfloat image at `coords` (which may lie outside the image).
int dipref_read_pixel_bc( float const* img, int ndims, int64_t const* sizes, int64_t const* coords, int const* bcs, float* out ) {
   try {
      dip::Image im = Wrap( img, 9, ndims, sizes, nullptr );
      dip::IntegerArray c( static_cast< dip::uint >( ndims ));
      dip::BoundaryConditionArray b( static_cast< dip::uint >( ndims ));
      for( int ii = 0; ii < ndims; ++ii ) {
         c[ ii ] = coords[ ii ];
         b[ ii ] = static_cast< dip::BoundaryCondition >( bcs[ ii ] );
      }
      *out = dip::ReadPixelWithBoundaryCondition( im, c, b ).As< float >();
      return 0;
   } catch( dip::Error const& ) {
      return 1;
   }
}

} // extern "C"
