// Test program, not product code: the device branch of dip::GaussFIR that INTEGRATION.md gives a
// DIPlib maintainer, compiled against DIPlib's own headers and linked with the DIPlib build of
// oracle/_ref (libdipref.so) and libdipcu.so.  Images are forged in device memory through a
// dip::ExternalInterface that allocates with cudaMalloc (include/diplib/library/image.h:97-135 in
// DIPlib); the branch runs on them and its results, copied back, are compared with the host
// dip::GaussFIR (src/linear/gauss.cpp:238-286) on the same inputs.  Exit status 0: every case
// within 1e-5 of the input range (float outputs) or 1 (integer outputs), and the reference's
// errors thrown for bad arguments.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "diplib.h"
#include "diplib/boundary.h"
#include "diplib/iterators.h"
#include "diplib/linear.h"
#include "dipcu.h"

namespace dropin {

using namespace dip;

// ---- the device branch, as INTEGRATION.md quotes it ---------------------------------------------

// Images whose data live in device memory: forged through this interface.
class CudaInterface : public dip::ExternalInterface {
   public:
      dip::DataSegment AllocateData( void*& origin, dip::DataType dataType, dip::UnsignedArray const& sizes,
                                     dip::IntegerArray& strides, dip::Tensor const& tensor, dip::sint& tensorStride ) override {
         dip::uint n = tensor.Elements();
         strides.resize( sizes.size() );
         dip::sint s = static_cast< dip::sint >( n );
         for( dip::uint ii = 0; ii < sizes.size(); ++ii ) {
            strides[ ii ] = s;
            s *= static_cast< dip::sint >( sizes[ ii ] );
         }
         tensorStride = 1;
         void* p = nullptr;
         if( cudaMalloc( &p, static_cast< size_t >( s ) * dataType.SizeOf() ) != cudaSuccess ) {
            DIP_THROW( "cudaMalloc failed" );
         }
         origin = p;
         return dip::DataSegment( p, []( void* q ) { cudaFree( q ); } );
      }
      dip::String Name() const override { return "CUDA device memory"; }
};

CudaInterface& DeviceInterface() {
   static CudaInterface ci;
   return ci;
}

bool IsDeviceImage( Image const& img ) {
   return img.ExternalInterface() == &DeviceInterface();
}

void* CurrentStream() {
   return nullptr;   // the legacy default stream; a DIPlib build with streams passes its own
}

int32_t DipTypeToDipcu( DataType dt ) {
   switch( dt.dt ) {
      case DataType::DT::BIN: return DIPCU_BIN;
      case DataType::DT::UINT8: return DIPCU_UINT8;
      case DataType::DT::UINT16: return DIPCU_UINT16;
      case DataType::DT::UINT32: return DIPCU_UINT32;
      case DataType::DT::UINT64: return DIPCU_UINT64;
      case DataType::DT::SINT8: return DIPCU_SINT8;
      case DataType::DT::SINT16: return DIPCU_SINT16;
      case DataType::DT::SINT32: return DIPCU_SINT32;
      case DataType::DT::SINT64: return DIPCU_SINT64;
      case DataType::DT::SFLOAT: return DIPCU_SFLOAT;
      case DataType::DT::DFLOAT: return DIPCU_DFLOAT;
      default: DIP_THROW( E::DATA_TYPE_NOT_SUPPORTED );
   }
}

dipcu_image_desc ToDesc( Image const& img ) {
   dipcu_image_desc d{};
   d.data = img.Origin();
   d.dtype = DipTypeToDipcu( img.DataType() );
   d.ndims = static_cast< int32_t >( img.Dimensionality() );
   for( dip::uint ii = 0; ii < img.Dimensionality(); ++ii ) {
      d.sizes[ ii ] = static_cast< int64_t >( img.Size( ii ));
      d.strides[ ii ] = img.Stride( ii );
   }
   return d;
}

void GaussFIR( Image const& in, Image& out, FloatArray sigmas, UnsignedArray order,
               StringArray const& boundaryCondition, dfloat truncation ) {
   DIP_THROW_IF( !in.IsForged(), E::IMAGE_NOT_FORGED );
   if( IsDeviceImage( in )) {
      dip::uint nDims = in.Dimensionality();
      DIP_STACK_TRACE_THIS( ArrayUseParameter( sigmas, nDims, 1.0 ));
      DIP_STACK_TRACE_THIS( ArrayUseParameter( order, nDims, dip::uint( 0 )));
      BoundaryConditionArray bc;
      DIP_STACK_TRACE_THIS( bc = StringArrayToBoundaryConditionArray( boundaryCondition ));
      DIP_STACK_TRACE_THIS( BoundaryArrayUseParameter( bc, nDims ));
      ExternalInterface* ei = in.ExternalInterface();
      Image ins = in.QuickCopy();               // keeps the input data when `out` is `in` (in-place call)
      if( out.Aliases( ins )) { out.Strip(); }  // the device kernels do not filter in place
      if( !out.IsForged() && !out.HasExternalInterface() ) { out.SetExternalInterface( ei ); }
      out.ReForge( ins.Sizes(), ins.TensorElements(), DataType::SuggestFlex( ins.DataType() ),
                   Option::AcceptDataTypeChange::DO_ALLOW );
      Image outs = out.QuickCopy();
      if( !ins.IsScalar() ) { ins.TensorToSpatial(); outs.TensorToSpatial(); }   // as AsScalarImage
      dipcu_image_desc di = ToDesc( ins );
      dipcu_image_desc dout = ToDesc( outs );
      std::vector< double > s( sigmas.begin(), sigmas.end() );
      std::vector< uint32_t > o( order.begin(), order.end() );
      std::vector< int32_t > b;
      for( auto c : bc ) { b.push_back( static_cast< int32_t >( c )); }
      if( !ins.IsScalar() ) { s.push_back( 0 ); o.push_back( 0 ); b.push_back( 0 ); }   // the tensor axis
      int st = dipcu_gauss_fir( &di, &dout, s.data(), o.data(), b.data(), truncation, CurrentStream() );
      if( st == DIPCU_ERR_ORDER_GT_3 ) { DIP_THROW( "Gaussian FIR filter not implemented for order > 3" ); }
      DIP_THROW_IF( st != DIPCU_OK, dipcu_last_error_message() );
      return;
   }
   dip::GaussFIR( in, out, sigmas, order, boundaryCondition, truncation );   // the existing host implementation
}

// ---- end of the device branch -----------------------------------------------------------------

} // namespace dropin

namespace {

using dip::Image;

// Host image -> device image (same sizes, type, tensor) and back, through normal strides.
Image ToDevice( Image const& host ) {
   Image dev;
   dev.SetExternalInterface( &dropin::DeviceInterface() );
   dev.ReForge( host.Sizes(), host.TensorElements(), host.DataType() );
   Image h = host.Copy();                     // normal strides, tensor stride 1 (same layout as the interface's)
   if( cudaMemcpy( dev.Origin(), h.Origin(), h.NumberOfPixels() * h.TensorElements() * h.DataType().SizeOf(),
                   cudaMemcpyHostToDevice ) != cudaSuccess ) {
      DIP_THROW( "cudaMemcpy to device failed" );
   }
   return dev;
}

Image ToHost( Image const& dev ) {
   Image host( dev.Sizes(), dev.TensorElements(), dev.DataType() );
   // `dev` has normal strides and tensor stride 1 (forged by the interface); so has a fresh host image.
   if( host.Stride( 0 ) != dev.Stride( 0 ) || host.TensorStride() != dev.TensorStride() ) { DIP_THROW( "layouts differ" ); }
   if( cudaMemcpy( host.Origin(), dev.Origin(), host.NumberOfPixels() * host.TensorElements() * host.DataType().SizeOf(),
                   cudaMemcpyDeviceToHost ) != cudaSuccess ) {
      DIP_THROW( "cudaMemcpy to host failed" );
   }
   return host;
}

Image Random( dip::UnsignedArray const& sizes, dip::uint tensor, dip::DataType dt, unsigned seed ) {
   Image img( sizes, tensor, dip::DT_DFLOAT );
   std::mt19937 gen( seed );
   std::uniform_real_distribution< double > u( 0.0, 1.0 );
   double const scale = dt.IsFloat() ? 1.0 : ( dt == dip::DT_UINT8 ? 255.0 : 4095.0 );
   dip::ImageIterator< dip::dfloat > it( img );
   do {
      for( auto& v : it ) { v = dt.IsFloat() ? u( gen ) : std::floor( u( gen ) * scale ); }
   } while( ++it );
   img.Convert( dt );
   return img;
}

// Largest |a - b| and the range of `a` over all samples (both converted to dfloat).
double MaxAbsDiff( Image const& a, Image const& b ) {
   Image da = dip::Convert( a, dip::DT_DFLOAT );
   Image db = dip::Convert( b, dip::DT_DFLOAT );
   dip::ImageIterator< dip::dfloat > ia( da ), ib( db );
   double m = 0.0;
   do {
      auto ta = ia.begin();
      auto tb = ib.begin();
      for( ; ta != ia.end(); ++ta, ++tb ) { m = std::max( m, std::abs( *ta - *tb )); }
   } while( ++ia, ++ib );
   return m;
}

double Range( Image const& a ) {
   Image da = dip::Convert( a, dip::DT_DFLOAT );
   dip::ImageIterator< dip::dfloat > it( da );
   double lo = 1e300, hi = -1e300;
   do {
      for( auto v : it ) { lo = std::min( lo, v ); hi = std::max( hi, v ); }
   } while( ++it );
   return hi - lo;
}

struct Case {
   char const* name;
   dip::UnsignedArray sizes;
   dip::uint tensor;
   dip::DataType dt;
   dip::FloatArray sigmas;
   dip::UnsignedArray order;
   dip::StringArray bc;
   dip::DataType protect_out;   // DT_BIN here: no protected output
   bool in_place;
};

bool Run( Case const& c ) {
   Image hin = Random( c.sizes, c.tensor, c.dt, 7 );
   Image ref;
   if( c.protect_out != dip::DT_BIN ) {
      ref.ReForge( c.sizes, c.tensor, c.protect_out );
      ref.Protect();
   }
   dip::GaussFIR( hin, ref, c.sigmas, c.order, c.bc, 3.0 );
   Image din = ToDevice( hin );
   Image dout;
   dout.SetExternalInterface( &dropin::DeviceInterface() );
   if( c.protect_out != dip::DT_BIN ) {
      dout.ReForge( c.sizes, c.tensor, c.protect_out );
      dout.Protect();
   }
   if( c.in_place ) {
      dropin::GaussFIR( din, din, c.sigmas, c.order, c.bc, 3.0 );   // one image as input and output
      dout = din;
   } else {
      dropin::GaussFIR( din, dout, c.sigmas, c.order, c.bc, 3.0 );
   }
   if( cudaDeviceSynchronize() != cudaSuccess ) { std::printf( "%s: CUDA error\n", c.name ); return false; }
   Image got = ToHost( dout );
   bool ok = got.DataType() == ref.DataType() && got.Sizes() == ref.Sizes() && got.TensorElements() == ref.TensorElements();
   double const err = ok ? MaxAbsDiff( got, ref ) : 1e30;
   double const range = Range( hin );
   double const tol = ref.DataType().IsFloat() ? 1e-5 * std::max( range, 1.0 ) : 1.0;
   ok = ok && err <= tol;
   std::printf( "%-40s out %-6s max abs err %.3e (tol %.3e) %s\n", c.name, ref.DataType().Name(), err, tol, ok ? "ok" : "FAIL" );
   return ok;
}

} // namespace

int main() {
   int devices = 0;
   if( cudaGetDeviceCount( &devices ) != cudaSuccess || devices < 1 ) {
      std::printf( "no CUDA device\n" );
      return 2;
   }
   bool ok = true;
   try {
      std::vector< Case > cases = {
         { "2D sfloat sigma (2,3) order (1,0) mirror", { 200, 150 }, 1, dip::DT_SFLOAT, { 2.0, 3.0 }, { 1, 0 }, {}, dip::DT_BIN, false },
         { "3D uint16 sigma (1.5,1.5,3) order (0,0,0)", { 64, 48, 40 }, 1, dip::DT_UINT16, { 1.5, 1.5, 3.0 }, { 0 }, { "mirror" }, dip::DT_BIN, false },
         { "3D uint16 sigma (1.5,1.5,3) order (1,0,0)", { 64, 48, 40 }, 1, dip::DT_UINT16, { 1.5, 1.5, 3.0 }, { 1, 0, 0 }, { "mirror" }, dip::DT_BIN, false },
         { "2D sfloat periodic / add zeros", { 131, 77 }, 1, dip::DT_SFLOAT, { 4.0 }, { 2, 1 }, { "periodic", "add zeros" }, dip::DT_BIN, false },
         { "2D uint8 -> sfloat, third order", { 90, 61 }, 1, dip::DT_UINT8, { 1.3, 2.2 }, { 2, 1 }, { "third order" }, dip::DT_BIN, false },
         { "2D sint32 -> dfloat", { 70, 50 }, 1, dip::DT_SINT32, { 2.0 }, { 0 }, {}, dip::DT_BIN, false },
         { "2D 3-channel sfloat (tensor axis)", { 80, 60 }, 3, dip::DT_SFLOAT, { 1.5 }, { 0 }, { "mirror" }, dip::DT_BIN, false },
         { "2D sfloat, protected uint16 output", { 100, 70 }, 1, dip::DT_SFLOAT, { 2.0 }, { 0 }, {}, dip::DT_UINT16, false },
         { "2D sfloat in place (stripped output)", { 120, 90 }, 1, dip::DT_SFLOAT, { 2.5 }, { 0, 2 }, { "zero order" }, dip::DT_BIN, true },
         { "1D dfloat sigma 8", { 500 }, 1, dip::DT_DFLOAT, { 8.0 }, { 3 }, { "asym mirror" }, dip::DT_BIN, false },
      };
      for( auto const& c : cases ) { ok = Run( c ) && ok; }
      // The reference's errors: order > 3, an unknown boundary condition, a wrong array length.
      Image din = ToDevice( Random( { 20, 20 }, 1, dip::DT_SFLOAT, 3 ));
      struct Bad { char const* name; dip::UnsignedArray order; dip::StringArray bc; dip::FloatArray sigmas; char const* msg; };
      std::vector< Bad > bad = {
         { "order 4", { 4 }, {}, { 1.0 }, "Gaussian FIR filter not implemented for order > 3" },
         { "unknown boundary condition", { 0 }, { "sideways" }, { 1.0 }, "Boundary condition not recognized" },
         { "three sigmas for a 2D image", { 0 }, {}, { 1.0, 1.0, 1.0 }, "Array parameter has the wrong number of elements" },
      };
      for( auto const& b : bad ) {
         bool thrown = false;
         std::string what;
         try {
            Image dout;
            dropin::GaussFIR( din, dout, b.sigmas, b.order, b.bc, 3.0 );
         } catch( dip::Error const& e ) {
            thrown = true;
            what = e.what();
         }
         bool const good = thrown && what.find( b.msg ) != std::string::npos;
         std::printf( "%-40s %s\n", b.name, good ? "throws the reference's error: ok" : ( "FAIL: " + what ).c_str() );
         ok = ok && good;
      }
   } catch( dip::Error const& e ) {
      std::printf( "DIPlib error: %s\n", e.what() );
      ok = false;
   }
   std::printf( "%s\n", ok ? "ALL OK" : "FAILED" );
   return ok ? 0 : 1;
}
