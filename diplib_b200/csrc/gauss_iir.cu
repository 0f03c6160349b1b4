// dip::GaussIIR (src/linear/gaussiir.cpp:725-790 in DIPlib) on the device: the recursive
// Gaussian (derivative) filter of van Vliet, Young and Verbeek, pass by pass along each axis.
//
// Design (host, FP64): the poles of the chosen recursion order and design method (the tables of
// FillPoleCoefficients, gaussiir.cpp:84-210), the scale q that gives the requested sigma (the
// closed form of the forward-backward design, or the fixed-point iteration on the discrete-time
// variance, gaussiir.cpp:268-310), the poles scaled by q, the recursive coefficients
// b_k = coefficients of prod_i (1 - x / p_i) (gaussiir.cpp:334-341 forms the same polynomial from
// the elementary symmetric functions of the poles), the gain c = (sum b)^2 and the derivative's
// non-recursive taps (gaussiir.cpp:356-390).
//
// Line filter (device, FP64, one thread per image line): the line is extended by `border` samples
// on both sides by the boundary condition (as dip::Framework::Separable's input buffer), scanned
// forward into a scratch line p1 and backward into the output, with the reference's start-up
// values (GaussIIRLineFilter::Filter, gaussiir.cpp:465-712): the scans that the reference
// unrolls start from a constant history equal to the first (last) value divided by the
// coefficients' sum; the others set their first `order` values to that constant.  Only the
// `n` samples of the line proper are written.  The scratch line holds p1 position-major
// ([position][line]) so that both scans read it with unit stride across a warp.
//
// Pass chain as dip::Framework::Separable with a dfloat buffer (gaussiir.cpp:770-787): axes by
// increasing input stride, in -> intermediate (dfloat, normal strides) -> ... -> out; the input is
// converted to double on load, the last pass converts to the output type (clamp_cast).  This file
// is compiled without FMA contraction (each scan step is the reference's sequence of double
// multiplies and subtractions).
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

namespace {

constexpr int kIirMaxOrder = 5;      // recursion order (number of poles)
constexpr int kIirThreads = 128;

using cplx = std::complex< double >;

// Everything the line filter of one axis needs.
struct IirAxis {
   int32_t nn;               // recursion order
   int64_t border;           // extension on each side
   double b[ 6 ];            // b[1..nn]: recursive coefficients, both scans
   double a1[ 3 ], a2[ 3 ];  // non-recursive taps of the forward and backward scans (derivatives)
   int32_t lo1, hi1, lo2, hi2;   // nonzero range of a1 / a2
   double c;                 // gain of the backward scan
   double den;               // 1 + b[1] + ... + b[5]: the start-up divisor
   int32_t order1, order2;   // start-up lengths of the generic scans
   int32_t copy1, copy2;     // the scan's input is the sample itself (order 0)
   int32_t fmode, bmode;     // 0 generic start-up, 1 constant history (copy), 2 / 3 the derivative forms
   int32_t fstep, bstep;     // unroll step of the reference's scan (its tail reverts to the generic form)
};

// ---------------------------------------------------------------------------------------------
// Host: filter design.
// ---------------------------------------------------------------------------------------------

// The z-domain poles for `nn` and the derivative order; `fb` is set when the design falls back
// to (or is) the forward-backward one.  Tables of gaussiir.cpp:84-210 (published design values).
std::vector< cplx > iir_poles( int nn, int order, bool& fb ) {
   if( !fb ) {
      switch( nn ) {
         case 5:
            if( order == 2 ) { return { { 0.70381, 1.38271 }, { 0.70381, -1.38271 }, { 1.42239, 0.77978 }, { 1.42239, -0.77978 }, { 1.69319, 0.0 } }; }
            if( order == 1 ) { return { { 0.70237, 1.38717 }, { 0.70237, -1.38717 }, { 1.43280, 0.77903 }, { 1.43280, -0.77903 }, { 1.70346, 0.0 } }; }
            return { { 0.85991, 1.45235 }, { 0.85991, -1.45235 }, { 1.60953, 0.83009 }, { 1.60953, -0.83009 }, { 1.87040, 0.0 } };
         case 4:
            if( order == 2 ) { return { { 0.94576, 1.21364 }, { 0.94576, -1.21364 }, { 1.59892, 0.42668 }, { 1.59892, -0.42668 } }; }
            if( order == 1 ) { return { { 1.04198, 1.25046 }, { 1.04198, -1.25046 }, { 1.69337, 0.45006 }, { 1.69337, -0.45006 } }; }
            return { { 1.13231, 1.28122 }, { 1.13231, -1.28122 }, { 1.78532, 0.46766 }, { 1.78532, -0.46766 } };
         case 3:
            if( order == 2 ) { return { { 1.21969, 0.91724 }, { 1.21969, -0.91724 }, { 1.69485, 0.0 } }; }
            if( order == 1 ) { return { { 1.32094, 0.97057 }, { 1.32094, -0.97057 }, { 1.77635, 0.0 } }; }
            return { { 1.41650, 1.00829 }, { 1.41650, -1.00829 }, { 1.86131, 0.0 } };
         case 2: return { { 1.69580, 0.59955 }, { 1.69580, -0.59955 } };
         case 1: return { { 2.00000, 0.00000 } };
         default: break;   // any other order: the forward-backward design of order 3 (Abramowitz and Stegun)
      }
      fb = true;
      return { { 2.1078345, 1.4058574 }, { 2.1078345, -1.4058574 }, { 2.1668048, 0.0 } };
   }
   switch( nn ) {
      case 5: return { { 2.19406, 1.90251 }, { 2.19406, -1.90251 }, { 2.31029, 0.598022 }, { 2.31029, -0.598022 }, { 7.64071, 0.0 } };
      case 4: return { { 2.06954, 1.90416 }, { 2.06954, -1.90416 }, { 2.18403, 0.593635 }, { 2.18403, -0.593635 } };
      default: return { { 2.1078345, 1.4058574 }, { 2.1078345, -1.4058574 }, { 2.1668048, 0.0 } };
   }
}

// A pole of the discrete-time design raised to the power 1/q, in polar form as the reference
// evaluates it (modulus^(1/q) through exp(log(.)/q), phase from atan(im/re)).
cplx pole_power( cplx p, double q ) {
   double m = std::sqrt( p.real() * p.real() + p.imag() * p.imag() );
   double ph = std::atan( p.imag() / p.real() );
   m = std::exp( std::log( m ) / q );
   ph = ph / q;
   return { m * std::cos( ph ), m * std::sin( ph ) };
}

// Standard deviation of the forward-backward filter with the discrete-time poles raised to 1/q:
// the sum of the variances of each conjugate pair and of the real pole (gaussiir.cpp:55-82).
double dtf_sigma( std::vector< cplx > const& pp, double q ) {
   size_t const nn = pp.size();
   double var = 0.0;
   for( size_t m = 0; m + 1 < nn; m += 2 ) {
      cplx const r = pole_power( pp[ m ], q );
      double const re = r.real(), im = r.imag();
      double d = 1 - 2 * re + re * re + im * im;
      d *= d;
      var += ( 4 * ( re + ( re - 2 ) * ( re * re + im * im ))) / d;
   }
   if( nn & 1u ) {
      double const re = pole_power( pp[ nn - 1 ], q ).real();
      var += ( 2 * re ) / (( re - 1 ) * ( re - 1 ));
   }
   return std::sqrt( var );
}

// Filter parameters of one axis (FillGaussIIRParams, gaussiir.cpp:241-446).  Returns DIPCU_OK or
// an error for derivative orders above 4.
int iir_design( double sigma, int order, int filter_order, bool forward_backward, double truncation, IirAxis& ax ) {
   if( order > 4 ) { return record_error( DIPCU_ERR_INVALID_ARG, "Not implemented" ); }
   if( truncation <= 0.0 ) { truncation = 3.0; }
   truncation = std::min( truncation, max_gauss_truncation( false ));
   ax = IirAxis{};
   ax.border = std::max< int64_t >( 5, static_cast< int64_t >( sigma * truncation + 0.5 ));
   bool fb = forward_backward;
   std::vector< cplx > pp = iir_poles( filter_order, order, fb );
   int const nn = static_cast< int >( pp.size() );
   double q = 0.0;
   if( fb ) {
      // The filter's variance is q2 q^2 + q1 q (pairs and the real pole); solve for sigma^2.
      double const q0 = -sigma * sigma;
      double q1 = 0.0, q2 = 0.0;
      for( int m = 0; m + 1 < nn; m += 2 ) {
         double const re = pp[ m ].real(), im = pp[ m ].imag();
         double const t1 = 4 * ( -1 + 3 * re - 3 * re * re - im * im + re * ( re * re + im * im ));
         double const t2 = 4 * ( 1 - 2 * re + re * re - im * im );
         double d = 1 - 2 * re + re * re + im * im;
         d *= d;
         q1 += t1 / d;
         q2 += t2 / d;
      }
      if( nn & 1 ) {
         double const d = pp[ nn - 1 ].real() - 1.0;
         q1 += 2.0 / d;
         q2 += 2.0 / ( d * d );
      }
      double const t = std::sqrt( q1 * q1 - 4.0 * q2 * q0 );
      double const ra = ( -q1 + t ) / ( 2 * q2 );
      double const rb = ( -q1 - t ) / ( 2 * q2 );
      q = ra > rb ? ra : rb;
      for( auto& p : pp ) { p = { 1.0 + ( p.real() - 1.0 ) / q, p.imag() / q }; }
   } else {
      // Fixed-point iteration q <- q + (sigma - sigma(q)) / 2 from q = sigma / 2, to 1e-6.
      q = sigma / 2.0;
      double const q0 = q;
      double qs = dtf_sigma( pp, q );
      for( int it = 0; std::abs( sigma - qs ) > 0.000001 && it < 100; ++it ) {
         q += q0 - qs / 2.0;
         qs = dtf_sigma( pp, q );
      }
      for( auto& p : pp ) { p = pole_power( p, q ); }
   }
   // Denominator prod_i (1 - x / p_i), expanded one pole at a time.
   std::vector< cplx > poly( 1, cplx( 1.0, 0.0 ));
   for( auto const& p : pp ) {
      std::vector< cplx > next( poly.size() + 1, cplx( 0.0, 0.0 ));
      cplx const r = cplx( 1.0, 0.0 ) / p;
      for( size_t k = 0; k < poly.size(); ++k ) {
         next[ k ] += poly[ k ];
         next[ k + 1 ] -= poly[ k ] * r;
      }
      poly.swap( next );
   }
   ax.nn = nn;
   double sum = 0.0;
   for( int k = 0; k <= nn; ++k ) {
      double const v = poly[ static_cast< size_t >( k ) ].real();
      if( k > 0 ) { ax.b[ k ] = v; }
      sum += k == 0 ? 1.0 : v;
   }
   ax.c = sum * sum;
   ax.den = 1.0;
   for( int k = 1; k <= 5; ++k ) { ax.den += ax.b[ k ]; }
   // Derivative taps: a1 acts on the input at offsets 0, 1, 2 back, a2 on p1 at 0, 1, 2 ahead.
   static double const taps1[ 5 ][ 3 ] = { { 1, 0, 0 }, { 0.5, 0, -0.5 }, { 1, -1, 0 }, { 1, -2, 1 }, { 1, -2, 1 } };
   static double const taps2[ 5 ][ 3 ] = { { 1, 0, 0 }, { 0, 1, 0 }, { -1, 1, 0 }, { -0.5, 0, 0.5 }, { 1, -2, 1 } };
   for( int k = 0; k < 3; ++k ) {
      ax.a1[ k ] = taps1[ order ][ k ];
      ax.a2[ k ] = taps2[ order ][ k ];
   }
   ax.lo1 = ax.lo2 = 3;
   ax.hi1 = ax.hi2 = -1;
   for( int k = 0; k < 3; ++k ) {
      if( ax.a1[ k ] != 0.0 ) { ax.lo1 = std::min( ax.lo1, k ); ax.hi1 = k; }
      if( ax.a2[ k ] != 0.0 ) { ax.lo2 = std::min( ax.lo2, k ); ax.hi2 = k; }
   }
   ax.order1 = std::max( nn, ax.hi1 );
   ax.order2 = std::max( nn, ax.hi2 );
   ax.copy1 = ax.hi1 == 0 && ax.a1[ 0 ] == 1.0;
   ax.copy2 = ax.hi2 == 0 && ax.a2[ 0 ] == 1.0;
   // The scans the reference writes out for recursion orders 3-5: order 0 (both scans), and the
   // first and second derivatives at their default orders 4 and 5.
   ax.fmode = ax.bmode = 0;
   if( ax.order1 >= 3 && ax.order1 <= 5 ) {
      if( ax.copy1 ) { ax.fmode = 1; }
      else if( ax.order1 == 4 && order == 1 ) { ax.fmode = 2; }
      else if( ax.order1 == 5 && order == 2 ) { ax.fmode = 3; }
   }
   if( ax.order2 >= 3 && ax.order2 <= 5 ) {
      if( ax.copy2 ) { ax.bmode = 1; }
      else if( ax.order2 == 4 && order == 1 ) { ax.bmode = 2; }
      else if( ax.order2 == 5 && order == 2 ) { ax.bmode = 3; }
   }
   ax.fstep = ax.order1;
   ax.bstep = ax.order2;
   return DIPCU_OK;
}

// Stream-ordered scratch buffers, freed (stream-ordered) when the call returns.
struct IirScratch {
   std::vector< void* > bufs;
   cudaStream_t st;
   ~IirScratch() { for( void* p : bufs ) { cudaFreeAsync( p, st ); } }
   void* get( size_t bytes ) {
      void* p = nullptr;
      if( cudaMallocAsync( &p, bytes, st ) != cudaSuccess ) { cudaGetLastError(); return nullptr; }
      bufs.push_back( p );
      return p;
   }
};

// ---------------------------------------------------------------------------------------------
// Device: one pass along one axis.
// ---------------------------------------------------------------------------------------------

struct IirPass {
   IirAxis ax;
   void const* src;
   int32_t src_dt;
   void* dst;
   int32_t dst_dt;
   double* p1;               // scratch: (n + 2 border) x nlines doubles, position-major
   int64_t n;                // line length
   int64_t ss, ds;           // strides along the axis
   int32_t bc;
   int32_t nouter;
   int64_t osz[ DIPCU_MAX_DIMS ], oss[ DIPCU_MAX_DIMS ], ods[ DIPCU_MAX_DIMS ];   // the other axes
   int64_t nlines;
};

__global__ void __launch_bounds__( kIirThreads ) iir_pass_kernel( IirPass const __grid_constant__ a ) {
   int64_t const line = static_cast< int64_t >( blockIdx.x ) * blockDim.x + threadIdx.x;
   if( line >= a.nlines ) { return; }
   int64_t so = 0, dof = 0;
   {
      int64_t t = line;
      for( int k = 0; k < a.nouter; ++k ) {
         int64_t const c = t % a.osz[ k ];
         t /= a.osz[ k ];
         so += c * a.oss[ k ];
         dof += c * a.ods[ k ];
      }
   }
   IirAxis const& ax = a.ax;
   int64_t const n = a.n, B = ax.border, L = n + 2 * B;
   auto load = [ & ]( int64_t i ) { return load_as< double >( a.src, a.src_dt, so + i * a.ss ); };
   // extended input sample at buffer position ii (the line proper starts at B)
   auto p0 = [ & ]( int64_t ii ) -> double {
      int64_t const j = ii - B;
      if( j >= 0 && j < n ) { return load( j ); }
      return bc_extend< double >( j, n, a.bc, B, load );
   };
   double* const p1 = a.p1 + line;
   int64_t const ps = a.nlines;
   int const nn = ax.nn;

   // ---- forward scan ----
   double R;
   int64_t s;
   switch( ax.fmode ) {
      case 1: R = p0( 0 ) / ax.den; s = 0; break;
      case 2: R = ( p0( 1 ) - p0( 0 )) / ax.den; s = 2; break;
      case 3: R = ( p0( 1 ) - p0( 0 )) / ax.den; s = 1; break;
      default: {
         double v = 0.0;
         for( int k = ax.lo1; k <= ax.hi1; ++k ) { v += ax.a1[ k ] * p0( ax.hi1 - k ); }
         R = v / ax.den;
         s = ax.order1;
      }
   }
   // the reference's unrolled scan stops at the first multiple of the step past L - step; the
   // remaining samples take the generic form
   int64_t tail = s;
   if( ax.fmode >= 2 && s < L - ax.fstep ) { tail = s + (( L - ax.fstep - s + ax.fstep - 1 ) / ax.fstep ) * ax.fstep; }
   double h[ kIirMaxOrder + 1 ];     // h[k] = p1[ii - k]
   for( int k = 1; k <= kIirMaxOrder; ++k ) { h[ k ] = R; }
   for( int64_t ii = 0; ii < s && ii < L; ++ii ) {
      p1[ ii * ps ] = R;
      for( int k = kIirMaxOrder; k > 1; --k ) { h[ k ] = h[ k - 1 ]; }
      h[ 1 ] = R;
   }
   double x1 = s >= 1 ? p0( s - 1 ) : 0.0, x2 = s >= 2 ? p0( s - 2 ) : 0.0;   // p0[ii - 1], p0[ii - 2]
   for( int64_t ii = s; ii < L; ++ii ) {
      double const x0 = p0( ii );
      double v;
      if( ax.copy1 ) {
         v = x0;
      } else if( ax.fmode == 2 && ii < tail ) {
         v = 0.5 * ( x0 - x2 );
      } else if( ax.fmode == 3 && ii < tail ) {
         v = x0 - x1;
      } else {
         double const xs[ 3 ] = { x0, x1, x2 };
         v = 0.0;
         for( int k = ax.lo1; k <= ax.hi1; ++k ) { v += ax.a1[ k ] * xs[ k ]; }
      }
      for( int k = 1; k <= nn; ++k ) { v -= ax.b[ k ] * h[ k ]; }
      p1[ ii * ps ] = v;
      for( int k = kIirMaxOrder; k > 1; --k ) { h[ k ] = h[ k - 1 ]; }
      h[ 1 ] = v;
      x2 = x1;
      x1 = x0;
   }

   // ---- backward scan ----
   auto out = [ & ]( int64_t ii, double v ) {
      int64_t const j = ii - B;
      if( j >= 0 && j < n ) { store_from< double >( a.dst, a.dst_dt, dof + j * a.ds, v ); }
   };
   double const c = ax.c;
   int64_t top;   // first sample the generic loop computes (going down)
   switch( ax.bmode ) {
      case 1: R = c * p1[ ( L - 1 ) * ps ] / ax.den; top = L - 1; break;
      case 2: R = c * p1[ ( L - 1 ) * ps ] / ax.den; top = L - 2; break;
      case 3: R = c * ( -p1[ ( L - 2 ) * ps ] + p1[ ( L - 1 ) * ps ] ) / ax.den; top = L - 2; break;
      default: {
         double v = 0.0;
         for( int k = ax.lo2; k <= ax.hi2; ++k ) { v += ax.a2[ k ] * p1[ ( L - 1 - ax.hi2 + k ) * ps ]; }
         R = v / ax.den;
         top = L - 1 - ax.order2;
      }
   }
   int64_t btail = top;   // samples at or below it take the generic form
   if( ax.bmode >= 2 ) { btail = top >= ax.bstep ? top - (( top - ax.bstep ) / ax.bstep + 1 ) * ax.bstep : top; }
   for( int k = 1; k <= kIirMaxOrder; ++k ) { h[ k ] = R; }   // h[k] = p2[ii + k]
   for( int64_t ii = L - 1; ii > top; --ii ) {
      double const v = ax.bmode == 0 ? c * R : R;
      out( ii, v );
      for( int k = kIirMaxOrder; k > 1; --k ) { h[ k ] = h[ k - 1 ]; }
      h[ 1 ] = v;
   }
   double y1 = top + 1 < L ? p1[ ( top + 1 ) * ps ] : 0.0, y2 = top + 2 < L ? p1[ ( top + 2 ) * ps ] : 0.0;
   for( int64_t ii = top; ii >= 0; --ii ) {
      double const y0 = p1[ ii * ps ];
      double v;
      if( ax.copy2 ) {
         v = c * y0;
      } else if( ax.bmode == 2 && ii > btail ) {
         v = c * y1;
      } else if( ax.bmode == 3 && ii > btail ) {
         v = c * ( -y0 + y1 );
      } else {
         double const ys[ 3 ] = { y0, y1, y2 };
         double m = 0.0;
         for( int k = ax.lo2; k <= ax.hi2; ++k ) { m += ax.a2[ k ] * ys[ k ]; }
         v = c * m;
      }
      for( int k = 1; k <= nn; ++k ) { v -= ax.b[ k ] * h[ k ]; }
      out( ii, v );
      for( int k = kIirMaxOrder; k > 1; --k ) { h[ k ] = h[ k - 1 ]; }
      h[ 1 ] = v;
      y2 = y1;
      y1 = y0;
   }
}

} // namespace

} // namespace dipcu

using namespace dipcu;

extern "C" {

int dipcu_gauss_iir( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sigmas,
                     uint32_t const* orders, int32_t const* bcs, uint32_t const* filter_orders, int32_t design,
                     double truncation, void* stream_ ) {
   cudaStream_t stream = static_cast< cudaStream_t >( stream_ );
   if( !sigmas || !orders || !bcs ) { return record_error( DIPCU_ERR_INVALID_ARG, "null parameter array" ); }
   if( design != DIPCU_IIR_DISCRETE_TIME_FIT && design != DIPCU_IIR_FORWARD_BACKWARD ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "Invalid flag" );
   }
   if( int st = check_pair( in, out )) { return st; }
   int const nd = in->ndims;
   // Per-axis parameters (GaussIIR, gaussiir.cpp:725-768): axes with sigma > 0 and size > 1;
   // default recursion order: order + 3, 5 above order 2.
   std::vector< IirAxis > ax( static_cast< size_t >( nd ));
   std::vector< bool > proc( static_cast< size_t >( nd ), false );
   for( int d = 0; d < nd; ++d ) {
      if( !( sigmas[ d ] > 0.0 ) || in->sizes[ d ] <= 1 ) { continue; }
      if( bcs[ d ] < 0 || bcs[ d ] >= BC_ALREADY_EXPANDED ) {
         return record_error( DIPCU_ERR_UNSUPPORTED_BC, "Boundary condition not supported" );
      }
      int const fo = filter_orders ? static_cast< int >( filter_orders[ d ] )
                                   : ( orders[ d ] > 2 ? 5 : static_cast< int >( orders[ d ] ) + 3 );
      if( int st = iir_design( sigmas[ d ], static_cast< int >( orders[ d ] ), fo, design == DIPCU_IIR_FORWARD_BACKWARD,
                               truncation, ax[ static_cast< size_t >( d ) ] )) {
         return st;
      }
      proc[ static_cast< size_t >( d ) ] = true;
   }
   std::vector< int > order;
   for( int d = 0; d < nd; ++d ) {
      if( proc[ static_cast< size_t >( d ) ] ) { order.push_back( d ); }
   }
   // by increasing input stride (stable), as Framework::Separable's sortIndices
   for( size_t i = 1; i < order.size(); ++i ) {
      int const e = order[ i ];
      size_t j = i;
      while( j > 0 && in->strides[ order[ j - 1 ]] > in->strides[ e ] ) { order[ j ] = order[ j - 1 ]; --j; }
      order[ j ] = e;
   }
   if( order.empty() ) { return run_convert( in, out, stream ); }
   int64_t npix = 1;
   for( int d = 0; d < nd; ++d ) { npix *= in->sizes[ d ]; }
   IirScratch sc{ {}, stream };
   // intermediate image (dfloat, normal strides) when the output is not dfloat and there are passes
   // to chain; a dfloat output is filtered in place, pass after pass (each line is read whole by
   // the forward scan before its backward scan writes it, and lines are disjoint)
   bool const inter = out->dtype != DT_DFLOAT && order.size() > 1;
   dipcu_image_desc mid{};
   if( inter ) {
      mid.dtype = DT_DFLOAT;
      mid.ndims = nd;
      int64_t st = 1;
      for( int d = 0; d < nd; ++d ) { mid.sizes[ d ] = in->sizes[ d ]; mid.strides[ d ] = st; st *= in->sizes[ d ]; }
      mid.data = sc.get( static_cast< size_t >( npix ) * 8 );
      if( !mid.data ) { return record_error( DIPCU_ERR_CUDA, "cudaMallocAsync (intermediate)" ); }
   }
   int64_t maxp1 = 0;
   for( int d : order ) {
      IirAxis const& x = ax[ static_cast< size_t >( d ) ];
      maxp1 = std::max( maxp1, ( npix / in->sizes[ d ] ) * ( in->sizes[ d ] + 2 * x.border ));
   }
   double* p1 = static_cast< double* >( sc.get( static_cast< size_t >( maxp1 ) * 8 ));
   if( !p1 ) { return record_error( DIPCU_ERR_CUDA, "cudaMallocAsync (scan line)" ); }
   dipcu_image_desc const* src = in;
   for( size_t r = 0; r < order.size(); ++r ) {
      int const d = order[ r ];
      bool const last = r + 1 == order.size();
      dipcu_image_desc const* dst = ( last || !inter ) ? out : &mid;
      IirPass p{};
      p.ax = ax[ static_cast< size_t >( d ) ];
      p.src = src->data;
      p.src_dt = src->dtype;
      p.dst = dst->data;
      p.dst_dt = dst->dtype;
      p.p1 = p1;
      p.n = in->sizes[ d ];
      p.ss = src->strides[ d ];
      p.ds = dst->strides[ d ];
      p.bc = bcs[ d ];
      p.nlines = npix / p.n;
      for( int k = 0; k < nd; ++k ) {
         if( k == d ) { continue; }
         p.osz[ p.nouter ] = in->sizes[ k ];
         p.oss[ p.nouter ] = src->strides[ k ];
         p.ods[ p.nouter ] = dst->strides[ k ];
         ++p.nouter;
      }
      int64_t const blocks = ( p.nlines + kIirThreads - 1 ) / kIirThreads;
      if( blocks > 0x7fffffff ) { return record_error( DIPCU_ERR_INVALID_ARG, "image too large" ); }
      iir_pass_kernel<<< static_cast< unsigned >( blocks ), kIirThreads, 0, stream >>>( p ); count_launch();
      cudaError_t const e = cudaGetLastError();
      if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
      src = dst;
   }
   return DIPCU_OK;
}

} // extern "C"
