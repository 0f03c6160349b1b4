// Shared host/device definitions of the dipcu Gaussian FIR path: sample types and conversions,
// boundary extension, and Gaussian kernel weights.  Everything here is __host__ __device__ so
// that the same code builds the weight tables on the host, runs inside the kernels, and is
// checked on the CPU against the oracle by tests/test_host_logic.py.
#pragma once

#include <stdint.h>

#if defined( __CUDACC__ ) || defined( __CUDACC_RTC__ )
#define DIPCU_HD __host__ __device__ __forceinline__
#else
#define DIPCU_HD inline
#include <math.h>
#endif

namespace dipcu {

// Sample type codes (identical to dipcu_dtype in include/dipcu.h).
enum DType : int32_t {
   DT_BIN = 0, DT_UINT8 = 1, DT_UINT16 = 2, DT_UINT32 = 3, DT_UINT64 = 4,
   DT_SINT8 = 5, DT_SINT16 = 6, DT_SINT32 = 7, DT_SINT64 = 8, DT_SFLOAT = 9, DT_DFLOAT = 10
};

// dip::BoundaryCondition enumerator values (include/diplib/boundary.h:65-80).
enum Bc : int32_t {
   BC_SYMMETRIC_MIRROR = 0, BC_ASYMMETRIC_MIRROR = 1, BC_ANTISYMMETRIC_REFLECT = 2, BC_PERIODIC = 3,
   BC_ASYMMETRIC_PERIODIC = 4, BC_ADD_ZEROS = 5, BC_ADD_MAX_VALUE = 6, BC_ADD_MIN_VALUE = 7,
   BC_ZERO_ORDER_EXTRAPOLATE = 8, BC_FIRST_ORDER_EXTRAPOLATE = 9, BC_SECOND_ORDER_EXTRAPOLATE = 10,
   BC_THIRD_ORDER_EXTRAPOLATE = 11, BC_ALREADY_EXPANDED = 12
};

DIPCU_HD int dtype_size( int32_t dt ) {
   switch( dt ) {
      case DT_BIN: case DT_UINT8: case DT_SINT8: return 1;
      case DT_UINT16: case DT_SINT16: return 2;
      case DT_UINT32: case DT_SINT32: case DT_SFLOAT: return 4;
      case DT_UINT64: case DT_SINT64: case DT_DFLOAT: return 8;
      default: return 0;
   }
}

// DataType::SuggestFlex (src/library/datatype.cpp:109-124 in DIPlib), real types.
DIPCU_HD int32_t suggest_flex( int32_t dt ) {
   switch( dt ) {
      case DT_UINT32: case DT_SINT32: case DT_UINT64: case DT_SINT64: case DT_DFLOAT: return DT_DFLOAT;
      default: return DT_SFLOAT;
   }
}

// ------------------------------------------------------------------------------------------
// Sample access.  `load_as<T>` is the conversion CopyBuffer applies when filling the line
// buffer (clamp_cast to a float type is a plain cast); `store_from<T>` is clamp_cast< outT >
// (include/diplib/library/clamp_cast.h:212-244): clamp to the target range, then truncate.
// ------------------------------------------------------------------------------------------

template< typename T >
DIPCU_HD T load_as( void const* p, int32_t dt, int64_t i ) {
   switch( dt ) {
      case DT_BIN: return static_cast< T >( static_cast< uint8_t const* >( p )[ i ] ? 1 : 0 );
      case DT_UINT8: return static_cast< T >( static_cast< uint8_t const* >( p )[ i ] );
      case DT_UINT16: return static_cast< T >( static_cast< uint16_t const* >( p )[ i ] );
      case DT_UINT32: return static_cast< T >( static_cast< uint32_t const* >( p )[ i ] );
      case DT_UINT64: return static_cast< T >( static_cast< uint64_t const* >( p )[ i ] );
      case DT_SINT8: return static_cast< T >( static_cast< int8_t const* >( p )[ i ] );
      case DT_SINT16: return static_cast< T >( static_cast< int16_t const* >( p )[ i ] );
      case DT_SINT32: return static_cast< T >( static_cast< int32_t const* >( p )[ i ] );
      case DT_SINT64: return static_cast< T >( static_cast< int64_t const* >( p )[ i ] );
      case DT_SFLOAT: return static_cast< T >( static_cast< float const* >( p )[ i ] );
      case DT_DFLOAT: return static_cast< T >( static_cast< double const* >( p )[ i ] );
      default: return T( 0 );
   }
}

template< typename T >
DIPCU_HD T clampv( T v, T lo, T hi ) { return v < lo ? lo : ( v > hi ? hi : v ); }

template< typename T >
DIPCU_HD void store_from( void* p, int32_t dt, int64_t i, T v ) {
   switch( dt ) {
      case DT_BIN: static_cast< uint8_t* >( p )[ i ] = ( v != T( 0 )) ? 1 : 0; break;
      case DT_UINT8: static_cast< uint8_t* >( p )[ i ] = static_cast< uint8_t >( clampv< T >( v, T( 0 ), T( 255 ))); break;
      case DT_UINT16: static_cast< uint16_t* >( p )[ i ] = static_cast< uint16_t >( clampv< T >( v, T( 0 ), T( 65535 ))); break;
      case DT_UINT32: static_cast< uint32_t* >( p )[ i ] = static_cast< uint32_t >( clampv< T >( v, T( 0 ), T( 4294967295.0 ))); break;
      case DT_UINT64: static_cast< uint64_t* >( p )[ i ] = static_cast< uint64_t >( clampv< T >( v, T( 0 ), T( 18446744073709549568.0 ))); break;
      case DT_SINT8: static_cast< int8_t* >( p )[ i ] = static_cast< int8_t >( clampv< T >( v, T( -128 ), T( 127 ))); break;
      case DT_SINT16: static_cast< int16_t* >( p )[ i ] = static_cast< int16_t >( clampv< T >( v, T( -32768 ), T( 32767 ))); break;
      case DT_SINT32: static_cast< int32_t* >( p )[ i ] = static_cast< int32_t >( clampv< T >( v, T( -2147483648.0 ), T( 2147483647.0 ))); break;
      case DT_SINT64: static_cast< int64_t* >( p )[ i ] = static_cast< int64_t >( clampv< T >( v, T( -9223372036854775808.0 ), T( 9223372036854774784.0 ))); break;
      case DT_SFLOAT: static_cast< float* >( p )[ i ] = static_cast< float >( v ); break;
      case DT_DFLOAT: static_cast< double* >( p )[ i ] = static_cast< double >( v ); break;
      default: break;
   }
}

// ------------------------------------------------------------------------------------------
// Boundary extension.
//
// DIPlib extends each image line into a buffer with detail::ExpandBuffer
// (src/library/copy_buffer.cpp:359-813), walking pointers away from the line ends.  The
// closed forms below give the same value at any position j outside [0, n) directly, which is
// what a tile kernel needs.  `border` is the extension length (the kernel half-width), which
// the polynomial extrapolations depend on.  `load(i)` returns in-range sample i as T.
//
//  mirror walk:   position -k (or n-1+k) reads sample T(k), a triangle wave of period
//                 2(n-1); the walk's sign flips after every visit of an end sample, so the
//                 asymmetric variant negates when floor((k-1)/(n-1)) is even.
//  periodic walk: -k reads (-k mod n), n-1+k reads (k-1 mod n); sign flips every n steps.
//  antisymmetric reflection: the reflection offset accumulates D = x[0]-x[n-1] per bounce.
// ------------------------------------------------------------------------------------------

DIPCU_HD int64_t pos_mod( int64_t a, int64_t m ) {
   int64_t r = a % m;
   return r < 0 ? r + m : r;
}

// Index mapping for the BCs that read an existing sample.  Returns the source index; *neg is
// set when the asymmetric variant inverts the sample.  Only valid for j outside [0, n), n >= 1.
DIPCU_HD int64_t bc_map_index( int64_t j, int64_t n, int32_t bc, bool* neg ) {
   *neg = false;
   if( n == 1 ) {
      *neg = ( bc == BC_ASYMMETRIC_MIRROR || bc == BC_ASYMMETRIC_PERIODIC );
      return 0;
   }
   switch( bc ) {
      case BC_SYMMETRIC_MIRROR:
      case BC_ASYMMETRIC_MIRROR:
      case BC_ANTISYMMETRIC_REFLECT: {
         int64_t p = n - 1;
         int64_t k = ( j < 0 ) ? -j : j - p;             // distance beyond the end sample, >= 1
         int64_t t = k % ( 2 * p );
         if( t > p ) { t = 2 * p - t; }                  // triangle wave T(k)
         if( bc == BC_ASYMMETRIC_MIRROR ) { *neg = ((( k - 1 ) / p ) % 2 ) == 0; }
         return ( j < 0 ) ? t : p - t;
      }
      case BC_PERIODIC:
      case BC_ASYMMETRIC_PERIODIC: {
         int64_t k = ( j < 0 ) ? -j : j - ( n - 1 );
         if( bc == BC_ASYMMETRIC_PERIODIC ) { *neg = ((( k - 1 ) / n ) % 2 ) == 0; }
         return pos_mod( j, n );
      }
      case BC_ZERO_ORDER_EXTRAPOLATE:
      default:
         return j < 0 ? 0 : n - 1;
   }
}

template< typename T > struct NumLimits;
template<> struct NumLimits< float > { static DIPCU_HD float max() { return 3.402823466e+38f; } };
template<> struct NumLimits< double > { static DIPCU_HD double max() { return 1.7976931348623157e+308; } };

// Value of the extended line at j (outside [0, n)) for any supported BC.
template< typename T, typename Load >
DIPCU_HD T bc_extend( int64_t j, int64_t n, int32_t bc, int64_t border, Load const& load ) {
   bool left = j < 0;
   int64_t k = left ? -j : j - ( n - 1 );                // 1 .. border
   switch( bc ) {
      case BC_SYMMETRIC_MIRROR:
      case BC_ASYMMETRIC_MIRROR:
      case BC_PERIODIC:
      case BC_ASYMMETRIC_PERIODIC:
      case BC_ZERO_ORDER_EXTRAPOLATE: {
         bool neg;
         int64_t i = bc_map_index( j, n, bc, &neg );
         T v = load( i );
         return neg ? -v : v;
      }
      case BC_ADD_ZEROS: return T( 0 );
      case BC_ADD_MAX_VALUE: return NumLimits< T >::max();
      case BC_ADD_MIN_VALUE: return -NumLimits< T >::max();
      case BC_ANTISYMMETRIC_REFLECT: {                   // ExpandBufferAntiSymReflect, copy_buffer.cpp:552-589
         if( n == 1 ) { return load( 0 ); }
         int64_t p = n - 1;
         bool neg;
         int64_t i = bc_map_index( j, n, BC_SYMMETRIC_MIRROR, &neg );
         double e0 = static_cast< double >( load( left ? 0 : p ));
         double e1 = static_cast< double >( load( left ? p : 0 ));
         double d = e0 - e1;
         int64_t s = ( k - 1 ) / p;                      // completed bounces
         double xi = static_cast< double >( load( i ));
         double v = ( s % 2 ) ? static_cast< double >( s + 1 ) * d + xi
                              : 2.0 * e0 + static_cast< double >( s ) * d - xi;
         return static_cast< T >( v );
      }
      case BC_THIRD_ORDER_EXTRAPOLATE:
         if( n > 1 ) {                                   // ExpandBufferThirdOrder, copy_buffer.cpp:469-513
            double b = static_cast< double >( border ) + 1.0;
            double b12 = ( b + 1 ) * ( b + 1 );
            double d0 = static_cast< double >( load( left ? 0 : n - 1 ));
            double f1 = static_cast< double >( load( left ? 1 : n - 2 ));
            double d1 = -( 2.0 * d0 ) / b + d0 - ( b * b * f1 ) / b12;
            double d2 = ( 2.0 * b * f1 ) / b12 - ( d0 * ( 2.0 * b - 1.0 )) / ( b * b );
            double d3 = d0 / ( b * b ) - f1 / b12;
            double x = static_cast< double >( k );
            return static_cast< T >( d0 + x * d1 + x * x * d2 + x * x * x * d3 );
         }
         // fallthrough (a single sample: DIPlib falls back to second, then first order)
      case BC_SECOND_ORDER_EXTRAPOLATE:
         if( n > 1 ) {                                   // ExpandBufferSecondOrder, copy_buffer.cpp:423-458
            double b = static_cast< double >( border ) + 1.0;
            double d0 = static_cast< double >( load( left ? 0 : n - 1 ));
            double f1 = static_cast< double >( load( left ? 1 : n - 2 ));
            double d1 = ( b - 1.0 ) / b * d0 - b / ( b + 1.0 ) * f1;
            double d2 = -1.0 / b * d0 + 1.0 / ( b + 1.0 ) * f1;
            double x = static_cast< double >( k );
            return static_cast< T >( d0 + x * d1 + x * x * d2 );
         }
         // fallthrough
      case BC_FIRST_ORDER_EXTRAPOLATE: {                 // ExpandBufferFirstOrder, copy_buffer.cpp:386-417
         double d0 = static_cast< double >( load( left ? 0 : n - 1 ));
         double d1 = d0 / static_cast< double >( border + 1 );
         for( int64_t ii = 0; ii < k; ++ii ) { d0 -= d1; } // the reference's repeated subtraction
         return static_cast< T >( d0 );
      }
      default:
         return T( 0 );
   }
}

// True for the BCs whose extension of an intermediate (already filtered along another axis)
// image equals filtering of the extended input.  For these, one fused kernel that extends the
// input once reproduces DIPlib's pass-by-pass semantics (Framework::Separable extends each
// pass's input, src/library/framework_separable.cpp:369-380).
DIPCU_HD bool bc_is_index_map( int32_t bc ) {
   return bc == BC_SYMMETRIC_MIRROR || bc == BC_ASYMMETRIC_MIRROR || bc == BC_PERIODIC ||
          bc == BC_ASYMMETRIC_PERIODIC || bc == BC_ZERO_ORDER_EXTRAPOLATE || bc == BC_ADD_ZEROS;
}

// ------------------------------------------------------------------------------------------
// Gaussian kernel weights: HalfGaussianSize and MakeHalfGaussianInternal,
// src/linear/gauss.cpp:38-146 in DIPlib, restated; plus the analytic derivative of the
// normalised discrete kernel with respect to sigma (no DIPlib counterpart; used by the
// adjoint).  Output is the REVERSED half kernel as InternOneDimensionalFilter stores it
// (src/linear/convolution.cpp:76-156): w[0] is the centre tap, w[k] the tap at distance k.
// ------------------------------------------------------------------------------------------

constexpr double kPi = 3.14159265358979323846264338327950288;

// Round-to-nearest double operations that no compiler flag contracts or reorders (on the device
// the explicit _rn intrinsics; on the host plain IEEE operations and the C library's fma).
DIPCU_HD double rn_add( double a, double b ) {
#ifdef __CUDA_ARCH__
   return __dadd_rn( a, b );
#else
   return a + b;
#endif
}
DIPCU_HD double rn_mul( double a, double b ) {
#ifdef __CUDA_ARCH__
   return __dmul_rn( a, b );
#else
   return a * b;
#endif
}
DIPCU_HD double rn_fma( double a, double b, double c ) {
#ifdef __CUDA_ARCH__
   return __fma_rn( a, b, c );
#else
   return fma( a, b, c );
#endif
}

// Double-double arithmetic (value = hi + lo, |lo| <= ulp(hi) / 2) with the error-free
// transforms of Knuth (TwoSum), Dekker (FastTwoSum) and the fused-multiply-add product.
struct DD { double hi, lo; };
DIPCU_HD DD dd_fast_two_sum( double a, double b ) {   // |a| >= |b|
   double s = rn_add( a, b );
   return { s, rn_add( b, -rn_add( s, -a )) };
}
DIPCU_HD DD dd_two_sum( double a, double b ) {
   double s = rn_add( a, b );
   double bb = rn_add( s, -a );
   return { s, rn_add( rn_add( a, -rn_add( s, -bb )), rn_add( b, -bb )) };
}
DIPCU_HD DD dd_mul( DD a, DD b ) {
   double p = rn_mul( a.hi, b.hi );
   double e = rn_fma( a.hi, b.hi, -p );
   e = rn_add( e, rn_add( rn_mul( a.hi, b.lo ), rn_mul( a.lo, b.hi )));
   return dd_fast_two_sum( p, e );
}
DIPCU_HD DD dd_div_small( DD a, double n ) {          // a / n, n a small positive integer
   double q = a.hi / n;
   double p = rn_mul( q, n );
   double pe = rn_fma( q, n, -p );
   double rem = rn_add( rn_add( rn_add( a.hi, -p ), -pe ), a.lo );
   return dd_fast_two_sum( q, rem / n );
}
DIPCU_HD DD dd_add_one( DD a ) {                       // 1 + a, |a| < 1
   DD s = dd_two_sum( 1.0, a.hi );
   return dd_fast_two_sum( s.hi, rn_add( s.lo, a.lo ));
}

// exp(x) rounded to the nearest double for results in the normal range (x >= -708.39; the
// double-double evaluation is good to ~1e-30 relative; below that the scaled high part can be one
// subnormal unit off, a range the weights never reach).  Cody-Waite reduction x = k ln2 + r with |r| <= ln2 / 2 in
// double-double (ln2 as a double-double constant), then the Taylor series of exp(r) to r^24 / 24!
// (< 1e-33 truncation) by Horner's rule in double-double, then scaling by 2^k.  The device
// weights use it where DIPlib calls the C library's exp (an IEEE-accurate function whose results
// are the correctly rounded ones except for rare arguments), so that the device taps are the
// reference's bit for bit after the cast to float.
DIPCU_HD double exp_rn( double x ) {
   if( x != x ) { return x; }
   if( x > 709.782712893384 ) { return 1.0 / 0.0; }
   if( x < -745.2 ) { return 0.0; }
   constexpr double kLn2Hi = 6.93147180559945286227e-01;     // ln 2 rounded to double
   constexpr double kLn2Lo = 2.31904681384629955842e-17;     // ln 2 - kLn2Hi
   constexpr double kInvLn2 = 1.44269504088896338700e+00;
   double const k = rint( rn_mul( x, kInvLn2 ));
   double const p = rn_mul( k, kLn2Hi );
   double const pe = rn_fma( k, kLn2Hi, -p );                 // k kLn2Hi = p + pe exactly
   DD r = dd_two_sum( x, -p );
   r = dd_fast_two_sum( r.hi, rn_add( rn_add( r.lo, -pe ), -rn_mul( k, kLn2Lo )));
   DD t = { 1.0, 0.0 };
   for( int n = 24; n >= 1; --n ) {
      t = dd_add_one( dd_div_small( dd_mul( r, t ), static_cast< double >( n )));
   }
   return scalbn( t.hi, static_cast< int >( k ));
}

// The exp of the weights: the C library's on the host (the function DIPlib calls), exp_rn on the
// device (and on the host when DIPCU_WEIGHT_EXP_RN is defined, which the CPU tests use to check
// the device arithmetic against the reference).
DIPCU_HD double weight_exp( double x ) {
#if defined( __CUDA_ARCH__ ) || defined( DIPCU_WEIGHT_EXP_RN )
   return exp_rn( x );
#else
   return exp( x );
#endif
}

// maximum_gauss_truncation<T>() (include/diplib/library/numeric.h:69-76) for float / double.
DIPCU_HD double max_gauss_truncation( bool dt_double ) {
   return dt_double ? 8.490424416849509 : 5.646660101844052; // sqrt( -2 ln eps )
}

// Half-width h (border) of the kernel; the half kernel has h + 1 taps.
DIPCU_HD int64_t half_gaussian_size( double sigma, uint32_t order, double truncation, bool dt_double ) {
   if( truncation <= 0 ) { truncation = 3; }
   double mt = max_gauss_truncation( dt_double );
   truncation = ( mt < truncation ) ? mt : truncation;
   truncation += 0.5 * static_cast< double >( order );
   double v = ceil( truncation * sigma );
   return v > 0.0 ? static_cast< int64_t >( v ) : 0;
}

// Number of taps of the half kernel (MakeHalfGaussian): 1 for sigma == 0.
DIPCU_HD int64_t half_gaussian_length( double sigma, uint32_t order, double truncation, bool dt_double ) {
   if( sigma == 0.0 ) { return 1; }
   int64_t n = 1 + half_gaussian_size( sigma, order, truncation, dt_double );
   if( order > 2 && n < 2 ) { n = 2; }
   return n;
}

// Writes `len` = half_gaussian_length() taps (reversed: centre first) into w, and if dw is not
// null, d(w)/d(sigma).  T is the precision of the stored result.
template< typename T >
DIPCU_HD void make_half_gaussian( double sigma, uint32_t order, int64_t len, T* w, T* dw ) {
   if( sigma == 0.0 || len < 1 ) {
      if( len >= 1 ) { w[ 0 ] = T( 1 ); if( dw ) { dw[ 0 ] = T( 0 ); } }
      return;
   }
   double s2 = sigma * sigma;
   int64_t r0 = len - 1;
   switch( order ) {
      case 0: {                                          // gauss.cpp:66-82
         double factor = -0.5 / s2;
         double norm = 0.0, dnorm = 0.0;
         for( int64_t r = 1; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double g = weight_exp( factor * ( rad * rad ));
            norm += g;
            dnorm += g * rad * rad;
         }
         double S = norm * 2 + 1;                        // sum of the full kernel
         double inv = 1.0 / S;
         double dS = 2.0 * dnorm / ( s2 * sigma );       // dS/dsigma
         for( int64_t r = 0; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double g = ( r == 0 ) ? 1.0 : weight_exp( factor * ( rad * rad ));
            w[ r ] = static_cast< T >( g * inv );
            if( dw ) {
               double dg = g * rad * rad / ( s2 * sigma );
               dw[ r ] = static_cast< T >( dg * inv - g * inv * dS * inv );
            }
         }
         break;
      }
      case 1: {                                          // gauss.cpp:83-98
         double factor = -0.5 / s2;
         double moment = 0.0, dmoment = 0.0;
         for( int64_t r = 1; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double g = rad * weight_exp( factor * ( rad * rad ));
            moment += rad * g;
            dmoment += rad * g * rad * rad / ( s2 * sigma );
         }
         double inv = 1.0 / ( 2.0 * moment );
         w[ 0 ] = T( 0 );
         if( dw ) { dw[ 0 ] = T( 0 ); }
         for( int64_t r = 1; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double g = rad * weight_exp( factor * ( rad * rad ));
            w[ r ] = static_cast< T >( g * inv );
            if( dw ) {
               double dg = g * rad * rad / ( s2 * sigma );
               dw[ r ] = static_cast< T >( dg * inv - g * inv * dmoment / moment );
            }
         }
         break;
      }
      case 2: {                                          // gauss.cpp:99-124
         double norm = 1.0 / ( sqrt( 2.0 * kPi ) * sigma * s2 );
         double sum = 0.0, dsum = 0.0;                   // over r >= 1
         for( int64_t r = 1; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double sr2 = rad * rad / s2;
            double e = weight_exp( -0.5 * sr2 );
            sum += ( sr2 - 1.0 ) * norm * e;
            dsum += e * sr2 * ( sr2 - 3.0 ) / sigma;     // d/dsigma of (sr2-1) e, unnormalised
         }
         double g0 = -norm;
         double mean = ( sum * 2.0 + g0 ) / ( static_cast< double >( r0 ) * 2.0 + 1.0 );
         // Unnormalised (norm = 1) derivative terms: the final normalisation by the moment
         // removes `norm`, so d(w)/d(sigma) can be taken on g/norm.
         double dmean = ( dsum * 2.0 ) / ( static_cast< double >( r0 ) * 2.0 + 1.0 );
         double mean1 = mean / norm;
         double moment = 0.0, moment1 = 0.0, dmoment1 = 0.0;
         for( int64_t r = 1; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double sr2 = rad * rad / s2;
            double e = weight_exp( -0.5 * sr2 );
            double f = ( sr2 - 1.0 ) * norm * e - mean;
            moment += rad * rad * f;
            double f1 = ( sr2 - 1.0 ) * e - mean1;
            moment1 += rad * rad * f1;
            dmoment1 += rad * rad * ( e * sr2 * ( sr2 - 3.0 ) / sigma - dmean );
         }
         double inv = 1.0 / moment;
         for( int64_t r = 0; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double sr2 = rad * rad / s2;
            double e = weight_exp( -0.5 * sr2 );
            double g = ( r == 0 ) ? g0 : ( sr2 - 1.0 ) * norm * e;
            w[ r ] = static_cast< T >(( g - mean ) * inv );
            if( dw ) {
               double f1 = ( r == 0 ) ? ( -1.0 - mean1 ) : (( sr2 - 1.0 ) * e - mean1 );
               double df1 = (( r == 0 ) ? 0.0 : e * sr2 * ( sr2 - 3.0 ) / sigma ) - dmean;
               dw[ r ] = static_cast< T >(( df1 - f1 * dmoment1 / moment1 ) / moment1 );
            }
         }
         break;
      }
      case 3: {                                          // gauss.cpp:125-141
         double norm = 1.0 / ( sqrt( 2.0 * kPi ) * sigma * s2 * s2 );
         double moment = 0.0, moment1 = 0.0, dmoment1 = 0.0;
         for( int64_t r = 1; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double rr2 = rad * rad;
            double sr2 = rr2 / s2;
            double e = weight_exp( -0.5 * sr2 );
            double g = norm * e * ( rad * ( 3.0 - sr2 ));
            moment += g * rr2 * rad;
            double g1 = e * ( rad * ( 3.0 - sr2 ));
            moment1 += g1 * rr2 * rad;
            dmoment1 += rad * e * sr2 * ( 5.0 - sr2 ) / sigma * rr2 * rad;
         }
         double inv = 3.0 / moment;
         w[ 0 ] = T( 0 );
         if( dw ) { dw[ 0 ] = T( 0 ); }
         for( int64_t r = 1; r <= r0; ++r ) {
            double rad = static_cast< double >( r );
            double rr2 = rad * rad;
            double sr2 = rr2 / s2;
            double e = weight_exp( -0.5 * sr2 );
            double g = norm * e * ( rad * ( 3.0 - sr2 ));
            w[ r ] = static_cast< T >( g * inv );
            if( dw ) {
               double g1 = e * ( rad * ( 3.0 - sr2 ));
               double dg1 = rad * e * sr2 * ( 5.0 - sr2 ) / sigma;
               dw[ r ] = static_cast< T >( 3.0 * ( dg1 - g1 * dmoment1 / moment1 ) / moment1 );
            }
         }
         break;
      }
      default:
         break;
   }
}

} // namespace dipcu
