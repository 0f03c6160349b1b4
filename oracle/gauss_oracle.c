/* Test infrastructure only: plain-C restatement of DIPlib's Gaussian FIR path (the parity
 * oracle).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and
 * only as a checker.  Every function cites the reference code it restates; the floating-point
 * operation order follows the reference so that, compiled without FMA contraction
 * (-ffp-contract=off), results are bit-identical to the reference's own x86-64 build.
 *
 * Parity of this file is pinned against the reference itself (oracle/_ref/libdipref.so) and
 * against fixtures generated from it (tests/golden/).
 */
#include "gauss_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846264338327950288 /* dip::pi, include/diplib/library/numeric.h */

/* ------------------------------------------------------------------------------------------ */
/* Kernel weights                                                                             */
/* ------------------------------------------------------------------------------------------ */

/* maximum_gauss_truncation<T>(), include/diplib/library/numeric.h:69-76. */
static double max_gauss_truncation( int dt_double ) {
   return sqrt( -2.0 * log( dt_double ? DBL_EPSILON : (double)FLT_EPSILON ));
}

/* HalfGaussianSize, src/linear/gauss.cpp:38-51 (clamp_cast<dip::uint>(double) clamps at 0). */
size_t or_half_gaussian_size( double sigma, unsigned order, double truncation, int dt_double ) {
   if( truncation <= 0 ) {
      truncation = 3;
   }
   double max_trunc = max_gauss_truncation( dt_double );
   truncation = ( max_trunc < truncation ) ? max_trunc : truncation; /* std::min */
   truncation += 0.5 * (double)order;
   double v = ceil( truncation * sigma );
   if( !( v > 0.0 )) {
      return 0;
   }
   return (size_t)v;
}

/* MakeHalfGaussianInternal + MakeHalfGaussian, src/linear/gauss.cpp:53-165.  The half kernel
 * has x=0 at the right end (index r0). */
int or_make_half_gaussian( double sigma, unsigned order, double truncation, int dt_double, double* filter, int cap ) {
   if( sigma == 0.0 ) {
      if( cap >= 1 ) { filter[ 0 ] = 1.0; }
      return 1;
   }
   if( order > 3 ) {
      return -1;
   }
   size_t halfFilterSize = 1 + or_half_gaussian_size( sigma, order, truncation, dt_double );
   if( order > 2 && halfFilterSize < 2 ) {
      halfFilterSize = 2;
   }
   if( (size_t)cap < halfFilterSize ) {
      return (int)halfFilterSize; /* caller retries with a larger buffer */
   }
   size_t r0 = halfFilterSize - 1;
   double sigma2 = sigma * sigma;
   switch( order ) {
      case 0: {
         double factor = -0.5 / sigma2;
         double normalization = 0;
         filter[ r0 ] = 1.0;
         for( size_t rr = 1; rr < halfFilterSize; rr++ ) {
            double rad = (double)rr;
            double g = exp( factor * ( rad * rad ));
            filter[ r0 - rr ] = g;
            normalization += g;
         }
         normalization = 1.0 / ( normalization * 2 + 1 );
         for( size_t rr = 0; rr < halfFilterSize; rr++ ) {
            filter[ rr ] *= normalization;
         }
         break;
      }
      case 1: {
         double factor = -0.5 / sigma2;
         double moment = 0.0;
         filter[ r0 ] = 0.0;
         for( size_t rr = 1; rr < halfFilterSize; rr++ ) {
            double rad = (double)rr;
            double g = rad * exp( factor * ( rad * rad ));
            filter[ r0 - rr ] = g;
            moment += rad * g;
         }
         double normalization = 1.0 / ( 2.0 * moment );
         for( size_t rr = 0; rr < halfFilterSize - 1; rr++ ) {
            filter[ rr ] *= normalization;
         }
         break;
      }
      case 2: {
         double norm = 1.0 / ( sqrt( 2.0 * OR_PI ) * sigma * sigma2 );
         double mean = 0.0;
         filter[ r0 ] = -norm;
         for( size_t rr = 1; rr < halfFilterSize; rr++ ) {
            double rad = (double)rr;
            double sr2 = rad * rad / sigma2;
            double g = ( sr2 - 1.0 ) * norm * exp( -0.5 * sr2 );
            filter[ r0 - rr ] = g;
            mean += g;
         }
         mean = ( mean * 2.0 + filter[ r0 ] ) / ( (double)r0 * 2.0 + 1.0 );
         filter[ r0 ] -= mean;
         double moment = 0.0;
         for( size_t rr = 1; rr < halfFilterSize; rr++ ) {
            double rad = (double)rr;
            filter[ r0 - rr ] -= mean;
            moment += rad * rad * filter[ r0 - rr ];
         }
         double normalization = 1.0 / moment;
         for( size_t rr = 0; rr < halfFilterSize; rr++ ) {
            filter[ rr ] *= normalization;
         }
         break;
      }
      case 3: {
         double norm = 1.0 / ( sqrt( 2.0 * OR_PI ) * sigma * sigma2 * sigma2 );
         filter[ r0 ] = 0.0;
         double moment = 0.0;
         for( size_t rr = 1; rr < halfFilterSize; rr++ ) {
            double rad = (double)rr;
            double rr2 = rad * rad;
            double sr2 = rr2 / sigma2;
            double g = norm * exp( -0.5 * sr2 ) * ( rad * ( 3.0 - sr2 ));
            filter[ r0 - rr ] = g;
            moment += g * rr2 * rad;
         }
         double normalization = 3.0 / moment;
         for( size_t rr = 0; rr < halfFilterSize; rr++ ) {
            filter[ rr ] *= normalization;
         }
         break;
      }
   }
   return (int)halfFilterSize;
}

/* ------------------------------------------------------------------------------------------ */
/* Boundary extension: detail::ExpandBuffer, src/library/copy_buffer.cpp:359-813               */
/* The reference walks pointers; the index walks below visit the same samples in the same      */
/* order.  Instantiated for float and double buffers (the only buffer types on this path).     */
/* ------------------------------------------------------------------------------------------ */

#define OR_DEFINE_EXPAND( T, SUFFIX, TMAX )                                                                 \
static void expand_constant_##SUFFIX( T* b, ptrdiff_t s, size_t n, size_t left, size_t right, T lv, T rv ) { \
   /* ExpandBufferConstant, copy_buffer.cpp:360-379 */                                                     \
   for( size_t ii = 0; ii < left; ++ii ) { b[ -(ptrdiff_t)( ii + 1 ) * s ] = lv; }                        \
   for( size_t ii = 0; ii < right; ++ii ) { b[ (ptrdiff_t)( n + ii ) * s ] = rv; }                       \
}                                                                                                          \
static void expand_first_##SUFFIX( T* b, ptrdiff_t s, size_t n, size_t left, size_t right ) {             \
   /* ExpandBufferFirstOrder, copy_buffer.cpp:386-417 */                                                   \
   if( left > 0 ) {                                                                                        \
      double d0 = (double)b[ 0 ];                                                                          \
      double d1 = d0 / (double)( left + 1 );                                                               \
      for( size_t ii = 0; ii < left; ii++ ) { d0 -= d1; b[ -(ptrdiff_t)( ii + 1 ) * s ] = (T)d0; }          \
   }                                                                                                       \
   if( right > 0 ) {                                                                                       \
      double d0 = (double)b[ (ptrdiff_t)( n - 1 ) * s ];                                                   \
      double d1 = d0 / (double)( right + 1 );                                                              \
      for( size_t ii = 0; ii < right; ii++ ) { d0 -= d1; b[ (ptrdiff_t)( n + ii ) * s ] = (T)d0; }          \
   }                                                                                                       \
}                                                                                                          \
static void expand_second_##SUFFIX( T* b, ptrdiff_t s, size_t n, size_t left, size_t right ) {            \
   /* ExpandBufferSecondOrder, copy_buffer.cpp:423-458 */                                                  \
   if( left > 0 ) {                                                                                        \
      double bb = (double)left + 1.0;                                                                      \
      double d0 = (double)b[ 0 ];                                                                          \
      double f1 = (double)b[ s ];                                                                          \
      double d1 = ( bb - 1.0 ) / bb * d0 - bb / ( bb + 1.0 ) * f1;                                         \
      double d2 = -1.0 / bb * d0 + 1.0 / ( bb + 1.0 ) * f1;                                                \
      for( size_t ii = 1; ii <= left; ii++ ) {                                                             \
         double x = (double)ii;                                                                            \
         b[ -(ptrdiff_t)ii * s ] = (T)( d0 + x * d1 + x * x * d2 );                                        \
      }                                                                                                    \
   }                                                                                                       \
   if( right > 0 ) {                                                                                       \
      double bb = (double)right + 1.0;                                                                     \
      double d0 = (double)b[ (ptrdiff_t)( n - 1 ) * s ];                                                   \
      double f1 = (double)b[ (ptrdiff_t)( n - 2 ) * s ];                                                   \
      double d1 = ( bb - 1.0 ) / bb * d0 - bb / ( bb + 1.0 ) * f1;                                         \
      double d2 = -1.0 / bb * d0 + 1.0 / ( bb + 1.0 ) * f1;                                                \
      for( size_t ii = 1; ii <= right; ii++ ) {                                                            \
         double x = (double)ii;                                                                            \
         b[ (ptrdiff_t)( n - 1 + ii ) * s ] = (T)( d0 + x * d1 + x * x * d2 );                             \
      }                                                                                                    \
   }                                                                                                       \
}                                                                                                          \
static void expand_third_##SUFFIX( T* b, ptrdiff_t s, size_t n, size_t left, size_t right ) {             \
   /* ExpandBufferThirdOrder, copy_buffer.cpp:469-513 */                                                   \
   if( left > 0 ) {                                                                                        \
      double bb = (double)left + 1.0;                                                                      \
      double b12 = ( bb + 1 ) * ( bb + 1 );                                                                \
      double d0 = (double)b[ 0 ];                                                                          \
      double f1 = (double)b[ s ];                                                                          \
      double d1 = -( 2.0 * d0 ) / bb + d0 - ( bb * bb * f1 ) / b12;                                        \
      double d2 = ( 2.0 * bb * f1 ) / b12 - ( d0 * ( 2.0 * bb - 1.0 )) / ( bb * bb );                      \
      double d3 = d0 / ( bb * bb ) - f1 / b12;                                                             \
      for( size_t ii = 1; ii <= left; ii++ ) {                                                             \
         double x = (double)ii;                                                                            \
         b[ -(ptrdiff_t)ii * s ] = (T)( d0 + x * d1 + x * x * d2 + x * x * x * d3 );                       \
      }                                                                                                    \
   }                                                                                                       \
   if( right > 0 ) {                                                                                       \
      double bb = (double)right + 1.0;                                                                     \
      double b12 = ( bb + 1 ) * ( bb + 1 );                                                                \
      double d0 = (double)b[ (ptrdiff_t)( n - 1 ) * s ];                                                   \
      double f1 = (double)b[ (ptrdiff_t)( n - 2 ) * s ];                                                   \
      double d1 = -( 2.0 * d0 ) / bb + d0 - ( bb * bb * f1 ) / b12;                                        \
      double d2 = ( 2.0 * bb * f1 ) / b12 - ( d0 * ( 2.0 * bb - 1.0 )) / ( bb * bb );                      \
      double d3 = d0 / ( bb * bb ) - f1 / b12;                                                             \
      for( size_t ii = 1; ii <= right; ii++ ) {                                                            \
         double x = (double)ii;                                                                            \
         b[ (ptrdiff_t)( n - 1 + ii ) * s ] = (T)( d0 + x * d1 + x * x * d2 + x * x * x * d3 );            \
      }                                                                                                    \
   }                                                                                                       \
}                                                                                                          \
static void expand_mirror_##SUFFIX( T* b, ptrdiff_t s, size_t n, size_t left, size_t right, int asym ) {   \
   /* ExpandBufferMirror, copy_buffer.cpp:516-549: bounce between the two end samples */                  \
   ptrdiff_t last = (ptrdiff_t)n - 1;                                                                      \
   ptrdiff_t in = 0;                                                                                       \
   int sign = -1;                                                                                          \
   for( size_t ii = 0; ii < left; ii++ ) {                                                                 \
      in -= sign;                                                                                          \
      T v = b[ in * s ];                                                                                   \
      b[ -(ptrdiff_t)( ii + 1 ) * s ] = ( asym && sign < 0 ) ? -v : v;                                     \
      if( in == last || in == 0 ) { sign = -sign; }                                                        \
   }                                                                                                       \
   in = last;                                                                                              \
   sign = -1;                                                                                              \
   for( size_t ii = 0; ii < right; ii++ ) {                                                                \
      in += sign;                                                                                          \
      T v = b[ in * s ];                                                                                   \
      b[ ( last + 1 + (ptrdiff_t)ii ) * s ] = ( asym && sign < 0 ) ? -v : v;                               \
      if( in == last || in == 0 ) { sign = -sign; }                                                        \
   }                                                                                                       \
}                                                                                                          \
static void expand_antisym_##SUFFIX( T* b, ptrdiff_t s, size_t n, size_t left, size_t right ) {            \
   /* ExpandBufferAntiSymReflect, copy_buffer.cpp:552-589 */                                               \
   ptrdiff_t last = (ptrdiff_t)n - 1;                                                                      \
   ptrdiff_t in = 0, out = 0;                                                                              \
   int sign = -1;                                                                                          \
   double offset = (double)b[ out * s ] - sign * (double)b[ in * s ];                                      \
   for( size_t ii = 0; ii < left; ii++ ) {                                                                 \
      in -= sign;                                                                                          \
      out -= 1;                                                                                            \
      b[ out * s ] = (T)( offset + sign * (double)b[ in * s ] );                                           \
      if( in == last || in == 0 ) {                                                                        \
         sign = -sign;                                                                                     \
         offset = (double)b[ out * s ] - sign * (double)b[ in * s ];                                       \
      }                                                                                                    \
   }                                                                                                       \
   in = last;                                                                                              \
   out = last;                                                                                             \
   sign = -1;                                                                                              \
   offset = (double)b[ out * s ] - sign * (double)b[ in * s ];                                             \
   for( size_t ii = 0; ii < right; ii++ ) {                                                                \
      in += sign;                                                                                          \
      out += 1;                                                                                            \
      b[ out * s ] = (T)( offset + sign * (double)b[ in * s ] );                                           \
      if( in == last || in == 0 ) {                                                                        \
         sign = -sign;                                                                                     \
         offset = (double)b[ out * s ] - sign * (double)b[ in * s ];                                       \
      }                                                                                                    \
   }                                                                                                       \
}                                                                                                          \
static void expand_periodic_##SUFFIX( T* b, ptrdiff_t s, size_t n, size_t left, size_t right, int asym ) { \
   /* ExpandBufferPeriodic, copy_buffer.cpp:592-629 */                                                     \
   ptrdiff_t last = (ptrdiff_t)n - 1;                                                                      \
   ptrdiff_t in = last;                                                                                    \
   int sign = -1;                                                                                          \
   for( size_t ii = 0; ii < left; ii++ ) {                                                                 \
      T v = b[ in * s ];                                                                                   \
      b[ -(ptrdiff_t)( ii + 1 ) * s ] = ( asym && sign < 0 ) ? -v : v;                                     \
      if( in == 0 ) { in = last; sign = -sign; } else { in -= 1; }                                         \
   }                                                                                                       \
   in = 0;                                                                                                 \
   sign = -1;                                                                                              \
   for( size_t ii = 0; ii < right; ii++ ) {                                                                \
      T v = b[ in * s ];                                                                                   \
      b[ ( last + 1 + (ptrdiff_t)ii ) * s ] = ( asym && sign < 0 ) ? -v : v;                               \
      if( in == last ) { in = 0; sign = -sign; } else { in += 1; }                                         \
   }                                                                                                       \
}                                                                                                          \
int or_expand_buffer_##SUFFIX( T* b, ptrdiff_t s, size_t n, size_t left, size_t right, int bc ) {          \
   /* ExpandBufferFromTo, copy_buffer.cpp:632-747 (float buffers: saturated_inv is negation) */            \
   if( left == 0 && right == 0 ) { return OR_OK; }                                                         \
   if( n == 0 ) { return OR_ERR_ARG; }                                                                     \
   switch( bc ) {                                                                                          \
      case OR_BC_SYMMETRIC_MIRROR:                                                                         \
         if( n == 1 ) { expand_constant_##SUFFIX( b, s, n, left, right, b[ 0 ], b[ 0 ] ); }                \
         else { expand_mirror_##SUFFIX( b, s, n, left, right, 0 ); }                                       \
         return OR_OK;                                                                                     \
      case OR_BC_ASYMMETRIC_MIRROR:                                                                        \
         if( n == 1 ) { expand_constant_##SUFFIX( b, s, n, left, right, -b[ 0 ], -b[ 0 ] ); }              \
         else { expand_mirror_##SUFFIX( b, s, n, left, right, 1 ); }                                       \
         return OR_OK;                                                                                     \
      case OR_BC_ANTISYMMETRIC_REFLECT:                                                                    \
         if( n == 1 ) { expand_constant_##SUFFIX( b, s, n, left, right, b[ 0 ], b[ 0 ] ); }                \
         else { expand_antisym_##SUFFIX( b, s, n, left, right ); }                                         \
         return OR_OK;                                                                                     \
      case OR_BC_PERIODIC:                                                                                 \
         if( n == 1 ) { expand_constant_##SUFFIX( b, s, n, left, right, b[ 0 ], b[ 0 ] ); }                \
         else { expand_periodic_##SUFFIX( b, s, n, left, right, 0 ); }                                     \
         return OR_OK;                                                                                     \
      case OR_BC_ASYMMETRIC_PERIODIC:                                                                      \
         if( n == 1 ) { expand_constant_##SUFFIX( b, s, n, left, right, -b[ 0 ], -b[ 0 ] ); }              \
         else { expand_periodic_##SUFFIX( b, s, n, left, right, 1 ); }                                     \
         return OR_OK;                                                                                     \
      case OR_BC_ADD_ZEROS:                                                                                \
         expand_constant_##SUFFIX( b, s, n, left, right, (T)0, (T)0 );                                     \
         return OR_OK;                                                                                     \
      case OR_BC_ADD_MAX_VALUE:                                                                            \
         expand_constant_##SUFFIX( b, s, n, left, right, TMAX, TMAX );                                     \
         return OR_OK;                                                                                     \
      case OR_BC_ADD_MIN_VALUE:                                                                            \
         expand_constant_##SUFFIX( b, s, n, left, right, -TMAX, -TMAX );                                   \
         return OR_OK;                                                                                     \
      case OR_BC_THIRD_ORDER_EXTRAPOLATE:                                                                  \
         if( n > 1 ) { expand_third_##SUFFIX( b, s, n, left, right ); return OR_OK; }                      \
         /* fallthrough */                                                                                 \
      case OR_BC_SECOND_ORDER_EXTRAPOLATE:                                                                 \
         if( n > 1 ) { expand_second_##SUFFIX( b, s, n, left, right ); return OR_OK; }                     \
         /* fallthrough */                                                                                 \
      case OR_BC_FIRST_ORDER_EXTRAPOLATE:                                                                  \
         expand_first_##SUFFIX( b, s, n, left, right );                                                    \
         return OR_OK;                                                                                     \
      case OR_BC_ZERO_ORDER_EXTRAPOLATE:                                                                   \
         expand_constant_##SUFFIX( b, s, n, left, right, b[ 0 ], b[ (ptrdiff_t)( n - 1 ) * s ] );          \
         return OR_OK;                                                                                     \
      default:                                                                                             \
         return OR_ERR_BC;                                                                                 \
   }                                                                                                       \
}

OR_DEFINE_EXPAND( float, f32, FLT_MAX )
OR_DEFINE_EXPAND( double, f64, DBL_MAX )

/* ------------------------------------------------------------------------------------------ */
/* Sample access with DIPlib's conversions (clamp_cast, include/diplib/library/clamp_cast.h)   */
/* ------------------------------------------------------------------------------------------ */

static size_t dtype_size( int dt ) {
   switch( dt ) {
      case OR_BIN: case OR_UINT8: case OR_SINT8: return 1;
      case OR_UINT16: case OR_SINT16: return 2;
      case OR_UINT32: case OR_SINT32: case OR_SFLOAT: return 4;
      case OR_UINT64: case OR_SINT64: case OR_DFLOAT: return 8;
      default: return 0;
   }
}

/* The value of a sample as a double.  Exact for every type except 64-bit integers above 2^53,
 * where the reference's static_cast< dfloat > rounds identically. */
static double get_sample( void const* p, int dt, ptrdiff_t idx ) {
   switch( dt ) {
      case OR_BIN: return ( (uint8_t const*)p )[ idx ] ? 1.0 : 0.0;
      case OR_UINT8: return ( (uint8_t const*)p )[ idx ];
      case OR_UINT16: return ( (uint16_t const*)p )[ idx ];
      case OR_UINT32: return ( (uint32_t const*)p )[ idx ];
      case OR_UINT64: return (double)( (uint64_t const*)p )[ idx ];
      case OR_SINT8: return ( (int8_t const*)p )[ idx ];
      case OR_SINT16: return ( (int16_t const*)p )[ idx ];
      case OR_SINT32: return ( (int32_t const*)p )[ idx ];
      case OR_SINT64: return (double)( (int64_t const*)p )[ idx ];
      case OR_SFLOAT: return ( (float const*)p )[ idx ];
      case OR_DFLOAT: return ( (double const*)p )[ idx ];
      default: return 0.0;
   }
}

/* clamp_cast< outT >( v ): clamp to the target range, then static_cast (truncation toward 0). */
#define OR_CLAMP( v, lo, hi ) ( ( v ) < ( lo ) ? ( lo ) : ( ( v ) > ( hi ) ? ( hi ) : ( v )))
static void put_sample( void* p, int dt, ptrdiff_t idx, double v ) {
   switch( dt ) {
      case OR_BIN: ( (uint8_t*)p )[ idx ] = ( v != 0.0 ); break;
      case OR_UINT8: ( (uint8_t*)p )[ idx ] = (uint8_t)OR_CLAMP( v, 0.0, 255.0 ); break;
      case OR_UINT16: ( (uint16_t*)p )[ idx ] = (uint16_t)OR_CLAMP( v, 0.0, 65535.0 ); break;
      case OR_UINT32: ( (uint32_t*)p )[ idx ] = (uint32_t)OR_CLAMP( v, 0.0, 4294967295.0 ); break;
      case OR_UINT64: ( (uint64_t*)p )[ idx ] = (uint64_t)OR_CLAMP( v, 0.0, 18446744073709549568.0 ); break;
      case OR_SINT8: ( (int8_t*)p )[ idx ] = (int8_t)OR_CLAMP( v, -128.0, 127.0 ); break;
      case OR_SINT16: ( (int16_t*)p )[ idx ] = (int16_t)OR_CLAMP( v, -32768.0, 32767.0 ); break;
      case OR_SINT32: ( (int32_t*)p )[ idx ] = (int32_t)OR_CLAMP( v, -2147483648.0, 2147483647.0 ); break;
      case OR_SINT64: ( (int64_t*)p )[ idx ] = (int64_t)OR_CLAMP( v, -9223372036854775808.0, 9223372036854774784.0 ); break;
      case OR_SFLOAT: ( (float*)p )[ idx ] = (float)v; break;
      case OR_DFLOAT: ( (double*)p )[ idx ] = v; break;
      default: break;
   }
}

/* DataType::SuggestFlex, src/library/datatype.cpp:109-124 (real types only). */
int or_suggest_flex( int dt ) {
   switch( dt ) {
      case OR_UINT32: case OR_SINT32: case OR_UINT64: case OR_SINT64: case OR_DFLOAT:
         return OR_DFLOAT;
      default:
         return OR_SFLOAT;
   }
}

/* ------------------------------------------------------------------------------------------ */
/* The line filter: SeparableConvolutionLineFilter::Filter, src/linear/convolution.cpp:184-241 */
/* EVEN and ODD cases, with the filter reversed as InternOneDimensionalFilter does (:76-156):  */
/* f[0] is the centre tap, f[k] the tap at distance k.                                         */
/* ------------------------------------------------------------------------------------------ */

static void line_filter_f32( float const* in, float* out, size_t length, float const* f, size_t dataSize, int odd ) {
   for( size_t ii = 0; ii < length; ++ii ) {
      float const* c = in + ii;
      float sum = f[ 0 ] * c[ 0 ];
      for( size_t k = 1; k < dataSize; ++k ) {
         sum += f[ k ] * ( odd ? ( c[ k ] - c[ -(ptrdiff_t)k ] ) : ( c[ k ] + c[ -(ptrdiff_t)k ] ));
      }
      out[ ii ] = sum;
   }
}

static void line_filter_f64( double const* in, double* out, size_t length, double const* f, size_t dataSize, int odd ) {
   for( size_t ii = 0; ii < length; ++ii ) {
      double const* c = in + ii;
      double sum = f[ 0 ] * c[ 0 ];
      for( size_t k = 1; k < dataSize; ++k ) {
         sum += f[ k ] * ( odd ? ( c[ k ] - c[ -(ptrdiff_t)k ] ) : ( c[ k ] + c[ -(ptrdiff_t)k ] ));
      }
      out[ ii ] = sum;
   }
}

/* ------------------------------------------------------------------------------------------ */
/* GaussFIR -> SeparableConvolution -> Framework::Separable                                   */
/* ------------------------------------------------------------------------------------------ */

#define OR_MAX_DIMS 16
#define OR_MAX_FILTER 4096

/* dip::SeparableConvolution (src/linear/convolution.cpp:319-421) for real EVEN / ODD filters given as
 * half kernels with the centre FIRST (the reversed storage of InternOneDimensionalFilter), driven by
 * Framework::Separable (src/library/framework_separable.cpp:35-431).  `taps[d]` NULL (or len 0) leaves
 * axis d unprocessed.  Taps are rounded to float when the buffer type is sfloat (convolution.cpp:149-150). */
int or_separable_fir( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                      void* out, int out_dtype, int64_t const* out_strides,
                      double const* const* taps, int const* lens, int const* odd, int const* bcs ) {
   if( ndims < 1 || ndims > OR_MAX_DIMS || dtype_size( in_dtype ) == 0 || dtype_size( out_dtype ) == 0 ) {
      return OR_ERR_ARG;
   }
   int buf_type = or_suggest_flex( in_dtype );
   int buf_double = ( buf_type == OR_DFLOAT );
   int process[ OR_MAX_DIMS ];
   size_t half[ OR_MAX_DIMS ];
   size_t npix = 1;
   for( int d = 0; d < ndims; ++d ) {
      npix *= (size_t)sizes[ d ];
      process[ d ] = taps && taps[ d ] && lens[ d ] > 0 && sizes[ d ] > 1;
      half[ d ] = process[ d ] ? (size_t)lens[ d ] - 1 : 0;
      if( process[ d ] && lens[ d ] == 1 && taps[ d ][ 0 ] == 1.0 ) { process[ d ] = 0; }
      if( process[ d ] && ( bcs[ d ] < 0 || bcs[ d ] >= OR_BC_ALREADY_EXPANDED )) { return OR_ERR_BC; }
   }

   /* Framework::Separable: processing order by input stride, stable insertion sort
    * (framework_separable.cpp:146-165; sortIndices, dimension_array.h:907-924). */
   int order[ OR_MAX_DIMS ];
   int nproc = 0;
   for( int d = 0; d < ndims; ++d ) {
      if( process[ d ] ) { order[ nproc++ ] = d; }
   }
   for( int ii = 1; ii < nproc; ++ii ) {
      int elem = order[ ii ];
      int jj = ii;
      while( jj > 0 && in_strides[ order[ jj - 1 ] ] > in_strides[ elem ] ) {
         order[ jj ] = order[ jj - 1 ];
         --jj;
      }
      order[ jj ] = elem;
   }
   if( nproc == 0 ) {
      /* output.Copy( input ) with conversion (framework_separable.cpp:155-159). */
      int64_t coord[ OR_MAX_DIMS ] = { 0 };
      for( size_t p = 0; p < npix; ++p ) {
         ptrdiff_t io = 0, oo = 0;
         for( int d = 0; d < ndims; ++d ) { io += coord[ d ] * in_strides[ d ]; oo += coord[ d ] * out_strides[ d ]; }
         put_sample( out, out_dtype, oo, get_sample( in, in_dtype, io ));
         for( int d = 0; d < ndims; ++d ) { if( ++coord[ d ] < sizes[ d ] ) { break; } coord[ d ] = 0; }
      }
      return OR_OK;
   }

   /* in -> output -> output ... (or via an intermediate of the buffer type when the output type
    * differs, framework_separable.cpp:181-206). */
   int use_intermediate = ( out_dtype != buf_type );
   void* inter = NULL;
   int64_t inter_strides[ OR_MAX_DIMS ];
   if( use_intermediate ) {
      inter = malloc( npix * dtype_size( buf_type ));
      int64_t s = 1;
      for( int d = 0; d < ndims; ++d ) { inter_strides[ d ] = s; s *= sizes[ d ]; }
   }
   size_t maxlen = 0, maxhalf = 0;
   for( int ii = 0; ii < nproc; ++ii ) {
      if( (size_t)sizes[ order[ ii ] ] > maxlen ) { maxlen = (size_t)sizes[ order[ ii ] ]; }
      if( half[ order[ ii ] ] > maxhalf ) { maxhalf = half[ order[ ii ] ]; }
   }
   size_t esz = buf_double ? 8 : 4;
   char* inbuf = (char*)malloc( esz * ( maxlen + 2 * maxhalf ));
   char* outbuf = (char*)malloc( esz * maxlen );
   float* ftaps = (float*)malloc( sizeof( float ) * ( maxhalf + 1 ));

   void const* src = in;
   int src_type = in_dtype;
   int64_t const* src_strides = in_strides;
   for( int rep = 0; rep < nproc; ++rep ) {
      int pd = order[ rep ];
      int last = ( rep == nproc - 1 );
      void* dst = ( last || !use_intermediate ) ? out : inter;
      int dst_type = ( last || !use_intermediate ) ? out_dtype : buf_type;
      int64_t const* dst_strides = ( last || !use_intermediate ) ? out_strides : inter_strides;
      size_t n = (size_t)sizes[ pd ];
      size_t h = half[ pd ];
      size_t nlines = npix / n;
      for( size_t k = 0; k <= h; ++k ) { ftaps[ k ] = (float)taps[ pd ][ k ]; }
      int64_t coord[ OR_MAX_DIMS ] = { 0 };
      for( size_t line = 0; line < nlines; ++line ) {
         ptrdiff_t so = 0, dof = 0;
         for( int d = 0; d < ndims; ++d ) { so += coord[ d ] * src_strides[ d ]; dof += coord[ d ] * dst_strides[ d ]; }
         /* CopyBuffer into the line buffer (framework_separable.cpp:357-368), ExpandBuffer
          * (:369-380), filter (:389), write back (:384-417). */
         if( buf_double ) {
            double* b = (double*)inbuf + h;
            double* o = (double*)outbuf;
            for( size_t i = 0; i < n; ++i ) { b[ i ] = get_sample( src, src_type, so + (ptrdiff_t)i * src_strides[ pd ] ); }
            or_expand_buffer_f64( b, 1, n, h, h, bcs[ pd ] );
            line_filter_f64( b, o, n, taps[ pd ], h + 1, odd[ pd ] );
            for( size_t i = 0; i < n; ++i ) { put_sample( dst, dst_type, dof + (ptrdiff_t)i * dst_strides[ pd ], o[ i ] ); }
         } else {
            float* b = (float*)inbuf + h;
            float* o = (float*)outbuf;
            for( size_t i = 0; i < n; ++i ) { b[ i ] = (float)get_sample( src, src_type, so + (ptrdiff_t)i * src_strides[ pd ] ); }
            or_expand_buffer_f32( b, 1, n, h, h, bcs[ pd ] );
            line_filter_f32( b, o, n, ftaps, h + 1, odd[ pd ] );
            for( size_t i = 0; i < n; ++i ) { put_sample( dst, dst_type, dof + (ptrdiff_t)i * dst_strides[ pd ], (double)o[ i ] ); }
         }
         for( int d = 0; d < ndims; ++d ) {
            if( d == pd ) { continue; }
            if( ++coord[ d ] < sizes[ d ] ) { break; }
            coord[ d ] = 0;
         }
      }
      src = dst;
      src_type = dst_type;
      src_strides = dst_strides;
   }
   free( inbuf );
   free( outbuf );
   free( ftaps );
   free( inter );
   return OR_OK;
}

int or_gauss_fir( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                  void* out, int out_dtype, int64_t const* out_strides,
                  double const* sigmas, unsigned const* orders, int const* bcs, double truncation ) {
   if( ndims < 1 || ndims > OR_MAX_DIMS || dtype_size( in_dtype ) == 0 || dtype_size( out_dtype ) == 0 ) {
      return OR_ERR_ARG;
   }
   /* GaussFIR: weight type (gauss.cpp:254) and per-dimension filters (:255-284). */
   int weights_double = ( in_dtype == OR_DFLOAT );
   double* taps[ OR_MAX_DIMS ] = { 0 };  /* reversed half kernel, f[0] = centre */
   int lens[ OR_MAX_DIMS ] = { 0 };
   int odd[ OR_MAX_DIMS ] = { 0 };
   int status = OR_OK;
   for( int d = 0; d < ndims; ++d ) {
      if( !(( sigmas[ d ] > 0.0 ) && ( sizes[ d ] > 1 ))) { continue; }
      if( orders[ d ] > 3 ) { status = OR_ERR_ORDER; goto done; }
      if( bcs[ d ] < 0 || bcs[ d ] >= OR_BC_ALREADY_EXPANDED ) { status = OR_ERR_BC; goto done; }
      int len = or_make_half_gaussian( sigmas[ d ], orders[ d ], truncation, weights_double, NULL, 0 );
      double* h = (double*)malloc( sizeof( double ) * (size_t)len );
      or_make_half_gaussian( sigmas[ d ], orders[ d ], truncation, weights_double, h, len );
      taps[ d ] = (double*)malloc( sizeof( double ) * (size_t)len );
      for( int k = 0; k < len; ++k ) { taps[ d ][ k ] = h[ len - 1 - k ]; }   /* CopyReverseData */
      free( h );
      lens[ d ] = len;
      odd[ d ] = ( orders[ d ] & 1 ) != 0;
   }
   status = or_separable_fir( in, in_dtype, ndims, sizes, in_strides, out, out_dtype, out_strides,
                              (double const* const*)taps, lens, odd, bcs );
done:
   for( int d = 0; d < ndims; ++d ) { free( taps[ d ] ); }
   return status;
}


/* ------------------------------------------------------------------------------------------ */
/* General real filters and the rectangular uniform filter (next to the Gaussian path):        */
/* dip::SeparableConvolution with dip::OneDimensionalFilter of any symmetry                    */
/* (src/linear/convolution.cpp:67-162 interning, :175-302 line filter, :319-421 driver) and    */
/* dip::Uniform with a rectangular kernel (src/linear/uniform.cpp:33-86).                      */
/* ------------------------------------------------------------------------------------------ */

/* One real filter as InternOneDimensionalFilter keeps it: f = the data reversed, `size` the full
 * length (symmetry expanded), `origin` the reversed origin. */
typedef struct {
   double f[ OR_MAX_FILTER ];
   size_t dataSize, size, origin;
   int symmetry;
} or_ifilter;

static int intern_filter( double const* data, size_t n, long origin, int symmetry, or_ifilter* out ) {
   if( n > OR_MAX_FILTER ) { return OR_ERR_ARG; }
   out->dataSize = n;
   out->size = n;
   out->symmetry = symmetry;
   if( n == 0 ) { out->origin = 0; return OR_OK; }
   switch( symmetry ) {
      case OR_SYM_GENERAL: break;
      case OR_SYM_EVEN: case OR_SYM_ODD: out->size = 2 * n - 1; break;
      case OR_SYM_D_EVEN: case OR_SYM_D_ODD: out->size = 2 * n; break;
      default: return OR_ERR_ARG;
   }
   size_t o = origin < 0 ? out->size / 2 : (size_t)origin;
   if( o >= out->size ) { return OR_ERR_ARG; }
   for( size_t i = 0; i < n; ++i ) { out->f[ i ] = data[ n - 1 - i ]; }    /* CopyReverseData */
   out->origin = out->size - o - 1;
   return OR_OK;
}

/* The line filter of convolution.cpp:184-302 for real data; `in` is the first sample of the line
 * (the buffer is extended by the border on both sides). */
#define DEFINE_GENERAL_LINE( SUFFIX, T )                                                              \
static void general_line_##SUFFIX( T const* in, T* out, size_t length, or_ifilter const* F, T const* f ) { \
   size_t const ds = F->dataSize;                                                                        \
   in -= F->origin;                                                                                      \
   switch( F->symmetry ) {                                                                               \
      case OR_SYM_GENERAL:                                                                               \
         for( size_t ii = 0; ii < length; ++ii, ++in ) {                                                 \
            T sum = 0;                                                                                   \
            for( size_t k = 0; k < ds; ++k ) { sum += f[ k ] * in[ k ]; }                                \
            out[ ii ] = sum;                                                                             \
         }                                                                                               \
         break;                                                                                          \
      case OR_SYM_EVEN: case OR_SYM_ODD: {                                                               \
         int const odd = F->symmetry == OR_SYM_ODD;                                                      \
         T const* c = in + ds - 1;                                                                       \
         for( size_t ii = 0; ii < length; ++ii, ++c ) {                                                  \
            T sum = f[ 0 ] * c[ 0 ];                                                                     \
            for( size_t k = 1; k < ds; ++k ) {                                                           \
               sum += f[ k ] * ( odd ? ( c[ k ] - c[ -(ptrdiff_t)k ] ) : ( c[ k ] + c[ -(ptrdiff_t)k ] )); \
            }                                                                                            \
            out[ ii ] = sum;                                                                             \
         }                                                                                               \
         break;                                                                                          \
      }                                                                                                  \
      default: {   /* D_EVEN, D_ODD */                                                                   \
         int const odd = F->symmetry == OR_SYM_D_ODD;                                                    \
         T const* r = in + ds - 1;                                                                       \
         for( size_t ii = 0; ii < length; ++ii, ++r ) {                                                  \
            T sum = 0;                                                                                   \
            for( size_t k = 0; k < ds; ++k ) {                                                           \
               sum += f[ k ] * ( odd ? ( r[ k ] - r[ -1 - (ptrdiff_t)k ] ) : ( r[ k ] + r[ -1 - (ptrdiff_t)k ] )); \
            }                                                                                            \
            out[ ii ] = sum;                                                                             \
         }                                                                                               \
         break;                                                                                          \
      }                                                                                                  \
   }                                                                                                     \
}                                                                                                        \
/* RectangularUniformLineFilter::Filter (uniform.cpp:41-62): a running sum. */                          \
static void uniform_line_##SUFFIX( T const* in, T* out, size_t length, size_t filterSize ) {             \
   T const norm = (T)1 / (T)filterSize;                                                                  \
   T const* left = in - (ptrdiff_t)( filterSize / 2 );                                                   \
   T const* right = in + (ptrdiff_t)(( filterSize + 1 ) / 2 );                                           \
   T sum = 0;                                                                                            \
   for( T const* p = left; p != right; ++p ) { sum += *p; }                                              \
   out[ 0 ] = sum * norm;                                                                                \
   for( size_t ii = 1; ii < length; ++ii ) {                                                             \
      sum -= *left;                                                                                      \
      sum += *right;                                                                                     \
      ++left;                                                                                            \
      ++right;                                                                                           \
      out[ ii ] = sum * norm;                                                                            \
   }                                                                                                     \
}

DEFINE_GENERAL_LINE( f32, float )
DEFINE_GENERAL_LINE( f64, double )

typedef struct or_iir_params or_iir_params;
static void iir_line( double const* in, double* out, size_t length, or_iir_params const* P, double* p1 );

/* Framework::Separable (framework_separable.cpp:35-431) around a per-axis line filter: kind 0 the
 * interned filters `F`, kind 1 the rectangular uniform filter of `usize[d]` samples, kind 2 the
 * recursive Gaussian of `I[d]` (a dfloat buffer whatever the input type, the filter writing the
 * output buffer's border too: gaussiir.cpp:770-787). */
static int separable_driver( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                             void* out, int out_dtype, int64_t const* out_strides, int const* process_in,
                             size_t const* border, int const* bcs, int kind, or_ifilter const* const* F,
                             size_t const* usize, or_iir_params const* const* I ) {
   if( ndims < 1 || ndims > OR_MAX_DIMS || dtype_size( in_dtype ) == 0 || dtype_size( out_dtype ) == 0 ) {
      return OR_ERR_ARG;
   }
   int buf_type = kind == 2 ? OR_DFLOAT : or_suggest_flex( in_dtype );
   int buf_double = ( buf_type == OR_DFLOAT );
   int process[ OR_MAX_DIMS ];
   size_t npix = 1;
   for( int d = 0; d < ndims; ++d ) {
      npix *= (size_t)sizes[ d ];
      process[ d ] = process_in[ d ] && sizes[ d ] > 1;
      if( process[ d ] && ( bcs[ d ] < 0 || bcs[ d ] >= OR_BC_ALREADY_EXPANDED )) { return OR_ERR_BC; }
   }
   int order[ OR_MAX_DIMS ];
   int nproc = 0;
   for( int d = 0; d < ndims; ++d ) {
      if( process[ d ] ) { order[ nproc++ ] = d; }
   }
   for( int ii = 1; ii < nproc; ++ii ) {
      int elem = order[ ii ];
      int jj = ii;
      while( jj > 0 && in_strides[ order[ jj - 1 ] ] > in_strides[ elem ] ) {
         order[ jj ] = order[ jj - 1 ];
         --jj;
      }
      order[ jj ] = elem;
   }
   if( nproc == 0 ) {
      int64_t coord[ OR_MAX_DIMS ] = { 0 };
      for( size_t p = 0; p < npix; ++p ) {
         ptrdiff_t io = 0, oo = 0;
         for( int d = 0; d < ndims; ++d ) { io += coord[ d ] * in_strides[ d ]; oo += coord[ d ] * out_strides[ d ]; }
         put_sample( out, out_dtype, oo, get_sample( in, in_dtype, io ));
         for( int d = 0; d < ndims; ++d ) { if( ++coord[ d ] < sizes[ d ] ) { break; } coord[ d ] = 0; }
      }
      return OR_OK;
   }
   int use_intermediate = ( out_dtype != buf_type );
   void* inter = NULL;
   int64_t inter_strides[ OR_MAX_DIMS ];
   if( use_intermediate ) {
      inter = malloc( npix * dtype_size( buf_type ));
      int64_t s = 1;
      for( int d = 0; d < ndims; ++d ) { inter_strides[ d ] = s; s *= sizes[ d ]; }
   }
   size_t maxlen = 0, maxb = 0;
   for( int ii = 0; ii < nproc; ++ii ) {
      if( (size_t)sizes[ order[ ii ] ] > maxlen ) { maxlen = (size_t)sizes[ order[ ii ] ]; }
      if( border[ order[ ii ] ] > maxb ) { maxb = border[ order[ ii ] ]; }
   }
   size_t esz = buf_double ? 8 : 4;
   char* inbuf = (char*)malloc( esz * ( maxlen + 2 * maxb ));
   char* outbuf = (char*)malloc( esz * ( maxlen + 2 * maxb ));
   double* scan = kind == 2 ? (double*)malloc( sizeof( double ) * ( maxlen + 2 * maxb )) : NULL;
   void const* src = in;
   int src_type = in_dtype;
   int64_t const* src_strides = in_strides;
   for( int rep = 0; rep < nproc; ++rep ) {
      int pd = order[ rep ];
      int last = ( rep == nproc - 1 );
      void* dst = ( last || !use_intermediate ) ? out : inter;
      int dst_type = ( last || !use_intermediate ) ? out_dtype : buf_type;
      int64_t const* dst_strides = ( last || !use_intermediate ) ? out_strides : inter_strides;
      size_t n = (size_t)sizes[ pd ];
      size_t b = border[ pd ];
      size_t nlines = npix / n;
      float ff[ OR_MAX_FILTER ];
      if( kind == 0 ) { for( size_t k = 0; k < F[ pd ]->dataSize; ++k ) { ff[ k ] = (float)F[ pd ]->f[ k ]; } }
      int64_t coord[ OR_MAX_DIMS ] = { 0 };
      for( size_t line = 0; line < nlines; ++line ) {
         ptrdiff_t so = 0, dof = 0;
         for( int d = 0; d < ndims; ++d ) { so += coord[ d ] * src_strides[ d ]; dof += coord[ d ] * dst_strides[ d ]; }
         if( buf_double ) {
            double* bb = (double*)inbuf + b;
            double* o = (double*)outbuf;
            for( size_t i = 0; i < n; ++i ) { bb[ i ] = get_sample( src, src_type, so + (ptrdiff_t)i * src_strides[ pd ] ); }
            or_expand_buffer_f64( bb, 1, n, b, b, bcs[ pd ] );
            if( kind == 0 ) { general_line_f64( bb, o, n, F[ pd ], F[ pd ]->f ); }
            else if( kind == 1 ) { uniform_line_f64( bb, o, n, usize[ pd ] ); }
            else { iir_line( bb - b, o, n + 2 * b, I[ pd ], scan ); o += b; }
            for( size_t i = 0; i < n; ++i ) { put_sample( dst, dst_type, dof + (ptrdiff_t)i * dst_strides[ pd ], o[ i ] ); }
         } else {
            float* bb = (float*)inbuf + b;
            float* o = (float*)outbuf;
            for( size_t i = 0; i < n; ++i ) { bb[ i ] = (float)get_sample( src, src_type, so + (ptrdiff_t)i * src_strides[ pd ] ); }
            or_expand_buffer_f32( bb, 1, n, b, b, bcs[ pd ] );
            if( kind == 0 ) { general_line_f32( bb, o, n, F[ pd ], ff ); } else { uniform_line_f32( bb, o, n, usize[ pd ] ); }
            for( size_t i = 0; i < n; ++i ) { put_sample( dst, dst_type, dof + (ptrdiff_t)i * dst_strides[ pd ], (double)o[ i ] ); }
         }
         for( int d = 0; d < ndims; ++d ) {
            if( d == pd ) { continue; }
            if( ++coord[ d ] < sizes[ d ] ) { break; }
            coord[ d ] = 0;
         }
      }
      src = dst;
      src_type = dst_type;
      src_strides = dst_strides;
   }
   free( inbuf );
   free( outbuf );
   free( inter );
   free( scan );
   return OR_OK;
}

int or_separable_convolution( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                              void* out, int out_dtype, int64_t const* out_strides, int nfilters,
                              double const* const* data, int const* lens, long const* origins, int const* symmetries,
                              int const* bcs, int const* process ) {
   if( ndims < 1 || ndims > OR_MAX_DIMS || ( nfilters != 1 && nfilters != ndims )) { return OR_ERR_ARG; }
   or_ifilter* fs = (or_ifilter*)calloc( (size_t)nfilters, sizeof( or_ifilter ));
   or_ifilter const* F[ OR_MAX_DIMS ];
   size_t border[ OR_MAX_DIMS ];
   int proc[ OR_MAX_DIMS ];
   int st = OR_OK;
   for( int i = 0; i < nfilters && st == OR_OK; ++i ) {
      st = intern_filter( data[ i ], (size_t)lens[ i ], origins[ i ], symmetries[ i ], &fs[ i ] );
   }
   if( st != OR_OK ) { free( fs ); return st; }
   for( int d = 0; d < ndims; ++d ) {
      or_ifilter const* f = &fs[ nfilters == 1 ? 0 : d ];
      F[ d ] = f;
      size_t b = f->origin;
      border[ d ] = f->size == 0 ? 0 : ( b > f->size - b - 1 ? b : f->size - b - 1 );
      proc[ d ] = process ? process[ d ] : 1;
      /* IsMeaninglessFilter (convolution.cpp:304-314): size 0, or a single unit tap (compared in the
       * buffer precision). */
      int meaningless = f->size == 0 || ( f->size == 1 && ( or_suggest_flex( in_dtype ) == OR_DFLOAT
                                                            ? f->f[ 0 ] == 1.0 : (float)f->f[ 0 ] == 1.0f ));
      if( meaningless ) { proc[ d ] = 0; }
   }
   st = separable_driver( in, in_dtype, ndims, sizes, in_strides, out, out_dtype, out_strides, proc, border, bcs, 0, F, NULL, NULL );
   free( fs );
   return st;
}

int or_uniform_rect( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                     void* out, int out_dtype, int64_t const* out_strides, int64_t const* filter_sizes, int const* bcs ) {
   if( ndims < 1 || ndims > OR_MAX_DIMS ) { return OR_ERR_ARG; }
   int proc[ OR_MAX_DIMS ];
   size_t border[ OR_MAX_DIMS ], usize[ OR_MAX_DIMS ];
   for( int d = 0; d < ndims; ++d ) {
      proc[ d ] = filter_sizes[ d ] > 1 && sizes[ d ] > 1;
      usize[ d ] = proc[ d ] ? (size_t)filter_sizes[ d ] : 1;
      border[ d ] = proc[ d ] ? usize[ d ] / 2 : 0;
   }
   return separable_driver( in, in_dtype, ndims, sizes, in_strides, out, out_dtype, out_strides, proc, border, bcs, 1, NULL, usize, NULL );
}

/* ------------------------------------------------------------------------------------------ */
/* dip::GaussIIR (src/linear/gaussiir.cpp)                                                     */
/* ------------------------------------------------------------------------------------------ */

#define OR_IIR_MAX 6

typedef struct { double re, im; } or_cplx;

static or_cplx cmul( or_cplx a, or_cplx b ) { or_cplx r = { a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re }; return r; }
static or_cplx cadd( or_cplx a, or_cplx b ) { or_cplx r = { a.re + b.re, a.im + b.im }; return r; }

/* GaussIIRParams, gaussiir.cpp:38-48. */
struct or_iir_params {
   size_t border;
   size_t num[ 6 ], den[ 6 ];                      /* iir_order_num, iir_order_den */
   double a1[ OR_IIR_MAX ], a2[ OR_IIR_MAX ], b1[ OR_IIR_MAX ], b2[ OR_IIR_MAX ];
   double cc;
};

/* FillPoleCoefficients, gaussiir.cpp:84-211: pp[1..nn], pp[0].re = nn; *fb set to 1 when the
 * forward-backward design is used. */
static void iir_fill_poles( size_t nn, or_cplx* pp, unsigned order, int* fb ) {
   static double const dtf5[ 3 ][ 10 ] = {
      { 0.85991, 1.45235, 0.85991, -1.45235, 1.60953, 0.83009, 1.60953, -0.83009, 1.87040, 0.0 },
      { 0.70237, 1.38717, 0.70237, -1.38717, 1.43280, 0.77903, 1.43280, -0.77903, 1.70346, 0.0 },
      { 0.70381, 1.38271, 0.70381, -1.38271, 1.42239, 0.77978, 1.42239, -0.77978, 1.69319, 0.0 } };
   static double const dtf4[ 3 ][ 8 ] = {
      { 1.13231, 1.28122, 1.13231, -1.28122, 1.78532, 0.46766, 1.78532, -0.46766 },
      { 1.04198, 1.25046, 1.04198, -1.25046, 1.69337, 0.45006, 1.69337, -0.45006 },
      { 0.94576, 1.21364, 0.94576, -1.21364, 1.59892, 0.42668, 1.59892, -0.42668 } };
   static double const dtf3[ 3 ][ 6 ] = {
      { 1.41650, 1.00829, 1.41650, -1.00829, 1.86131, 0.0 },
      { 1.32094, 0.97057, 1.32094, -0.97057, 1.77635, 0.0 },
      { 1.21969, 0.91724, 1.21969, -0.91724, 1.69485, 0.0 } };
   static double const dtf2[ 4 ] = { 1.69580, 0.59955, 1.69580, -0.59955 };
   static double const fb5[ 10 ] = { 2.19406, 1.90251, 2.19406, -1.90251, 2.31029, 0.598022, 2.31029, -0.598022, 7.64071, 0.0 };
   static double const fb4[ 8 ] = { 2.06954, 1.90416, 2.06954, -1.90416, 2.18403, 0.593635, 2.18403, -0.593635 };
   static double const as3[ 6 ] = { 2.1078345, 1.4058574, 2.1078345, -1.4058574, 2.1668048, 0.0 };
   double const* t = NULL;
   size_t o = order > 2 ? 0 : order;       /* the tables' "default" rows are order 0 */
   if( !*fb ) {
      switch( nn ) {
         case 5: t = dtf5[ o ]; break;
         case 4: t = dtf4[ o ]; break;
         case 3: t = dtf3[ o ]; break;
         case 2: t = dtf2; break;
         case 1: { static double const one[ 2 ] = { 2.0, 0.0 }; t = one; break; }
         default: *fb = 1; nn = 3; t = as3; break;
      }
   } else {
      switch( nn ) {
         case 5: t = fb5; break;
         case 4: t = fb4; break;
         default: nn = 3; t = as3; break;
      }
   }
   pp[ 0 ].re = (double)nn;
   pp[ 0 ].im = 0.0;
   for( size_t m = 1; m <= nn; ++m ) { pp[ m ].re = t[ 2 * ( m - 1 ) ]; pp[ m ].im = t[ 2 * ( m - 1 ) + 1 ]; }
}

/* A pole raised to 1/q in polar form, as q2sigma and the pole scaling (gaussiir.cpp:61-68, 318-323). */
static or_cplx iir_pole_pow( or_cplx p, double q ) {
   double modulus = sqrt( p.re * p.re + p.im * p.im );
   double phase = atan( p.im / p.re );
   modulus = exp( log( modulus ) / q );
   phase = phase / q;
   or_cplx r = { modulus * cos( phase ), modulus * sin( phase ) };
   return r;
}

/* q2sigma, gaussiir.cpp:55-82. */
static double iir_q2sigma( size_t nn, or_cplx const* pp, double q ) {
   double var = 0.0;
   for( size_t mm = 1; mm <= ( nn - ( nn & 1u )); mm += 2 ) {
      or_cplx r = iir_pole_pow( pp[ mm ], q );
      double d = 1 - 2 * r.re + r.re * r.re + r.im * r.im;
      d *= d;
      var += ( 4 * ( r.re + ( r.re - 2 ) * ( r.re * r.re + r.im * r.im ))) / d;
   }
   if( nn & 1u ) {
      double re = iir_pole_pow( pp[ nn ], q ).re;
      var += ( 2 * re ) / (( re - 1 ) * ( re - 1 ));
   }
   return sqrt( var );
}

/* FilterCoefficients, gaussiir.cpp:213-239: bb[nn - mm] accumulates the products of mm poles with
 * decreasing indices, in the recursion's order. */
static void iir_esym( size_t mm, size_t nn, or_cplx const* pp, size_t start, size_t stop, or_cplx tmp, or_cplx* bb ) {
   if( start == mm && stop == nn ) {
      tmp.re = 1.0; tmp.im = 0.0;
      bb[ nn - mm ].re = 0.0; bb[ nn - mm ].im = 0.0;
   }
   if( start > 1 ) {
      for( size_t ii = start; ii <= stop; ++ii ) { iir_esym( mm, nn, pp, start - 1, ii - 1, cmul( tmp, pp[ ii ] ), bb ); }
   } else if( start == 1 ) {
      for( size_t ii = start; ii <= stop; ++ii ) { bb[ nn - mm ] = cadd( cmul( tmp, pp[ ii ] ), bb[ nn - mm ] ); }
   } else if( start == 0 && mm == 0 ) {
      bb[ nn ].re = 1.0; bb[ nn ].im = 0.0;
   }
}

/* FillGaussIIRParams, gaussiir.cpp:241-446. */
static int iir_design( double sigma, unsigned order, size_t filter_order, int fb, double truncation, or_iir_params* P ) {
   if( order > 4 ) { return OR_ERR_ORDER; }
   if( truncation <= 0.0 ) { truncation = 3; }
   truncation = truncation < max_gauss_truncation( 0 ) ? truncation : max_gauss_truncation( 0 );
   memset( P, 0, sizeof( *P ));
   size_t b = (size_t)( sigma * truncation + 0.5 );
   P->border = b > 5 ? b : 5;
   or_cplx pp[ 10 ];
   iir_fill_poles( filter_order, pp, order, &fb );
   size_t nn = (size_t)pp[ 0 ].re;
   double q = 0;
   if( fb ) {
      double q0term = -sigma * sigma, q1term = 0.0, q2term = 0.0;
      for( size_t mm = 1; mm <= ( nn - ( nn & 1u )); mm += 2 ) {
         double re = pp[ mm ].re, im = pp[ mm ].im;
         double t1 = 4 * ( -1 + 3 * re - 3 * re * re - im * im + re * ( re * re + im * im ));
         double t2 = 4 * ( 1 - 2 * re + re * re - im * im );
         double d = 1 - 2 * re + re * re + im * im;
         d *= d;
         q1term += t1 / d;
         q2term += t2 / d;
      }
      if( nn & 1u ) {
         double d = pp[ nn ].re - 1.0;
         q1term += 2.0 / d;
         q2term += 2.0 / ( d * d );
      }
      double t = sqrt( q1term * q1term - 4.0 * q2term * q0term );
      double r1 = ( -q1term + t ) / ( 2 * q2term );
      double r2 = ( -q1term - t ) / ( 2 * q2term );
      q = r1 > r2 ? r1 : r2;
      for( size_t mm = 1; mm <= nn; ++mm ) {
         or_cplx np = { 1.0 + ( pp[ mm ].re - 1.0 ) / q, pp[ mm ].im / q };
         pp[ mm ] = np;
      }
   } else {
      q = sigma / 2.0;
      double q0 = q;
      double qs = iir_q2sigma( nn, pp, q );
      size_t n_iter = 0;
      while( fabs( sigma - qs ) > 0.000001 && n_iter < 100 ) {
         q += q0 - qs / 2.0;
         qs = iir_q2sigma( nn, pp, q );
         ++n_iter;
      }
      for( size_t mm = 1; mm <= nn; ++mm ) { pp[ mm ] = iir_pole_pow( pp[ mm ], q ); }
   }
   or_cplx bb[ 10 ];
   or_cplx zero = { 0.0, 0.0 };
   for( size_t mm = 0; mm <= nn; ++mm ) { iir_esym( mm, nn, pp, mm, nn, zero, bb ); }
   for( size_t mm = 0; mm <= nn; ++mm ) {
      double s = pow( -1.0, (double)( nn - mm )) / bb[ 0 ].re;
      bb[ nn - mm ].re *= s;
      bb[ nn - mm ].im *= s;
      P->b1[ nn - mm ] = P->b2[ nn - mm ] = bb[ nn - mm ].re;
   }
   P->cc = 0.0;
   for( size_t mm = 0; mm <= nn; ++mm ) { P->cc += P->b1[ mm ]; }
   P->cc = P->cc * P->cc;
   P->den[ 0 ] = nn; P->den[ 1 ] = 1; P->den[ 2 ] = nn;
   P->den[ 3 ] = nn; P->den[ 4 ] = 1; P->den[ 5 ] = nn;
   static double const A1[ 5 ][ 3 ] = { { 1, 0, 0 }, { 0.5, 0, -0.5 }, { 1, -1, 0 }, { 1, -2, 1 }, { 1, -2, 1 } };
   static double const A2[ 5 ][ 3 ] = { { 1, 0, 0 }, { 0, 1, 0 }, { -1, 1, 0 }, { -0.5, 0, 0.5 }, { 1, -2, 1 } };
   for( int k = 0; k < 3; ++k ) { P->a1[ k ] = A1[ order ][ k ]; P->a2[ k ] = A2[ order ][ k ]; }
   for( int j = 0; j < 6; ++j ) { P->num[ j ] = OR_IIR_MAX + 1; }
   for( size_t jj = 0; jj < OR_IIR_MAX; ++jj ) {
      if( P->a1[ jj ] != 0.0 && P->num[ 1 ] > OR_IIR_MAX ) { P->num[ 1 ] = jj; }
      if( P->a2[ jj ] != 0.0 && P->num[ 4 ] > OR_IIR_MAX ) { P->num[ 4 ] = jj; }
   }
   for( size_t jj = OR_IIR_MAX; jj > 0; ) {
      --jj;
      if( P->a1[ jj ] != 0.0 && P->num[ 2 ] > OR_IIR_MAX ) { P->num[ 2 ] = jj; }
      if( P->a2[ jj ] != 0.0 && P->num[ 5 ] > OR_IIR_MAX ) { P->num[ 5 ] = jj; }
   }
   P->num[ 0 ] = P->num[ 2 ];
   P->num[ 3 ] = P->num[ 5 ];
   return OR_OK;
}

/* GaussIIRLineFilter::Filter, gaussiir.cpp:465-712, restated: `in` and `out` are the whole
 * buffers (border included, `length` samples), `p1` scratch of `length`.  The reference writes
 * out the recursions of orders 3-5 for order 0 (both scans) and for the derivative forms of its
 * default orders; those start from a constant history R (the first / last value over the
 * coefficients' sum), the generic scans set their first `order` values to R instead.  After an
 * unrolled scan the reference finishes the line with the generic form (the same arithmetic up to
 * rounding of the derivative's difference, kept here as the reference has it). */
static void iir_line( double const* p0, double* p2, size_t length, or_iir_params const* P, double* p1 ) {
   double const* a1 = P->a1;
   double const* a2 = P->a2;
   double const* b1 = P->b1;
   double const* b2 = P->b2;
   double const c = P->cc;
   size_t const* MA = P->num;
   size_t const* AR = P->den;
   size_t order1 = AR[ 0 ] > MA[ 0 ] ? AR[ 0 ] : MA[ 0 ];
   size_t order2 = AR[ 3 ] > MA[ 3 ] ? AR[ 3 ] : MA[ 3 ];
   int copy_f = MA[ 0 ] == 0 && a1[ 0 ] == 1.0;
   int copy_b = MA[ 3 ] == 0 && a2[ 0 ] == 1.0;
   double const dsum1 = 1.0 + b1[ 1 ] + b1[ 2 ] + b1[ 3 ] + b1[ 4 ] + b1[ 5 ];
   double const dsum2 = 1.0 + b2[ 1 ] + b2[ 2 ] + b2[ 3 ] + b2[ 4 ] + b2[ 5 ];
   size_t nn1 = AR[ 2 ];
   /* forward: which written-out form applies */
   int fform = 0;                    /* 0 generic, 1 copy, 2 half difference (order 1), 3 difference (order 2) */
   if( order1 >= 3 && order1 <= 5 ) {
      if( copy_f ) { fform = 1; }
      else if( order1 == 4 && a1[ 0 ] == 0.5 && a1[ 1 ] == 0.0 && a1[ 2 ] == -0.5 && a1[ 3 ] == 0.0 ) { fform = 2; }
      else if( order1 == 5 && a1[ 0 ] == 1.0 && a1[ 1 ] == -1.0 && a1[ 2 ] == 0.0 && a1[ 3 ] == 0.0 ) { fform = 3; }
   }
   double R;
   size_t ii = 0, s = 0, stop = 0;
   if( fform == 1 ) { R = p0[ 0 ] / dsum1; s = 0; }
   else if( fform == 2 ) { R = ( p0[ 1 ] - p0[ 0 ] ) / dsum1; s = 2; }
   else if( fform == 3 ) { R = ( p0[ 1 ] - p0[ 0 ] ) / dsum1; s = 1; }
   else {
      double val = 0.0;
      for( size_t jj = MA[ 1 ]; jj <= MA[ 2 ]; ++jj ) { val += a1[ jj ] * p0[ MA[ 2 ] - jj ]; }
      R = val / dsum1;
      s = order1;
   }
   for( ii = 0; ii < s; ++ii ) { p1[ ii ] = R; }
   stop = s;                         /* the written-out scan covers [s, stop) */
   if( fform ) { while( stop < length - order1 ) { stop += order1; } }
   for( ii = s; ii < length; ++ii ) {
      double val;
      if( ii < stop && fform == 1 ) { val = p0[ ii ]; }
      else if( ii < stop && fform == 2 ) { val = 0.5 * ( p0[ ii ] - p0[ ii - 2 ] ); }
      else if( ii < stop && fform == 3 ) { val = p0[ ii ] - p0[ ii - 1 ]; }
      else if( copy_f ) { val = p0[ ii ]; }
      else {
         val = 0.0;
         for( size_t jj = MA[ 1 ]; jj <= MA[ 2 ]; ++jj ) { val += a1[ jj ] * p0[ ii - jj ]; }
      }
      for( size_t jj = AR[ 1 ]; jj <= nn1; ++jj ) { val -= b1[ jj ] * ( ii >= jj ? p1[ ii - jj ] : R ); }
      p1[ ii ] = val;
   }
   /* backward */
   size_t nn2 = AR[ 5 ];
   int bform = 0;
   if( order2 >= 3 && order2 <= 5 ) {
      if( copy_b ) { bform = 1; }
      else if( order2 == 4 && a2[ 0 ] == 0.0 && a2[ 1 ] == 1.0 && a2[ 2 ] == 0.0 && a2[ 3 ] == 0.0 ) { bform = 2; }
      else if( order2 == 5 && a2[ 0 ] == -1.0 && a2[ 1 ] == 1.0 && a2[ 2 ] == 0.0 && a2[ 3 ] == 0.0 ) { bform = 3; }
   }
   size_t top;                       /* p2[top + 1 .. length - 1] are set before the scan */
   if( bform == 1 ) { R = c * p1[ length - 1 ] / dsum2; top = length - 1; }
   else if( bform == 2 ) { R = c * p1[ length - 1 ] / dsum2; p2[ length - 1 ] = R; top = length - 2; }
   else if( bform == 3 ) { R = c * ( -p1[ length - 2 ] + p1[ length - 1 ] ) / dsum2; p2[ length - 1 ] = R; top = length - 2; }
   else {
      double val = 0.0;
      for( size_t jj = MA[ 4 ]; jj <= MA[ 5 ]; ++jj ) { val += a2[ jj ] * p1[ length - 1 - MA[ 5 ] + jj ]; }
      R = val / dsum2;
      for( ii = length - 1; ii > length - 1 - order2; --ii ) { p2[ ii ] = c * R; }
      top = length - 1 - order2;
   }
   /* the written-out scan covers (low, top]: steps of order2 while the step's start is >= order2 */
   size_t low = top + 1;
   if( bform ) {
      size_t i = top;
      while( i >= order2 ) { i -= order2; }
      low = i + 1;                   /* samples below `low` take the generic form */
      if( top < order2 ) { low = top + 1; }
   }
   for( size_t k = top + 1; k-- > 0; ) {
      double val;
      int wo = bform && k >= low;
      if( wo && bform == 1 ) { val = c * p1[ k ]; }
      else if( wo && bform == 2 ) { val = c * p1[ k + 1 ]; }
      else if( wo && bform == 3 ) { val = c * ( -p1[ k ] + p1[ k + 1 ] ); }
      else if( copy_b ) { val = c * p1[ k ]; }
      else {
         val = 0.0;
         for( size_t jj = MA[ 4 ]; jj <= MA[ 5 ]; ++jj ) { val += a2[ jj ] * p1[ k + jj ]; }
         val = c * val;
      }
      for( size_t jj = AR[ 4 ]; jj <= nn2; ++jj ) { val -= b2[ jj ] * ( k + jj < length ? p2[ k + jj ] : R ); }
      p2[ k ] = val;
   }
}

int or_gauss_iir( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                  void* out, int out_dtype, int64_t const* out_strides, double const* sigmas, unsigned const* orders,
                  int const* bcs, unsigned const* filter_orders, int forward_backward, double truncation ) {
   if( ndims < 1 || ndims > OR_MAX_DIMS ) { return OR_ERR_ARG; }
   or_iir_params P[ OR_MAX_DIMS ];
   or_iir_params const* I[ OR_MAX_DIMS ];
   int proc[ OR_MAX_DIMS ];
   size_t border[ OR_MAX_DIMS ];
   for( int d = 0; d < ndims; ++d ) {
      proc[ d ] = sigmas[ d ] > 0.0 && sizes[ d ] > 1;
      border[ d ] = 0;
      I[ d ] = &P[ d ];
      if( !proc[ d ] ) { continue; }
      size_t fo = filter_orders ? filter_orders[ d ] : ( orders[ d ] > 2 ? 5 : orders[ d ] + 3 );
      int st = iir_design( sigmas[ d ], orders[ d ], fo, forward_backward, truncation, &P[ d ] );
      if( st != OR_OK ) { return st; }
      border[ d ] = P[ d ].border;
   }
   return separable_driver( in, in_dtype, ndims, sizes, in_strides, out, out_dtype, out_strides, proc, border, bcs,
                            2, NULL, NULL, I );
}
