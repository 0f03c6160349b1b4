// Several Gaussian derivatives of one image from one read of it: the components of dip::Gradient,
// dip::Hessian and dip::Laplace (src/linear/derivative.cpp:142-172, 330-418 in DIPlib), each of
// which the reference computes as its own dip::GaussFIR call, and the gradient products of
// dip::StructureTensor (src/analysis/structure_tensor.cpp:33-59).
//
// One CTA per output tile (32 x TY x TZ samples, x y z):
//   1. the input tile plus its halo, extended by the boundary condition (an index mapping per
//      axis, or zeros), is read once into shared memory as float (batches of loads in flight);
//   2. z passes: every z order any component needs, over the tile's x-y halo region (each thread
//      one (x, y) column, its z window in registers, all z orders from one load of the window);
//   3. y passes: every (y order, z order) pair any component needs, over the x halo region (a
//      thread per column and segment of 8 rows);
//   4. x passes: each thread a segment of 8 outputs of one row, every component from the
//      y-filtered buffers, then the epilogue: the components themselves, their symmetric products
//      (DIPlib's symmetric-matrix order), their sum, or the square root of the sum of squares.
// The taps are GaussFIR's own (build_filters, rounded to float), applied in GaussFIR's form:
// centre tap plus, per distance k, tap k times the sum (even orders) or difference (odd orders)
// of the samples at +k and -k.  For the index-mapping boundary conditions and "add zeros",
// extending the input once and filtering is the same as the reference's per-pass extension of
// each intermediate.  Computation in float (inputs whose flex type is sfloat).
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

namespace {

constexpr int kMdMaxComp = 6;    // components (a 3D Hessian)
constexpr int kMdMaxOrd = 4;     // distinct filters per axis
constexpr int kMdTX = 32;        // tile width
constexpr int kMdR = 8;          // outputs per thread in the x pass
constexpr int kMdThreads = 256;
constexpr int kMdLoadBatch = 8;  // tile elements per thread whose loads are in flight together
constexpr int kMdYS = 8;         // rows per thread in the y pass

struct MdArgs {
   void const* src;
   int32_t src_dt;
   int64_t ss[ 3 ];
   int32_t n[ 3 ];                      // image sizes x, y, z (z = 1 in 2D)
   int32_t bc[ 3 ];
   int32_t tiles[ 3 ];
   int32_t nord[ 3 ];                   // distinct filters per axis
   int32_t fodd[ 3 ][ kMdMaxOrd ];
   float taps[ 3 ][ kMdMaxOrd ][ 9 ];   // centre first, zero beyond each filter's half-width
   int32_t ncomp;
   int32_t cx[ kMdMaxComp ];            // x filter slot of each component
   int32_t ccombo[ kMdMaxComp ];        // (y, z) pair of each component
   int32_t ncombo;
   int32_t combo_y[ kMdMaxComp ], combo_z[ kMdMaxComp ];
   int32_t mode;                        // 0 components, 1 symmetric products, 2 sum, 3 sqrt of sum of squares
   int32_t nout;
   void* dst[ kMdMaxComp ];
   int32_t dst_dt[ kMdMaxComp ];
   int64_t ds[ kMdMaxComp ][ 3 ];
   int32_t off_a, off_b;                // shared-memory offsets (floats) of the z- and y-pass buffers
   int32_t all_float;                   // every output is sfloat
};

// Source index of extended position j along an axis of n samples (-1: a zero of "add zeros").
__device__ __forceinline__ int64_t md_map( int64_t j, int64_t n, int32_t bc, bool* neg ) {
   *neg = false;
   if( j >= 0 && j < n ) { return j; }
   if( bc == BC_ADD_ZEROS ) { return -1; }
   return bc_map_index( j, n, bc, neg );
}

// One filter of half-width up to HB applied at window position c (centre) of `v`.
template< int HB, int LEN >
__device__ __forceinline__ float md_tap( float const ( &v )[ LEN ], int c, float const* t, bool odd ) {
   float s = t[ 0 ] * v[ c ];
#pragma unroll
   for( int k = 1; k <= HB; ++k ) { s = fmaf( t[ k ], odd ? v[ c + k ] - v[ c - k ] : v[ c + k ] + v[ c - k ], s ); }
   return s;
}

template< int HB, int TY, int TZ >
__global__ void __launch_bounds__( kMdThreads ) multi_deriv_kernel( MdArgs const __grid_constant__ a ) {
   constexpr int HZ = TZ > 1 ? HB : 0;
   constexpr int W0 = kMdTX + 2 * HB, W1 = TY + 2 * HB, W2 = TZ + 2 * HZ;
   constexpr int YP = W0 | 1;       // row stride of the y-pass buffers (odd: conflict-free x pass)
   extern __shared__ float md_smem[];
   float* const tin = md_smem;                          // [W2][W1][W0]
   float* const za = TZ > 1 ? md_smem + a.off_a : tin;  // [nord_z][TZ][W1][W0]
   float* const yb = md_smem + a.off_b;                 // [ncombo][TZ][TY][YP]
   int const tid = static_cast< int >( threadIdx.x );

   int64_t t = blockIdx.x;
   int const tx = static_cast< int >( t % a.tiles[ 0 ] );
   t /= a.tiles[ 0 ];
   int const ty = static_cast< int >( t % a.tiles[ 1 ] );
   int const tz = static_cast< int >( t / a.tiles[ 1 ] );
   int const x0 = tx * kMdTX, y0 = ty * TY, z0 = tz * TZ;

   // 1. input tile with halo: each thread a batch of kMdLoadBatch elements whose loads are all
   //    issued before any is stored (the loads' latency overlaps), source rows mapped through the
   //    boundary condition, columns directly where the tile lies inside the image along x
   {
      bool const xin = x0 - HB >= 0 && x0 - HB + W0 <= a.n[ 0 ];
      bool const fsrc = a.src_dt == DT_SFLOAT;
      constexpr int NE = W0 * W1 * W2;
      for( int e0 = 0; e0 < NE; e0 += kMdThreads * kMdLoadBatch ) {
         float v[ kMdLoadBatch ];
#pragma unroll
         for( int u = 0; u < kMdLoadBatch; ++u ) {
            int const e = e0 + u * kMdThreads + tid;
            v[ u ] = 0.f;
            if( e < NE ) {
               int const i = e % W0, j = ( e / W0 ) % W1, k = e / ( W0 * W1 );
               bool n0 = false, n1, n2;
               int64_t const sy = md_map( y0 - HB + j, a.n[ 1 ], a.bc[ 1 ], &n1 );
               int64_t const sz = TZ > 1 ? md_map( z0 - HZ + k, a.n[ 2 ], a.bc[ 2 ], &n2 ) : ( n2 = false, z0 );
               int64_t sx = x0 - HB + i;
               if( !xin ) { sx = md_map( sx, a.n[ 0 ], a.bc[ 0 ], &n0 ); }
               if( sx >= 0 && sy >= 0 && sz >= 0 ) {
                  int64_t const off = sx * a.ss[ 0 ] + sy * a.ss[ 1 ] + sz * a.ss[ 2 ];
                  float const t = fsrc ? __ldg( static_cast< float const* >( a.src ) + off ) : load_as< float >( a.src, a.src_dt, off );
                  v[ u ] = ( n0 != ( n1 != n2 )) ? -t : t;
               }
            }
         }
#pragma unroll
         for( int u = 0; u < kMdLoadBatch; ++u ) {
            int const e = e0 + u * kMdThreads + tid;
            if( e < NE ) { tin[ e ] = v[ u ]; }
         }
      }
   }
   __syncthreads();

   // 2. z passes: column (i, j) of the x-y halo region, every z filter
   if constexpr( TZ > 1 ) {
      for( int col = tid; col < W0 * W1; col += kMdThreads ) {
         float v[ W2 ];
#pragma unroll
         for( int k = 0; k < W2; ++k ) { v[ k ] = tin[ k * W0 * W1 + col ]; }
         for( int s = 0; s < a.nord[ 2 ]; ++s ) {
            float const* const tp = a.taps[ 2 ][ s ];
            bool const odd = a.fodd[ 2 ][ s ] != 0;
#pragma unroll
            for( int z = 0; z < TZ; ++z ) { za[ ( s * TZ + z ) * W0 * W1 + col ] = md_tap< HZ >( v, z + HZ, tp, odd ); }
         }
      }
      __syncthreads();
   }

   // 3. y passes: column (i, z) of the x halo region and a segment of kMdYS rows, every (y, z) pair
   constexpr int YSEG = TY / kMdYS;
   for( int task = tid; task < W0 * TZ * YSEG; task += kMdThreads ) {
      int const i = task % W0, z = ( task / W0 ) % TZ, ys = task / ( W0 * TZ );
      for( int s = 0; s < ( TZ > 1 ? a.nord[ 2 ] : 1 ); ++s ) {
         bool need = false;
         for( int b = 0; b < a.ncombo; ++b ) { need = need || a.combo_z[ b ] == s; }
         if( !need ) { continue; }
         float v[ kMdYS + 2 * HB ];
         float const* const src = za + ( s * TZ + z ) * W0 * W1 + ys * kMdYS * W0 + i;
#pragma unroll
         for( int j = 0; j < kMdYS + 2 * HB; ++j ) { v[ j ] = src[ j * W0 ]; }
         for( int b = 0; b < a.ncombo; ++b ) {
            if( a.combo_z[ b ] != s ) { continue; }
            float const* const tp = a.taps[ 1 ][ a.combo_y[ b ]];
            bool const odd = a.fodd[ 1 ][ a.combo_y[ b ]] != 0;
            float* const dst = yb + ( b * TZ + z ) * TY * YP + ys * kMdYS * YP + i;
#pragma unroll
            for( int y = 0; y < kMdYS; ++y ) { dst[ y * YP ] = md_tap< HB >( v, y + HB, tp, odd ); }
         }
      }
   }
   __syncthreads();

   // 4. x passes and the epilogue: row (y, z), segment of kMdR outputs
   constexpr int SEGS = kMdTX / kMdR;
   // a warp: 4 segments x 8 rows; with the odd row stride YP its reads fall in distinct banks
   for( int task = tid; task < SEGS * TY * TZ; task += kMdThreads ) {
      int const seg = task % SEGS, y = ( task / SEGS ) % TY, z = task / ( SEGS * TY );
      int const xo = x0 + seg * kMdR, yo = y0 + y, zo = z0 + z;
      if( yo >= a.n[ 1 ] || zo >= a.n[ 2 ] || xo >= a.n[ 0 ] ) { continue; }
      float o[ kMdMaxComp ][ kMdR ];
#pragma unroll
      for( int c = 0; c < kMdMaxComp; ++c ) {
#pragma unroll
         for( int r = 0; r < kMdR; ++r ) { o[ c ][ r ] = 0.f; }
      }
      for( int b = 0; b < a.ncombo; ++b ) {
         float v[ kMdR + 2 * HB ];
         float const* const src = yb + ( b * TZ + z ) * TY * YP + y * YP + seg * kMdR;
#pragma unroll
         for( int k = 0; k < kMdR + 2 * HB; ++k ) { v[ k ] = src[ k ]; }
#pragma unroll
         for( int c = 0; c < kMdMaxComp; ++c ) {
            if( c >= a.ncomp || a.ccombo[ c ] != b ) { continue; }
            float const* const tp = a.taps[ 0 ][ a.cx[ c ]];
            bool const odd = a.fodd[ 0 ][ a.cx[ c ]] != 0;
#pragma unroll
            for( int r = 0; r < kMdR; ++r ) { o[ c ][ r ] = md_tap< HB >( v, r + HB, tp, odd ); }
         }
      }
      int const nr = a.n[ 0 ] - xo < kMdR ? a.n[ 0 ] - xo : kMdR;
      // sfloat outputs take plain stores
      auto store = [ & ]( int q, int r, float val ) {
         int64_t const off = ( xo + r ) * a.ds[ q ][ 0 ] + yo * a.ds[ q ][ 1 ] + zo * a.ds[ q ][ 2 ];
         if( a.all_float ) { static_cast< float* >( a.dst[ q ] )[ off ] = val; }
         else { store_from< float >( a.dst[ q ], a.dst_dt[ q ], off, val ); }
      };
      for( int r = 0; r < kMdR; ++r ) {
         if( r >= nr ) { break; }
         if( a.mode == 0 ) {
#pragma unroll
            for( int c = 0; c < kMdMaxComp; ++c ) { if( c < a.ncomp ) { store( c, r, o[ c ][ r ] ); } }
         } else if( a.mode == 1 ) {
            // diagonal first, then the upper triangle column by column
            int q = 0;
#pragma unroll
            for( int c = 0; c < kMdMaxComp; ++c ) { if( c < a.ncomp ) { store( q++, r, o[ c ][ r ] * o[ c ][ r ] ); } }
#pragma unroll
            for( int j = 1; j < kMdMaxComp; ++j ) {
#pragma unroll
               for( int i = 0; i < j; ++i ) { if( j < a.ncomp ) { store( q++, r, o[ i ][ r ] * o[ j ][ r ] ); } }
            }
         } else {
            float acc = 0.f;
#pragma unroll
            for( int c = 0; c < kMdMaxComp; ++c ) {
               if( c < a.ncomp ) { acc = a.mode == 2 ? acc + o[ c ][ r ] : fmaf( o[ c ][ r ], o[ c ][ r ], acc ); }
            }
            store( 0, r, a.mode == 2 ? acc : sqrtf( acc ));
         }
      }
   }
}

// A distinct filter of one axis: GaussFIR's taps for one order (identity when not processed).
struct MdSlot {
   int64_t h = 0;
   int32_t odd = 0;
   std::vector< double > taps{ 1.0 };
   bool operator==( MdSlot const& o ) const { return h == o.h && odd == o.odd && taps == o.taps; }
};

// Fills `a` (all but the outputs) for `ncomp` order vectors; DIPCU_OK, a GaussFIR error of the
// parameters, or -1 when the kernel does not take the case (the caller then filters per
// component).  `hb` receives the halo bucket (4 or 8).
int md_build( dipcu_image_desc const* in, uint32_t const* orders, int ncomp, double const* sigmas, int32_t const* bcs,
              double truncation, MdArgs& a, int& hb ) {
   int const nd = in->ndims;
   if( nd < 2 || nd > 3 || ncomp < 1 || ncomp > kMdMaxComp ) { return -1; }
   if( suggest_flex( in->dtype ) != DT_SFLOAT ) { return -1; }
   for( int d = 0; d < nd; ++d ) {
      if( in->sizes[ d ] > 0x3fffffff ) { return -1; }
   }
   a = MdArgs{};
   std::vector< MdSlot > slots[ 3 ];
   std::vector< int > cs[ 3 ];                 // slot of each component per axis
   int64_t hmax = 0;
   for( int c = 0; c < ncomp; ++c ) {
      std::vector< AxisFilter > f;
      if( int st = build_filters( in, sigmas, orders + static_cast< size_t >( c ) * nd, bcs, truncation, f, nullptr )) { return st; }
      for( int d = 0; d < 3; ++d ) {
         MdSlot s;
         if( d < nd && f[ static_cast< size_t >( d ) ].process ) {
            AxisFilter const& af = f[ static_cast< size_t >( d ) ];
            if( !( bc_is_index_map( af.bc ))) { return -1; }
            s.h = af.h;
            s.odd = af.odd;
            s.taps = af.taps;
            hmax = s.h > hmax ? s.h : hmax;
         }
         int k = 0;
         while( k < static_cast< int >( slots[ d ].size() ) && !( slots[ d ][ static_cast< size_t >( k ) ] == s )) { ++k; }
         if( k == static_cast< int >( slots[ d ].size() )) {
            if( k == kMdMaxOrd ) { return -1; }
            slots[ d ].push_back( s );
         }
         cs[ d ].push_back( k );
      }
   }
   if( hmax > 8 ) { return -1; }
   hb = hmax <= 4 ? 4 : 8;
   std::vector< std::pair< int, int >> combos;
   for( int c = 0; c < ncomp; ++c ) {
      std::pair< int, int > p{ cs[ 1 ][ static_cast< size_t >( c ) ], cs[ 2 ][ static_cast< size_t >( c ) ] };
      size_t b = 0;
      while( b < combos.size() && combos[ b ] != p ) { ++b; }
      if( b == combos.size() ) { combos.push_back( p ); }
      a.ccombo[ c ] = static_cast< int32_t >( b );
      a.cx[ c ] = cs[ 0 ][ static_cast< size_t >( c ) ];
   }
   a.ncomp = ncomp;
   a.ncombo = static_cast< int32_t >( combos.size() );
   for( size_t b = 0; b < combos.size(); ++b ) {
      a.combo_y[ b ] = combos[ b ].first;
      a.combo_z[ b ] = combos[ b ].second;
   }
   for( int d = 0; d < 3; ++d ) {
      a.nord[ d ] = static_cast< int32_t >( slots[ d ].size() );
      for( size_t s = 0; s < slots[ d ].size(); ++s ) {
         a.fodd[ d ][ s ] = slots[ d ][ s ].odd;
         for( size_t k = 0; k < slots[ d ][ s ].taps.size() && k < 9; ++k ) {
            a.taps[ d ][ s ][ k ] = static_cast< float >( slots[ d ][ s ].taps[ k ] );
         }
      }
      a.n[ d ] = d < nd ? static_cast< int32_t >( in->sizes[ d ] ) : 1;
      a.ss[ d ] = d < nd ? in->strides[ d ] : 0;
      a.bc[ d ] = d < nd ? bcs[ d ] : BC_SYMMETRIC_MIRROR;
   }
   a.src = in->data;
   a.src_dt = in->dtype;
   return DIPCU_OK;
}

template< int HB, int TY, int TZ >
int md_run( MdArgs& a, cudaStream_t stream ) {
   constexpr int HZ = TZ > 1 ? HB : 0;
   constexpr int W0 = kMdTX + 2 * HB, W1 = TY + 2 * HB, W2 = TZ + 2 * HZ;
   int64_t const tin = static_cast< int64_t >( W0 ) * W1 * W2;
   int64_t const za = TZ > 1 ? static_cast< int64_t >( a.nord[ 2 ] ) * TZ * W1 * W0 : 0;
   constexpr int YP = W0 | 1;
   int64_t const yb = static_cast< int64_t >( a.ncombo ) * TZ * TY * YP;
   a.off_a = static_cast< int32_t >( tin );
   // in 3D the y-pass buffers may reuse the input tile (dead after the z passes); in 2D the y
   // passes read the input tile itself
   a.off_b = static_cast< int32_t >(( TZ > 1 && yb <= tin ) ? 0 : tin + za );
   size_t const smem = static_cast< size_t >(( TZ > 1 && yb <= tin ) ? tin + za : tin + za + yb ) * sizeof( float );
   if( smem > 227 * 1024 ) { return -1; }
   auto kern = multi_deriv_kernel< HB, TY, TZ >;
   if( cudaFuncSetAttribute( kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( smem )) != cudaSuccess ) {
      cudaGetLastError();
      return -1;
   }
   a.tiles[ 0 ] = ( a.n[ 0 ] + kMdTX - 1 ) / kMdTX;
   a.tiles[ 1 ] = ( a.n[ 1 ] + TY - 1 ) / TY;
   a.tiles[ 2 ] = ( a.n[ 2 ] + TZ - 1 ) / TZ;
   int64_t const ntiles = static_cast< int64_t >( a.tiles[ 0 ] ) * a.tiles[ 1 ] * a.tiles[ 2 ];
   if( ntiles > 0x7fffffff ) { return -1; }
   kern<<< static_cast< unsigned >( ntiles ), kMdThreads, smem, stream >>>( a ); count_launch();
   cudaError_t const e = cudaGetLastError();
   if( e != cudaSuccess ) { return record_error( DIPCU_ERR_CUDA, cudaGetErrorString( e )); }
   return DIPCU_OK;
}

int md_outputs( int mode, int ncomp ) {
   switch( mode ) {
      case 0: return ncomp;
      case 1: return ncomp * ( ncomp + 1 ) / 2;
      case 2: case 3: return 1;
      default: return -1;
   }
}

} // namespace

// Several GaussFIR outputs of one input from one read of it (see the top of this file); -1 when
// the tile kernel does not take the case, so that the caller filters per component.
int multi_gauss_fir( dipcu_image_desc const* in, dipcu_image_desc const* outs, int nout, uint32_t const* orders, int ncomp,
                     int mode, double const* sigmas, int32_t const* bcs, double truncation, cudaStream_t stream ) {
   if( md_outputs( mode, ncomp ) != nout || nout > kMdMaxComp ) { return -1; }
   MdArgs a;
   int hb = 4;
   if( int st = md_build( in, orders, ncomp, sigmas, bcs, truncation, a, hb )) { return st; }
   a.mode = mode;
   a.nout = nout;
   a.all_float = 1;
   for( int q = 0; q < nout; ++q ) {
      a.dst[ q ] = outs[ q ].data;
      a.dst_dt[ q ] = outs[ q ].dtype;
      a.all_float = a.all_float && outs[ q ].dtype == DT_SFLOAT;
      for( int d = 0; d < 3; ++d ) { a.ds[ q ][ d ] = d < in->ndims ? outs[ q ].strides[ d ] : 0; }
   }
   if( in->ndims == 3 ) { return hb == 4 ? md_run< 4, 8, 8 >( a, stream ) : md_run< 8, 8, 4 >( a, stream ); }
   return hb == 4 ? md_run< 4, 64, 1 >( a, stream ) : md_run< 8, 64, 1 >( a, stream );
}

bool multi_gauss_fir_supported( dipcu_image_desc const* in, uint32_t const* orders, int ncomp, double const* sigmas,
                                int32_t const* bcs, double truncation ) {
   MdArgs a;
   int hb = 4;
   int const st = md_build( in, orders, ncomp, sigmas, bcs, truncation, a, hb );
   return st == DIPCU_OK;
}

} // namespace dipcu

using namespace dipcu;

extern "C" {

int dipcu_gauss_fir_multi( dipcu_image_desc const* in, dipcu_image_desc const* outs, int nout, uint32_t const* orders,
                           int ncomp, int32_t mode, double const* sigmas, int32_t const* bcs, double truncation, void* stream ) {
   if( !in || !outs || !orders || !sigmas || !bcs ) { return record_error( DIPCU_ERR_INVALID_ARG, "null parameter array" ); }
   if( md_outputs( mode, ncomp ) < 1 || md_outputs( mode, ncomp ) != nout ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "wrong number of outputs for the mode" );
   }
   for( int q = 0; q < nout; ++q ) {
      if( int st = check_pair( in, &outs[ q ] )) { return st; }
   }
   int const st = multi_gauss_fir( in, outs, nout, orders, ncomp, mode, sigmas, bcs, truncation, static_cast< cudaStream_t >( stream ));
   if( st == -1 ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "multi-output derivatives: not taken by the tile kernel "
                                                  "(see dipcu_gauss_fir_multi_supported)" );
   }
   return st;
}

int dipcu_gauss_fir_multi_supported( dipcu_image_desc const* in, uint32_t const* orders, int ncomp, double const* sigmas,
                                     int32_t const* bcs, double truncation ) {
   if( !in || !orders || !sigmas || !bcs || ncomp < 1 ) { return 0; }
   return multi_gauss_fir_supported( in, orders, ncomp, sigmas, bcs, truncation ) ? 1 : 0;
}

} // extern "C"
