// K1: fused multi-axis Gaussian FIR tile kernels.
//
// DIPlib's Framework::Separable (src/library/framework_separable.cpp:243-430) filters one axis
// per pass and writes every pass to the output image, so an nD filter reads and writes the
// whole image n times.  These kernels apply all filtered axes in one launch: a CTA stages a
// tile of the input plus its boundary-extended halo in shared memory (converting the sample
// type to float once), applies the y pass and the x pass from shared memory with register
// blocking, and for 3D marches along z keeping the z taps in a register ring, so each input
// voxel is read from HBM about once and each output voxel written once.
//
// Boundary extension is applied to the input once.  For the boundary conditions accepted here
// (index-mapping ones and "add zeros", see bc_is_index_map) extending the filtered
// intermediate along the next axis, as DIPlib does, equals filtering the extended input, so the
// result is DIPlib's up to float rounding order.
#pragma once

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

// Exact integer -> float conversion by exponent-bias insertion (valid for |v| < 2^22).
template< typename TIn > __device__ __forceinline__ float to_f32( TIn v );
template<> __device__ __forceinline__ float to_f32< float >( float v ) { return v; }
template<> __device__ __forceinline__ float to_f32< uint16_t >( uint16_t v ) {
   return __uint_as_float( 0x4B000000u | static_cast< uint32_t >( v )) - 8388608.0f;
}
template<> __device__ __forceinline__ float to_f32< uint8_t >( uint8_t v ) {
   return __uint_as_float( 0x4B000000u | static_cast< uint32_t >( v )) - 8388608.0f;
}
template<> __device__ __forceinline__ float to_f32< int16_t >( int16_t v ) {
   return __int_as_float( 0x4B400000 + static_cast< int32_t >( v )) - 12582912.0f;
}

// Maps coordinate j of an axis of length n to a source index; fl bit 0 = negate, bit 1 = zero.
__device__ __forceinline__ void map_coord( int64_t j, int64_t n, int32_t bc, int64_t& idx, uint8_t& fl ) {
   fl = 0;
   if( j >= 0 && j < n ) { idx = j; return; }
   if( bc == BC_ADD_ZEROS ) { idx = 0; fl = 2; return; }
   bool neg;
   idx = bc_map_index( j, n, bc, &neg );
   fl = neg ? 1 : 0;
}

template< int N > struct AlignUp4 { static constexpr int value = ( N + 3 ) / 4 * 4; };

// Shared-memory layout of a tile: staged input A [WY][WX], y-filtered B [TY][PB], and the
// boundary maps of the tile's rows and columns.
template< int TX, int TY, int HX, int HY >
struct TileLayout {
   static constexpr int WX = TX + 2 * HX;
   static constexpr int WY = TY + 2 * HY;
   static constexpr int PB = AlignUp4< WX >::value + 4;     // float4 reads may run 3 past
   static constexpr int A_FLOATS = AlignUp4< WY * WX >::value;
   static constexpr int B_FLOATS = TY * PB;
   static constexpr size_t bytes() {
      return ( A_FLOATS + B_FLOATS ) * sizeof( float ) + WY * sizeof( int64_t ) + WX * sizeof( int32_t ) + WY + WX + 16;
   }
};

struct TileMaps {
   int64_t* rowoff;
   int32_t* colidx;
   uint8_t* rfl;
   uint8_t* cfl;
};

template< int TX, int TY, int HX, int HY >
__device__ __forceinline__ void build_maps( FusedArgs const& a, int64_t x0, int64_t y0, TileMaps m, int tid, int nt ) {
   using L = TileLayout< TX, TY, HX, HY >;
   for( int r = tid; r < L::WY; r += nt ) {
      int64_t idx; uint8_t fl;
      map_coord( y0 - HY + r, a.n[ 1 ], a.bc[ 1 ], idx, fl );
      m.rowoff[ r ] = idx * a.ss[ 1 ];
      m.rfl[ r ] = fl;
   }
   for( int c = tid; c < L::WX; c += nt ) {
      int64_t idx; uint8_t fl;
      map_coord( x0 - HX + c, a.n[ 0 ], a.bc[ 0 ], idx, fl );
      m.colidx[ c ] = static_cast< int32_t >( idx );
      m.cfl[ c ] = fl;
   }
}

// Stage one input plane (base `src`, extra flags `pfl` for the plane) into A.
template< typename TIn, int TX, int TY, int HX, int HY, int NT >
__device__ __forceinline__ void stage_plane( TIn const* __restrict__ src, int64_t sy, bool interior, int64_t x0, int64_t y0,
                                             uint8_t pfl, TileMaps const& m, float* A, int tid ) {
   using L = TileLayout< TX, TY, HX, HY >;
   if( pfl & 2 ) {
#pragma unroll 1
      for( int e = tid; e < L::WY * L::WX; e += NT ) { A[ e ] = 0.0f; }
      return;
   }
   if( interior ) {
      TIn const* base = src + ( y0 - HY ) * sy + ( x0 - HX );
      bool neg = pfl & 1;
#pragma unroll 4
      for( int e = tid; e < L::WY * L::WX; e += NT ) {
         int r = e / L::WX;
         int c = e - r * L::WX;
         float v = to_f32< TIn >( base[ r * sy + c ] );
         A[ e ] = neg ? -v : v;
      }
   } else {
#pragma unroll 4
      for( int e = tid; e < L::WY * L::WX; e += NT ) {
         int r = e / L::WX;
         int c = e - r * L::WX;
         uint8_t fl = static_cast< uint8_t >( m.rfl[ r ] | m.cfl[ c ] );
         float v = 0.0f;
         if( !( fl & 2 )) {
            v = to_f32< TIn >( src[ m.rowoff[ r ] + m.colidx[ c ] ] );
            if(( m.rfl[ r ] ^ m.cfl[ c ] ^ pfl ) & 1 ) { v = -v; }
         }
         A[ e ] = v;
      }
   }
}

// y pass over all WX staged columns: B[y][c] = sum_k wy_k A[y + HY + k][c].
template< int TX, int TY, int HX, int HY, int RY, bool ODDY, int NT >
__device__ __forceinline__ void y_pass( FusedArgs const& a, float const* A, float* B, int tid ) {
   using L = TileLayout< TX, TY, HX, HY >;
   constexpr int NYB = TY / RY;
#pragma unroll 1
   for( int item = tid; item < L::WX * NYB; item += NT ) {
      int c = item % L::WX;
      int yb = item / L::WX;
      float v[ RY + 2 * HY ];
#pragma unroll
      for( int i = 0; i < RY + 2 * HY; ++i ) { v[ i ] = A[ ( yb * RY + i ) * L::WX + c ]; }
#pragma unroll
      for( int o = 0; o < RY; ++o ) {
         float s = ODDY ? 0.0f : a.w[ 1 ][ 0 ] * v[ o + HY ];
#pragma unroll
         for( int k = 1; k <= HY; ++k ) {
            s = fmaf( a.w[ 1 ][ k ], ODDY ? ( v[ o + HY + k ] - v[ o + HY - k ] ) : ( v[ o + HY + k ] + v[ o + HY - k ] ), s );
         }
         B[ ( yb * RY + o ) * L::PB + c ] = s;
      }
   }
}

// x pass of RX consecutive outputs of row r starting at column s*RX (float4 reads of B).
template< int TX, int TY, int HX, int HY, int RX, bool ODDX >
__device__ __forceinline__ void x_pass( FusedArgs const& a, float const* B, int r, int s, float* out ) {
   using L = TileLayout< TX, TY, HX, HY >;
   constexpr int NV = AlignUp4< RX + 2 * HX >::value;
   float v[ NV ];
   float4 const* row = reinterpret_cast< float4 const* >( B + r * L::PB + s * RX );
#pragma unroll
   for( int i = 0; i < NV / 4; ++i ) {
      float4 q = row[ i ];
      v[ 4 * i ] = q.x; v[ 4 * i + 1 ] = q.y; v[ 4 * i + 2 ] = q.z; v[ 4 * i + 3 ] = q.w;
   }
#pragma unroll
   for( int o = 0; o < RX; ++o ) {
      float acc = ODDX ? 0.0f : a.w[ 0 ][ 0 ] * v[ o + HX ];
#pragma unroll
      for( int k = 1; k <= HX; ++k ) {
         acc = fmaf( a.w[ 0 ][ k ], ODDX ? ( v[ o + HX + k ] - v[ o + HX - k ] ) : ( v[ o + HX + k ] + v[ o + HX - k ] ), acc );
      }
      out[ o ] = acc;
   }
}

template< int RX >
__device__ __forceinline__ void store_row( float* dst, int64_t x, int64_t nx, float const* v ) {
   if( RX == 4 && x + 4 <= nx && ( reinterpret_cast< uintptr_t >( dst ) & 15 ) == 0 ) {
      *reinterpret_cast< float4* >( dst ) = make_float4( v[ 0 ], v[ 1 ], v[ 2 ], v[ 3 ] );
   } else {
#pragma unroll
      for( int i = 0; i < RX; ++i ) {
         if( x + i < nx ) { dst[ i ] = v[ i ]; }
      }
   }
}

// ---- 2D ---------------------------------------------------------------------------------

template< typename TIn, int HX, int HY, bool ODDX, bool ODDY, int TX, int TY, int RX, int RY, int NT >
__global__ void __launch_bounds__( NT ) fused2d_kernel( FusedArgs const __grid_constant__ a ) {
   using L = TileLayout< TX, TY, HX, HY >;
   extern __shared__ float4 smem4[];
   float* A = reinterpret_cast< float* >( smem4 );
   float* B = A + L::A_FLOATS;
   TileMaps m;
   m.rowoff = reinterpret_cast< int64_t* >( B + L::B_FLOATS );
   m.colidx = reinterpret_cast< int32_t* >( m.rowoff + L::WY );
   m.rfl = reinterpret_cast< uint8_t* >( m.colidx + L::WX );
   m.cfl = m.rfl + L::WY;

   int const tid = static_cast< int >( threadIdx.x );
   int64_t t = blockIdx.x;
   int64_t const tx = t % a.tiles_x; t /= a.tiles_x;
   int64_t const ty = t % a.tiles_y; t /= a.tiles_y;
   int64_t const b = t;
   int64_t const x0 = tx * TX, y0 = ty * TY;
   TIn const* src = static_cast< TIn const* >( a.src ) + b * a.sb;
   float* dst = a.dst + b * a.db;
   bool const interior = x0 - HX >= 0 && x0 + TX + HX <= a.n[ 0 ] && y0 - HY >= 0 && y0 + TY + HY <= a.n[ 1 ];
   if( !interior ) {
      build_maps< TX, TY, HX, HY >( a, x0, y0, m, tid, NT );
      __syncthreads();
   }
   stage_plane< TIn, TX, TY, HX, HY, NT >( src, a.ss[ 1 ], interior, x0, y0, 0, m, A, tid );
   __syncthreads();
   y_pass< TX, TY, HX, HY, RY, ODDY, NT >( a, A, B, tid );
   __syncthreads();
   constexpr int NSEG = TX / RX;
#pragma unroll 1
   for( int item = tid; item < TY * NSEG; item += NT ) {
      int s = item % NSEG;
      int r = item / NSEG;
      int64_t y = y0 + r;
      if( y >= a.n[ 1 ] ) { continue; }
      float out[ RX ];
      x_pass< TX, TY, HX, HY, RX, ODDX >( a, B, r, s, out );
      int64_t x = x0 + s * RX;
      if( x < a.n[ 0 ] ) { store_row< RX >( dst + y * a.ds[ 1 ] + x, x, a.n[ 0 ], out ); }
   }
}

// ---- 3D ---------------------------------------------------------------------------------

template< typename TIn, int HX, int HY, int HZ, bool ODDX, bool ODDY, bool ODDZ, int TX, int TY, int RY, int NT >
__global__ void __launch_bounds__( NT, 2 ) fused3d_kernel( FusedArgs const __grid_constant__ a ) {
   constexpr int RX = 4;
   constexpr int NSEG = TX / RX;
   static_assert( TY * NSEG == NT, "one x-pass item per thread" );
   constexpr int M = 2 * HZ + 1;
   using L = TileLayout< TX, TY, HX, HY >;
   extern __shared__ float4 smem4[];
   float* A = reinterpret_cast< float* >( smem4 );
   float* B = A + L::A_FLOATS;
   TileMaps m;
   m.rowoff = reinterpret_cast< int64_t* >( B + L::B_FLOATS );
   m.colidx = reinterpret_cast< int32_t* >( m.rowoff + L::WY );
   m.rfl = reinterpret_cast< uint8_t* >( m.colidx + L::WX );
   m.cfl = m.rfl + L::WY;

   int const tid = static_cast< int >( threadIdx.x );
   int64_t t = blockIdx.x;
   int64_t const tx = t % a.tiles_x; t /= a.tiles_x;
   int64_t const ty = t % a.tiles_y; t /= a.tiles_y;
   int64_t const zc = t % a.zchunks; t /= a.zchunks;
   int64_t const b = t;
   int64_t const x0 = tx * TX, y0 = ty * TY, z0 = zc * a.lz;
   int64_t const zlen = ( a.n[ 2 ] - z0 ) < a.lz ? ( a.n[ 2 ] - z0 ) : a.lz;
   TIn const* src = static_cast< TIn const* >( a.src ) + b * a.sb;
   float* dst = a.dst + b * a.db;
   bool const interior = x0 - HX >= 0 && x0 + TX + HX <= a.n[ 0 ] && y0 - HY >= 0 && y0 + TY + HY <= a.n[ 1 ];
   if( !interior ) {
      build_maps< TX, TY, HX, HY >( a, x0, y0, m, tid, NT );
      __syncthreads();
   }
   int const r_own = tid / NSEG;
   int const s_own = tid % NSEG;
   int64_t const y_own = y0 + r_own;
   int64_t const x_own = x0 + s_own * RX;
   bool const own_valid = y_own < a.n[ 1 ] && x_own < a.n[ 0 ];
   float* dst_own = dst + y_own * a.ds[ 1 ] + x_own;

   float acc[ M ][ RX ];
#pragma unroll
   for( int sl = 0; sl < M; ++sl ) {
#pragma unroll
      for( int i = 0; i < RX; ++i ) { acc[ sl ][ i ] = 0.0f; }
   }
   int64_t const nplanes = zlen + 2 * HZ;
#pragma unroll 1
   for( int64_t q0 = 0; q0 < nplanes; q0 += M ) {
#pragma unroll
      for( int j = 0; j < M; ++j ) {
         int64_t const q = q0 + j;
         if( q >= nplanes ) { break; }
         int64_t zi; uint8_t zfl;
         map_coord( z0 - HZ + q, a.n[ 2 ], a.bc[ 2 ], zi, zfl );
         stage_plane< TIn, TX, TY, HX, HY, NT >( src + zi * a.ss[ 2 ], a.ss[ 1 ], interior, x0, y0, zfl, m, A, tid );
         __syncthreads();
         y_pass< TX, TY, HX, HY, RY, ODDY, NT >( a, A, B, tid );
         __syncthreads();
         float v[ RX ];
         x_pass< TX, TY, HX, HY, RX, ODDX >( a, B, r_own, s_own, v );
         // Ring: plane q contributes to outputs t = q - d, d = 0 .. 2HZ, with z offset d - HZ.
#pragma unroll
         for( int d = 0; d <= 2 * HZ; ++d ) {
            constexpr int dummy = 0;
            (void)dummy;
            int const slot = ( j - d + M ) % M;
            int const kk = d - HZ;
            int const ak = kk < 0 ? -kk : kk;
            if( ODDZ && kk == 0 ) {
               if( d == 0 ) {
#pragma unroll
                  for( int i = 0; i < RX; ++i ) { acc[ slot ][ i ] = 0.0f; }
               }
               continue;
            }
            float const c = ( ODDZ && kk < 0 ) ? -a.w[ 2 ][ ak ] : a.w[ 2 ][ ak ];
#pragma unroll
            for( int i = 0; i < RX; ++i ) {
               acc[ slot ][ i ] = ( d == 0 ) ? c * v[ i ] : fmaf( c, v[ i ], acc[ slot ][ i ] );
            }
         }
         int64_t const to = q - 2 * HZ;
         if( to >= 0 && to < zlen && own_valid ) {
            store_row< RX >( dst_own + ( z0 + to ) * a.ds[ 2 ], x_own, a.n[ 0 ], acc[ ( j + 1 ) % M ] );
         }
      }
   }
}

} // namespace dipcu
