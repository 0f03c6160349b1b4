// Launchers and the instantiation table of the fused tile kernels (K1).  Each entry fixes the
// per-axis half-widths and symmetry at compile time so that the tap loops unroll fully and the
// weights are read as constant-bank operands; configurations without an entry run on the line
// kernel (K2).
#include <cuda_runtime.h>

#include "fused.cuh"

namespace dipcu {

namespace {

constexpr int kNT = 256;

template< typename TIn, int HX, int HY, bool OX, bool OY >
cudaError_t run2d( FusedArgs& a, cudaStream_t s ) {
   constexpr int TX = 64, TY = 32, RX = 4, RY = 8;
   using L = TileLayout< TX, TY, HX, HY >;
   auto kern = fused2d_kernel< TIn, HX, HY, OX, OY, TX, TY, RX, RY, kNT >;
   size_t smem = L::bytes();
   if( smem > 48 * 1024 ) {
      cudaError_t e = cudaFuncSetAttribute( kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( smem ));
      if( e != cudaSuccess ) { return e; }
   }
   a.tiles_x = static_cast< int32_t >(( a.n[ 0 ] + TX - 1 ) / TX);
   a.tiles_y = static_cast< int32_t >(( a.n[ 1 ] + TY - 1 ) / TY);
   a.zchunks = 1;
   a.lz = 1;
   int64_t grid = static_cast< int64_t >( a.tiles_x ) * a.tiles_y * a.nb;
   if( grid > 0x7fffffff ) { return cudaErrorInvalidValue; }
   kern<<< static_cast< unsigned >( grid ), kNT, smem, s >>>( a );
   return cudaGetLastError();
}

template< typename TIn, int HX, int HY, int HZ, bool OX, bool OY, bool OZ >
cudaError_t run3d( FusedArgs& a, cudaStream_t s ) {
   constexpr int TX = 64, TY = 16, RY = 8;
   using L = TileLayout< TX, TY, HX, HY >;
   auto kern = fused3d_kernel< TIn, HX, HY, HZ, OX, OY, OZ, TX, TY, RY, kNT >;
   size_t smem = L::bytes();
   if( smem > 48 * 1024 ) {
      cudaError_t e = cudaFuncSetAttribute( kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( smem ));
      if( e != cudaSuccess ) { return e; }
   }
   a.tiles_x = static_cast< int32_t >(( a.n[ 0 ] + TX - 1 ) / TX);
   a.tiles_y = static_cast< int32_t >(( a.n[ 1 ] + TY - 1 ) / TY);
   int64_t base = static_cast< int64_t >( a.tiles_x ) * a.tiles_y * a.nb;
   // Split z so that about two CTAs per SM are busy, keeping chunks long against the 2*HZ
   // planes of halo each chunk re-reads.
   int64_t const target = 2 * 148;
   int64_t zchunks = ( target + base - 1 ) / base;
   int64_t max_chunks = a.n[ 2 ] / ( 4 * HZ + 4 );
   if( max_chunks < 1 ) { max_chunks = 1; }
   if( zchunks > max_chunks ) { zchunks = max_chunks; }
   if( zchunks < 1 ) { zchunks = 1; }
   int64_t lz = ( a.n[ 2 ] + zchunks - 1 ) / zchunks;
   zchunks = ( a.n[ 2 ] + lz - 1 ) / lz;
   a.zchunks = static_cast< int32_t >( zchunks );
   a.lz = static_cast< int32_t >( lz );
   int64_t grid = base * zchunks;
   if( grid > 0x7fffffff ) { return cudaErrorInvalidValue; }
   kern<<< static_cast< unsigned >( grid ), kNT, smem, s >>>( a );
   return cudaGetLastError();
}

using Runner = cudaError_t ( * )( FusedArgs&, cudaStream_t );

struct Entry {
   int32_t ndims, in_dt, hx, hy, hz, ox, oy, oz;
   Runner run;
};

// (input type, half-widths, odd flags) instantiated ahead of time.  The set covers the
// benchmark workloads (2D sigma 2; 2D sigma 3 orders 0..2; 3D sigma (1.5, 1.5, 3) orders
// (0,0,0)/(1,0,0); the structure tensor's sigma 1 gradients and sigma 4 smoothing) and
// small-sigma configurations used by the parity tests.
#define E2( T, DT, HX, HY, OX, OY ) { 2, DT, HX, HY, 0, OX, OY, 0, &run2d< T, HX, HY, OX, OY > }
#define E3( T, DT, HX, HY, HZ, OX, OY, OZ ) { 3, DT, HX, HY, HZ, OX, OY, OZ, &run3d< T, HX, HY, HZ, OX, OY, OZ > }

Entry const kTable[] = {
   // 2D sigma 2 (13 taps), sigma 1 (7 taps), mixed
   E2( float, DT_SFLOAT, 6, 6, 0, 0 ),
   E2( float, DT_SFLOAT, 3, 3, 0, 0 ),
   E2( float, DT_SFLOAT, 4, 3, 1, 0 ),
   E2( float, DT_SFLOAT, 3, 4, 0, 1 ),
   E2( uint16_t, DT_UINT16, 6, 6, 0, 0 ),
   E2( uint8_t, DT_UINT8, 6, 6, 0, 0 ),
   // 2D sigma 3: orders (0,0), (1,0), (0,1), (2,0)
   E2( float, DT_SFLOAT, 9, 9, 0, 0 ),
   E2( float, DT_SFLOAT, 11, 9, 1, 0 ),
   E2( float, DT_SFLOAT, 9, 11, 0, 1 ),
   E2( float, DT_SFLOAT, 12, 9, 0, 0 ),
   // 3D sigma (1.5, 1.5, 3): orders (0,0,0), (1,0,0)
   E3( uint16_t, DT_UINT16, 5, 5, 9, 0, 0, 0 ),
   E3( uint16_t, DT_UINT16, 6, 5, 9, 1, 0, 0 ),
   E3( float, DT_SFLOAT, 5, 5, 9, 0, 0, 0 ),
   // 3D sigma 1 gradients and smoothing
   E3( float, DT_SFLOAT, 4, 3, 3, 1, 0, 0 ),
   E3( float, DT_SFLOAT, 3, 4, 3, 0, 1, 0 ),
   E3( float, DT_SFLOAT, 3, 3, 4, 0, 0, 1 ),
   E3( float, DT_SFLOAT, 3, 3, 3, 0, 0, 0 ),
   // 3D sigma 4 smoothing (structure tensor)
   E3( float, DT_SFLOAT, 12, 12, 12, 0, 0, 0 ),
};

#undef E2
#undef E3

Entry const* find( FusedKey const& k ) {
   for( auto const& e : kTable ) {
      if( e.ndims != k.ndims || e.in_dt != k.in_dt ) { continue; }
      if( e.hx != k.h[ 0 ] || e.hy != k.h[ 1 ] || e.ox != k.odd[ 0 ] || e.oy != k.odd[ 1 ] ) { continue; }
      if( k.ndims == 3 && ( e.hz != k.h[ 2 ] || e.oz != k.odd[ 2 ] )) { continue; }
      return &e;
   }
   return nullptr;
}

} // namespace

bool fused_available( FusedKey const& key ) {
   return find( key ) != nullptr;
}

cudaError_t launch_fused( FusedKey const& key, FusedArgs& args, cudaStream_t stream ) {
   Entry const* e = find( key );
   if( !e ) { return cudaErrorNotSupported; }
   return e->run( args, stream );
}

} // namespace dipcu
