// Launchers and the instantiation table of the fused tile kernels (K1).  Each entry fixes the
// per-axis half-widths and symmetry at compile time so that the tap loops unroll fully and the
// weights are read as constant-bank operands; configurations without an entry run on the line
// kernel (K2).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include "fused.cuh"
#include "fused3d_tma.cuh"
#include "fused3d_ws.cuh"
#include "fused2d_ws.cuh"
#include "fused2d_adj.cuh"

namespace dipcu {

// Device status word: kernels that give up a bounded wait store DIPCU_ERR_TIMEOUT here.
__device__ int32_t g_device_status;

int32_t* device_status_ptr() {
   int dev = 0;
   cudaGetDevice( &dev );
   static std::mutex mu;
   static int32_t* ptrs[ 64 ] = {};
   std::lock_guard< std::mutex > lock( mu );
   if( dev < 0 || dev >= 64 ) { return nullptr; }
   if( !ptrs[ dev ] ) {
      void* p = nullptr;
      if( cudaGetSymbolAddress( &p, g_device_status ) != cudaSuccess ) { return nullptr; }
      ptrs[ dev ] = static_cast< int32_t* >( p );
   }
   return ptrs[ dev ];
}

namespace {

constexpr int kNT = 256;

int sm_count() {
   static int cached[ 64 ] = {};
   int dev = 0;
   cudaGetDevice( &dev );
   if( dev < 0 || dev >= 64 ) { return 148; }
   if( !cached[ dev ] ) {
      int n = 148;
      cudaDeviceGetAttribute( &n, cudaDevAttrMultiProcessorCount, dev );
      cached[ dev ] = n;
   }
   return cached[ dev ];
}

// Small cache of encoded tensor maps: encoding costs host microseconds per call, and the same
// images are filtered over and over.
struct TmapEntry {
   bool used;
   int device;
   void const* ptr;
   cuuint64_t dims[ 4 ], strides[ 3 ];
   cuuint32_t box[ 4 ];
   CUtensorMapDataType dt;
   CUtensorMap map;
   uint64_t stamp;
};

CUresult encode_tmap( CUtensorMap* out, CUtensorMapDataType dt, void const* ptr, cuuint64_t const* dims,
                      cuuint64_t const* strides, cuuint32_t const* box ) {
   static std::mutex mu;
   static TmapEntry cache[ 32 ];
   static uint64_t clock = 0;
   int dev = 0;
   cudaGetDevice( &dev );
   std::lock_guard< std::mutex > lock( mu );
   TmapEntry* victim = &cache[ 0 ];
   for( auto& e : cache ) {
      if( e.used && e.device == dev && e.ptr == ptr && e.dt == dt &&
          std::memcmp( e.dims, dims, sizeof( e.dims )) == 0 && std::memcmp( e.strides, strides, sizeof( e.strides )) == 0 &&
          std::memcmp( e.box, box, sizeof( e.box )) == 0 ) {
         e.stamp = ++clock;
         *out = e.map;
         return CUDA_SUCCESS;
      }
      if( !e.used || e.stamp < victim->stamp ) { victim = &e; }
   }
   // The driver entry point is resolved through the runtime, so that libdipcu.so has no
   // link-time dependency on libcuda (it loads on machines without a GPU driver).
   using EncodeFn = CUresult ( * )( CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, cuuint64_t const*,
                                    cuuint64_t const*, cuuint32_t const*, cuuint32_t const*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill );
   static EncodeFn encode = nullptr;
   if( !encode ) {
      void* fn = nullptr;
      cudaDriverEntryPointQueryResult q;
      if( cudaGetDriverEntryPoint( "cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q ) != cudaSuccess ||
          q != cudaDriverEntryPointSuccess || !fn ) {
         return CUDA_ERROR_NOT_FOUND;
      }
      encode = reinterpret_cast< EncodeFn >( fn );
   }
   cuuint32_t estr[ 4 ] = { 1, 1, 1, 1 };
   CUresult r = encode( out, dt, 4, const_cast< void* >( ptr ), dims, strides, box, estr,
                                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE );
   if( r != CUDA_SUCCESS ) { return r; }
   victim->used = true;
   victim->device = dev;
   victim->ptr = ptr;
   victim->dt = dt;
   std::memcpy( victim->dims, dims, sizeof( victim->dims ));
   std::memcpy( victim->strides, strides, sizeof( victim->strides ));
   std::memcpy( victim->box, box, sizeof( victim->box ));
   victim->map = *out;
   victim->stamp = ++clock;
   return CUDA_SUCCESS;
}

// Per-kernel, per-device launch set-up done once: the dynamic shared-memory opt-in and the
// number of co-resident CTAs per SM.
template< typename Kern >
int prepare_kernel( Kern kern, int threads, size_t smem ) {
   static std::mutex mu;
   static std::map< std::pair< void const*, int >, int > per_sm;
   int dev = 0;
   cudaGetDevice( &dev );
   auto key = std::make_pair( reinterpret_cast< void const* >( kern ), dev );
   std::lock_guard< std::mutex > lock( mu );
   auto it = per_sm.find( key );
   if( it != per_sm.end() ) { return it->second; }
   if( smem > 48 * 1024 &&
       cudaFuncSetAttribute( kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( smem )) != cudaSuccess ) {
      return -1;
   }
   int n = 0;
   if( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &n, kern, threads, smem ) != cudaSuccess || n < 1 ) { return -1; }
   per_sm[ key ] = n;
   return n;
}

// TMA-pipelined 3D kernel; returns cudaErrorNotSupported when the layout does not allow TMA
// (negative or unaligned strides), so that the caller falls back to the plain-load kernel.
template< typename TIn, int HX, int HY, int HZ, bool OX, bool OY, bool OZ >
cudaError_t run3d_tma( FusedArgs& a, cudaStream_t s ) {
   using G = Z3Geom< TIn, HX, HY, HZ >;
   constexpr int esz = sizeof( TIn );
   if( a.ss[ 1 ] <= 0 || a.ss[ 2 ] <= 0 || ( a.nb > 1 && a.sb <= 0 )) { return cudaErrorNotSupported; }
   if(( reinterpret_cast< uintptr_t >( a.src ) & 15 ) != 0 ) { return cudaErrorNotSupported; }
   if(( a.ss[ 1 ] * esz ) % 16 || ( a.ss[ 2 ] * esz ) % 16 || ( a.nb > 1 && ( a.sb * esz ) % 16 )) { return cudaErrorNotSupported; }
   if( a.n[ 0 ] > 0x7fffffff || a.n[ 1 ] > 0x7fffffff || a.n[ 2 ] > 0x7fffffff || a.nb > 0x7fffffff ) { return cudaErrorNotSupported; }
   Z3Args z{};
   CUtensorMapDataType dt = sizeof( TIn ) == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                          : sizeof( TIn ) == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
   cuuint64_t dims[ 4 ] = { static_cast< cuuint64_t >( a.n[ 0 ] ), static_cast< cuuint64_t >( a.n[ 1 ] ),
                            static_cast< cuuint64_t >( a.n[ 2 ] ), static_cast< cuuint64_t >( a.nb ) };
   cuuint64_t strides[ 3 ] = { static_cast< cuuint64_t >( a.ss[ 1 ] * esz ), static_cast< cuuint64_t >( a.ss[ 2 ] * esz ),
                               static_cast< cuuint64_t >(( a.nb > 1 ? a.sb : a.ss[ 2 ] * a.n[ 2 ] ) * esz ) };
   if( strides[ 2 ] % 16 ) { strides[ 2 ] = ( strides[ 2 ] + 15 ) / 16 * 16; }
   cuuint32_t box[ 4 ] = { static_cast< cuuint32_t >( G::WXA ), static_cast< cuuint32_t >( G::WY ), 1, 1 };
   if( encode_tmap( &z.tmap, dt, a.src, dims, strides, box ) != CUDA_SUCCESS ) { return cudaErrorNotSupported; }
   z.src = a.src;
   z.dst = a.dst;
   for( int i = 0; i < 3; ++i ) {
      z.n[ i ] = a.n[ i ];
      z.ss[ i ] = a.ss[ i ];
      z.ds[ i ] = a.ds[ i ];
      z.bc[ i ] = a.bc[ i ];
      for( int k = 0; k < kFusedMaxTaps; ++k ) { z.w[ i ][ k ] = make_float2( a.w[ i ][ k ], a.w[ i ][ k ] ); }
   }
   z.nb = a.nb;
   z.sb = a.sb;
   z.db = a.db;
   z.tiles_x = static_cast< int32_t >(( a.n[ 0 ] + G::TX - 1 ) / G::TX );
   z.tiles_y = static_cast< int32_t >(( a.n[ 1 ] + G::TY - 1 ) / G::TY );
   z.units = static_cast< int64_t >( z.tiles_x ) * z.tiles_y * a.nb * a.n[ 2 ];
   z.status = device_status_ptr();
   if( !z.status ) { return cudaErrorUnknown; }
   auto kern = fused3d_tma_kernel< TIn, HX, HY, HZ, OX, OY, OZ >;
   size_t smem = G::BYTES;
   int per_sm = prepare_kernel( kern, G::NT, smem );
   if( per_sm < 1 ) { return cudaErrorInvalidConfiguration; }
   static int const want = getenv( "DIPCU_Z3_CTAS_PER_SM" ) ? atoi( getenv( "DIPCU_Z3_CTAS_PER_SM" )) : 2;
   if( per_sm > want ) { per_sm = want; }
   if( per_sm < 1 ) { per_sm = 1; }
   int64_t nctas = static_cast< int64_t >( sm_count() ) * per_sm;
   int64_t max_ctas = z.units / ( 4 * HZ + 4 );   // keep chunks long against the 2*HZ halo planes
   if( nctas > max_ctas ) { nctas = max_ctas; }
   if( nctas < 1 ) { nctas = 1; }
   kern<<< static_cast< unsigned >( nctas ), G::NT, smem, s >>>( z ); count_launch();
   return cudaGetLastError();
}

// Warp-specialised 3D kernel; cudaErrorNotSupported when its conditions do not hold (TMA layout,
// x-y boundary conditions whose halo sources leave the box), so that the caller falls back.
template< typename TIn, int HX, int HY, int HZ, bool OX, bool OY, bool OZ >
cudaError_t run3d_ws( FusedArgs& a, cudaStream_t s ) {
   using G = W5Geom< TIn, HX, HY, HZ >;
   if constexpr( !G::fits ) {
      return cudaErrorNotSupported;
   } else {
      constexpr int esz = sizeof( TIn );
      if( a.ss[ 1 ] <= 0 || a.ss[ 2 ] <= 0 || ( a.nb > 1 && a.sb <= 0 )) { return cudaErrorNotSupported; }
      if(( reinterpret_cast< uintptr_t >( a.src ) & 15 ) != 0 ) { return cudaErrorNotSupported; }
      if(( a.ss[ 1 ] * esz ) % 16 || ( a.ss[ 2 ] * esz ) % 16 || ( a.nb > 1 && ( a.sb * esz ) % 16 )) { return cudaErrorNotSupported; }
      if( a.n[ 0 ] > 0x3fffffff || a.n[ 1 ] > 0x3fffffff || a.n[ 2 ] > 0x3fffffff || a.nb > 0x3fffffff ) { return cudaErrorNotSupported; }
      bool const flt = std::is_same< TIn, float >::value;
      for( int d = 0; d < 2; ++d ) {
         int32_t const bc = a.bc[ d ];
         bool ok = bc == BC_SYMMETRIC_MIRROR || bc == BC_ZERO_ORDER_EXTRAPOLATE || bc == BC_ADD_ZEROS ||
                   ( flt && bc == BC_ASYMMETRIC_MIRROR );
         int64_t const h = d == 0 ? HX : HY;
         if( !ok || a.n[ d ] <= h ) { return cudaErrorNotSupported; }   // single reflection: sources in the box
      }
      if( !bc_is_index_map( a.bc[ 2 ] )) { return cudaErrorNotSupported; }
      W5Args z{};
      CUtensorMapDataType dt = sizeof( TIn ) == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
      cuuint64_t dims[ 4 ] = { static_cast< cuuint64_t >( a.n[ 0 ] ), static_cast< cuuint64_t >( a.n[ 1 ] ),
                               static_cast< cuuint64_t >( a.n[ 2 ] ), static_cast< cuuint64_t >( a.nb ) };
      cuuint64_t strides[ 3 ] = { static_cast< cuuint64_t >( a.ss[ 1 ] * esz ), static_cast< cuuint64_t >( a.ss[ 2 ] * esz ),
                                  static_cast< cuuint64_t >(( a.nb > 1 ? a.sb : a.ss[ 2 ] * a.n[ 2 ] ) * esz ) };
      if( strides[ 2 ] % 16 ) { strides[ 2 ] = ( strides[ 2 ] + 15 ) / 16 * 16; }
      cuuint32_t box1[ 4 ] = { static_cast< cuuint32_t >( G::BW ), static_cast< cuuint32_t >( G::BH ), 1, 1 };
      cuuint32_t box2[ 4 ] = { static_cast< cuuint32_t >( G::BW ), static_cast< cuuint32_t >( G::BH ), a.n[ 2 ] >= 2 ? 2u : 1u, 1 };
      if( encode_tmap( &z.tmap1, dt, a.src, dims, strides, box1 ) != CUDA_SUCCESS ||
          encode_tmap( &z.tmap2, dt, a.src, dims, strides, box2 ) != CUDA_SUCCESS ) {
         return cudaErrorNotSupported;
      }
      z.dst = a.dst;
      for( int i = 0; i < 3; ++i ) {
         z.n[ i ] = static_cast< int32_t >( a.n[ i ] );
         z.ds[ i ] = a.ds[ i ];
         z.bc[ i ] = a.bc[ i ];
         for( int k = 0; k < kFusedMaxTaps; ++k ) { z.w[ i ][ k ] = make_float2( a.w[ i ][ k ], a.w[ i ][ k ] ); }
      }
      z.nb = static_cast< int32_t >( a.nb );
      z.db = a.db;
      z.vec_store = (( reinterpret_cast< uintptr_t >( a.dst ) & 7 ) == 0 && a.ds[ 1 ] % 2 == 0 && a.ds[ 2 ] % 2 == 0 &&
                     ( a.nb <= 1 || a.db % 2 == 0 )) ? 1 : 0;
      z.tiles_x = static_cast< int32_t >(( a.n[ 0 ] + G::OFF + G::TX - 1 ) / G::TX );
      z.tiles_y = static_cast< int32_t >(( a.n[ 1 ] + G::TY - 1 ) / G::TY );
      z.units = static_cast< int64_t >( z.tiles_x ) * z.tiles_y * a.nb * a.n[ 2 ];
      z.status = device_status_ptr();
      if( !z.status ) { return cudaErrorUnknown; }
      auto kern = fused3d_ws_kernel< TIn, HX, HY, HZ, OX, OY, OZ >;
      size_t smem = G::BYTES;
      int per_sm = prepare_kernel( kern, G::NT, smem );
      if( per_sm < 1 ) { return cudaErrorInvalidConfiguration; }
      static int const want = getenv( "DIPCU_W5_CTAS_PER_SM" ) ? atoi( getenv( "DIPCU_W5_CTAS_PER_SM" )) : 4;
      if( per_sm > want ) { per_sm = want; }
      if( per_sm < 1 ) { per_sm = 1; }
      int64_t nctas = static_cast< int64_t >( sm_count() ) * per_sm;
      int64_t max_ctas = z.units / ( 4 * HZ + 4 );   // keep chunks long against the 2*HZ halo planes
      if( nctas > max_ctas ) { nctas = max_ctas; }
      if( nctas < 1 ) { nctas = 1; }
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3( static_cast< unsigned >( nctas ));
      cfg.blockDim = dim3( G::NT );
      cfg.dynamicSmemBytes = smem;
      cfg.stream = s;
      cudaLaunchAttribute attr[ 1 ];
      attr[ 0 ].id = cudaLaunchAttributeProgrammaticStreamSerialization;   // see the 2D launch
      attr[ 0 ].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      cudaError_t const le = cudaLaunchKernelEx( &cfg, kern, z );
      count_launch();
      if( le != cudaSuccess ) { return le; }
      return cudaGetLastError();
   }
}

// Warp-per-tile 2D kernel for half-widths up to B on both axes (taps zero beyond each axis' h);
// cudaErrorNotSupported when its conditions do not hold, so that the caller falls back.
template< typename TIn, int B >
cudaError_t run2d_ws( FusedArgs& a, int32_t const* odd, cudaStream_t s ) {
   constexpr int TYP = 32;
   using G = W2Geom< TIn, B, TYP >;
   static_assert( G::fits, "shared memory" );
   constexpr int esz = sizeof( TIn );
   if( a.ss[ 0 ] != 1 || a.ss[ 1 ] <= 0 || ( a.nb > 1 && a.sb <= 0 )) { return cudaErrorNotSupported; }
   if(( reinterpret_cast< uintptr_t >( a.src ) & 15 ) != 0 ) { return cudaErrorNotSupported; }
   if(( a.ss[ 1 ] * esz ) % 16 || ( a.nb > 1 && ( a.sb * esz ) % 16 )) { return cudaErrorNotSupported; }
   if( a.n[ 0 ] > 0x3fffffff || a.n[ 1 ] > 0x3fffffff || a.nb > 0x3fffffff ) { return cudaErrorNotSupported; }
   bool const flt = std::is_same< TIn, float >::value;
   for( int d = 0; d < 2; ++d ) {
      int32_t const bc = a.bc[ d ];
      bool ok = bc == BC_SYMMETRIC_MIRROR || bc == BC_ZERO_ORDER_EXTRAPOLATE || bc == BC_ADD_ZEROS ||
                ( flt && bc == BC_ASYMMETRIC_MIRROR );
      if( !ok || a.n[ d ] <= B ) { return cudaErrorNotSupported; }
   }
   W2Args z{};
   CUtensorMapDataType dt = sizeof( TIn ) == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
   cuuint64_t dims[ 4 ] = { static_cast< cuuint64_t >( a.n[ 0 ] ), static_cast< cuuint64_t >( a.n[ 1 ] ), 1,
                            static_cast< cuuint64_t >( a.nb ) };
   cuuint64_t strides[ 3 ] = { static_cast< cuuint64_t >( a.ss[ 1 ] * esz ),
                               static_cast< cuuint64_t >( a.ss[ 1 ] * a.n[ 1 ] * esz ),
                               static_cast< cuuint64_t >(( a.nb > 1 ? a.sb : a.ss[ 1 ] * a.n[ 1 ] ) * esz ) };
   for( auto& v : strides ) { if( v % 16 ) { v = ( v + 15 ) / 16 * 16; } }
   cuuint32_t box[ 4 ] = { static_cast< cuuint32_t >( G::BW ), static_cast< cuuint32_t >( G::BH ), 1, 1 };
   if( encode_tmap( &z.tmap, dt, a.src, dims, strides, box ) != CUDA_SUCCESS ) { return cudaErrorNotSupported; }
   z.dst = a.dst;
   // TMA stores of whole tiles when the destination layout allows them.
   z.tma_store = 0;
   if( a.ds[ 0 ] == 1 && a.ds[ 1 ] > 0 && ( reinterpret_cast< uintptr_t >( a.dst ) & 15 ) == 0 && ( a.ds[ 1 ] * 4 ) % 16 == 0 &&
       ( a.nb <= 1 || ( a.db > 0 && ( a.db * 4 ) % 16 == 0 )) && !getenv( "DIPCU_NO_TMA_STORE" )) {
      cuuint64_t od[ 4 ] = { static_cast< cuuint64_t >( a.n[ 0 ] ), static_cast< cuuint64_t >( a.n[ 1 ] ), 1,
                             static_cast< cuuint64_t >( a.nb ) };
      cuuint64_t os[ 3 ] = { static_cast< cuuint64_t >( a.ds[ 1 ] * 4 ), static_cast< cuuint64_t >( a.ds[ 1 ] * a.n[ 1 ] * 4 ),
                             static_cast< cuuint64_t >(( a.nb > 1 ? a.db : a.ds[ 1 ] * a.n[ 1 ] ) * 4 ) };
      for( auto& v : os ) { if( v % 16 ) { v = ( v + 15 ) / 16 * 16; } }
      cuuint32_t ob[ 4 ] = { static_cast< cuuint32_t >( G::TX ), static_cast< cuuint32_t >( G::TY ), 1, 1 };
      if( encode_tmap( &z.tout, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a.dst, od, os, ob ) == CUDA_SUCCESS ) { z.tma_store = 1; }
   }
   for( int i = 0; i < 2; ++i ) {
      z.n[ i ] = static_cast< int32_t >( a.n[ i ] );
      z.ds[ i ] = a.ds[ i ];
      z.bc[ i ] = a.bc[ i ];
      float const sg = odd[ i ] ? -1.f : 1.f;
      z.sgn[ i ] = make_float2( sg, sg );
      for( int k = 0; k < kFusedMaxTaps; ++k ) { z.w[ i ][ k ] = make_float2( a.w[ i ][ k ], a.w[ i ][ k ] ); }
   }
   z.nb = static_cast< int32_t >( a.nb );
   z.db = a.db;
   z.vec_store = (( reinterpret_cast< uintptr_t >( a.dst ) & 7 ) == 0 && a.ds[ 1 ] % 2 == 0 &&
                  ( a.nb <= 1 || a.db % 2 == 0 )) ? 1 : 0;
   z.tiles_x = static_cast< int32_t >(( a.n[ 0 ] + G::OFF + G::TX - 1 ) / G::TX );
   z.tiles_y = static_cast< int32_t >(( a.n[ 1 ] + G::TY - 1 ) / G::TY );
   z.ntiles = static_cast< int64_t >( z.tiles_x ) * z.tiles_y * a.nb;
   z.status = device_status_ptr();
   if( !z.status ) { return cudaErrorUnknown; }
   auto kern = fused2d_ws_kernel< TIn, B, TYP >;
   size_t smem = G::BYTES;
   int per_sm = prepare_kernel( kern, G::NT, smem );
   if( per_sm < 1 ) { return cudaErrorInvalidConfiguration; }
   int64_t nctas = static_cast< int64_t >( sm_count() ) * per_sm;
   int64_t const need = ( z.ntiles + G::NW - 1 ) / G::NW;
   if( nctas > need ) { nctas = need; }
   if( nctas < 1 ) { nctas = 1; }
   {
      // launched as a programmatic dependent of the previous kernel in the stream (the kernel waits
      // for it before touching memory), so consecutive filters overlap their launch latency
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3( static_cast< unsigned >( nctas ));
      cfg.blockDim = dim3( G::NT );
      cfg.dynamicSmemBytes = smem;
      cfg.stream = s;
      cudaLaunchAttribute attr[ 1 ];
      attr[ 0 ].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[ 0 ].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      cudaError_t const le = cudaLaunchKernelEx( &cfg, kern, z );
      count_launch();
      if( le != cudaSuccess ) { return le; }
   }
   return cudaGetLastError();
}

template< typename TIn, int B >
cudaError_t run_adj2d( Adj2Params const& p, cudaStream_t s ) {
   using G = A2Geom< TIn, B >;
   static_assert( G::fits, "shared memory" );
   bool const sig = p.x != nullptr && p.dsig[ 0 ] && p.dsig[ 1 ];
   if( p.gys1 <= 0 || ( p.nb > 1 && p.gyb <= 0 )) { return cudaErrorNotSupported; }
   if(( reinterpret_cast< uintptr_t >( p.gy ) & 15 ) || ( p.gys1 * 4 ) % 16 || ( p.nb > 1 && ( p.gyb * 4 ) % 16 )) {
      return cudaErrorNotSupported;
   }
   constexpr int esz = sizeof( TIn );
   if( sig && (( reinterpret_cast< uintptr_t >( p.x ) & 15 ) || p.xs1 <= 0 || ( p.xs1 * esz ) % 16 ||
               ( p.nb > 1 && ( p.xb <= 0 || ( p.xb * esz ) % 16 )))) {
      return cudaErrorNotSupported;
   }
   if( p.n[ 0 ] > 0x3fffffff || p.n[ 1 ] > 0x3fffffff || p.nb > 0x3fffffff ) { return cudaErrorNotSupported; }
   for( int d = 0; d < 2; ++d ) {
      int32_t const bc = p.bc[ d ];
      bool ok = bc == BC_SYMMETRIC_MIRROR || bc == BC_ZERO_ORDER_EXTRAPOLATE || bc == BC_ADD_ZEROS || bc == BC_ASYMMETRIC_MIRROR;
      if( !ok || p.n[ d ] <= B || p.h[ d ] > B || p.h[ d ] < 1 ) { return cudaErrorNotSupported; }
   }
   A2Args z{};
   {
      cuuint64_t dims[ 4 ] = { static_cast< cuuint64_t >( p.n[ 0 ] ), static_cast< cuuint64_t >( p.n[ 1 ] ), 1,
                               static_cast< cuuint64_t >( p.nb ) };
      cuuint64_t st[ 3 ] = { static_cast< cuuint64_t >( p.gys1 * 4 ), static_cast< cuuint64_t >( p.gys1 * p.n[ 1 ] * 4 ),
                             static_cast< cuuint64_t >(( p.nb > 1 ? p.gyb : p.gys1 * p.n[ 1 ] ) * 4 ) };
      for( auto& v : st ) { if( v % 16 ) { v = ( v + 15 ) / 16 * 16; } }
      cuuint32_t box[ 4 ] = { static_cast< cuuint32_t >( G::BW ), static_cast< cuuint32_t >( G::BH ), 1, 1 };
      if( encode_tmap( &z.tg, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.gy, dims, st, box ) != CUDA_SUCCESS ) { return cudaErrorNotSupported; }
   }
   if( sig ) {
      cuuint64_t dims[ 4 ] = { static_cast< cuuint64_t >( p.n[ 0 ] ), static_cast< cuuint64_t >( p.n[ 1 ] ), 1,
                               static_cast< cuuint64_t >( p.nb ) };
      cuuint64_t st[ 3 ] = { static_cast< cuuint64_t >( p.xs1 * esz ), static_cast< cuuint64_t >( p.xs1 * p.n[ 1 ] * esz ),
                             static_cast< cuuint64_t >(( p.nb > 1 ? p.xb : p.xs1 * p.n[ 1 ] ) * esz ) };
      for( auto& v : st ) { if( v % 16 ) { v = ( v + 15 ) / 16 * 16; } }
      cuuint32_t box[ 4 ] = { static_cast< cuuint32_t >( G::TX ), static_cast< cuuint32_t >( G::TY ), 1, 1 };
      CUtensorMapDataType dt = esz == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
      if( encode_tmap( &z.tx, dt, p.x, dims, st, box ) != CUDA_SUCCESS ) { return cudaErrorNotSupported; }
   }
   z.gx = p.gx;
   z.tma_store = 0;
   if( p.gx && p.gxs1 > 0 && ( reinterpret_cast< uintptr_t >( p.gx ) & 15 ) == 0 && ( p.gxs1 * 4 ) % 16 == 0 &&
       ( p.nb <= 1 || ( p.gxb > 0 && ( p.gxb * 4 ) % 16 == 0 )) && !getenv( "DIPCU_NO_TMA_STORE" )) {
      cuuint64_t od[ 4 ] = { static_cast< cuuint64_t >( p.n[ 0 ] ), static_cast< cuuint64_t >( p.n[ 1 ] ), 1,
                             static_cast< cuuint64_t >( p.nb ) };
      cuuint64_t os[ 3 ] = { static_cast< cuuint64_t >( p.gxs1 * 4 ), static_cast< cuuint64_t >( p.gxs1 * p.n[ 1 ] * 4 ),
                             static_cast< cuuint64_t >(( p.nb > 1 ? p.gxb : p.gxs1 * p.n[ 1 ] ) * 4 ) };
      for( auto& v : os ) { if( v % 16 ) { v = ( v + 15 ) / 16 * 16; } }
      cuuint32_t ob[ 4 ] = { static_cast< cuuint32_t >( G::TX ), static_cast< cuuint32_t >( G::TY ), 1, 1 };
      if( encode_tmap( &z.tgx, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.gx, od, os, ob ) == CUDA_SUCCESS ) { z.tma_store = 1; }
   }
   z.dsig[ 0 ] = sig ? p.dsig[ 0 ] : nullptr;
   z.dsig[ 1 ] = sig ? p.dsig[ 1 ] : nullptr;
   z.nb = static_cast< int32_t >( p.nb );
   z.gs1 = p.gxs1;
   z.gb = p.gxb;
   for( int d = 0; d < 2; ++d ) {
      z.n[ d ] = static_cast< int32_t >( p.n[ d ] );
      z.bc[ d ] = p.bc[ d ];
      z.h[ d ] = p.h[ d ];
      float const sg = p.odd[ d ] ? -1.f : 1.f;
      z.s[ d ] = make_float2( sg, sg );
      for( int k = 0; k <= p.h[ d ]; ++k ) {
         // C^T in the forward's pair form: the flipped taps of an odd kernel are its negation.
         float const w = static_cast< float >( p.taps[ d ][ k ] ) * ( k > 0 ? sg : 1.f );
         z.w[ d ][ k ] = make_float2( w, w );
         if( sig ) {
            float const wd = static_cast< float >( p.dtaps[ d ][ k ] ) * ( k > 0 ? sg : 1.f );
            z.wd[ d ][ k ] = make_float2( wd, wd );
         }
      }
   }
   z.vec_store = p.gx && (( reinterpret_cast< uintptr_t >( p.gx ) & 7 ) == 0 && p.gxs1 % 2 == 0 && ( p.nb <= 1 || p.gxb % 2 == 0 )) ? 1 : 0;
   z.tiles_x = static_cast< int32_t >(( p.n[ 0 ] + G::TX - 1 ) / G::TX );
   z.tiles_y = static_cast< int32_t >(( p.n[ 1 ] + G::TY - 1 ) / G::TY );
   z.ntiles = static_cast< int64_t >( z.tiles_x ) * z.tiles_y * p.nb;
   z.status = device_status_ptr();
   if( !z.status ) { return cudaErrorUnknown; }
   auto kern = fused2d_adj_kernel< TIn, B >;
   size_t smem = G::BYTES;
   int per_sm = prepare_kernel( kern, G::NT, smem );
   if( per_sm < 1 ) { return cudaErrorInvalidConfiguration; }
   int64_t nctas = static_cast< int64_t >( sm_count() ) * per_sm;
   int64_t const need = ( z.ntiles + G::NW - 1 ) / G::NW;
   if( nctas > need ) { nctas = need; }
   if( nctas < 1 ) { nctas = 1; }
   kern<<< static_cast< unsigned >( nctas ), G::NT, smem, s >>>( z ); count_launch();
   return cudaGetLastError();
}

template< typename TIn >
cudaError_t run_adj2d_bucket( Adj2Params const& p, cudaStream_t s ) {
   int const hm = p.h[ 0 ] > p.h[ 1 ] ? p.h[ 0 ] : p.h[ 1 ];
   if( hm <= 4 ) { return run_adj2d< TIn, 4 >( p, s ); }
   if( hm <= 6 ) { return run_adj2d< TIn, 6 >( p, s ); }
   if( hm <= 9 ) { return run_adj2d< TIn, 9 >( p, s ); }
   if( hm <= 12 ) { return run_adj2d< TIn, 12 >( p, s ); }
   return cudaErrorNotSupported;
}

template< typename TIn >
cudaError_t run2d_ws_bucket( FusedArgs& a, int32_t const* h, int32_t const* odd, cudaStream_t s ) {
   int const hm = h[ 0 ] > h[ 1 ] ? h[ 0 ] : h[ 1 ];
   if( hm <= 4 ) { return run2d_ws< TIn, 4 >( a, odd, s ); }
   if( hm <= 6 ) { return run2d_ws< TIn, 6 >( a, odd, s ); }
   if( hm <= 9 ) { return run2d_ws< TIn, 9 >( a, odd, s ); }
   if( hm <= 12 ) { return run2d_ws< TIn, 12 >( a, odd, s ); }
   return cudaErrorNotSupported;
}

template< typename TIn, int HX, int HY, bool OX, bool OY >
cudaError_t run2d( FusedArgs& a, cudaStream_t s ) {
   constexpr int TX = 64, TY = 32, RX = 4, RY = 8;
   using L = TileLayout< TX, TY, HX, HY >;
   auto kern = fused2d_kernel< TIn, HX, HY, OX, OY, TX, TY, RX, RY, kNT >;
   size_t smem = L::bytes();
   if( prepare_kernel( kern, kNT, smem ) < 1 ) { return cudaErrorInvalidConfiguration; }
   a.tiles_x = static_cast< int32_t >(( a.n[ 0 ] + TX - 1 ) / TX);
   a.tiles_y = static_cast< int32_t >(( a.n[ 1 ] + TY - 1 ) / TY);
   a.zchunks = 1;
   a.lz = 1;
   int64_t grid = static_cast< int64_t >( a.tiles_x ) * a.tiles_y * a.nb;
   if( grid > 0x7fffffff ) { return cudaErrorInvalidValue; }
   kern<<< static_cast< unsigned >( grid ), kNT, smem, s >>>( a ); count_launch();
   return cudaGetLastError();
}

template< typename TIn, int HX, int HY, int HZ, bool OX, bool OY, bool OZ >
cudaError_t run3d( FusedArgs& a, cudaStream_t s ) {
   if( !getenv( "DIPCU_NO_TMA" )) {
      if constexpr( sizeof( TIn ) == 2 || std::is_same< TIn, float >::value ) {
         if( !getenv( "DIPCU_NO_WS" )) {
            cudaError_t e = run3d_ws< TIn, HX, HY, HZ, OX, OY, OZ >( a, s );
            if( e != cudaErrorNotSupported ) { return e; }
         }
      }
      cudaError_t e = run3d_tma< TIn, HX, HY, HZ, OX, OY, OZ >( a, s );
      if( e != cudaErrorNotSupported ) { return e; }
   }
   constexpr int TX = 64, TY = 16, RY = 8;
   using L = TileLayout< TX, TY, HX, HY >;
   auto kern = fused3d_kernel< TIn, HX, HY, HZ, OX, OY, OZ, TX, TY, RY, kNT >;
   size_t smem = L::bytes();
   if( prepare_kernel( kern, kNT, smem ) < 1 ) { return cudaErrorInvalidConfiguration; }
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
   kern<<< static_cast< unsigned >( grid ), kNT, smem, s >>>( a ); count_launch();
   return cudaGetLastError();
}

using Runner = cudaError_t ( * )( FusedArgs&, cudaStream_t );

struct Entry {
   int32_t ndims, in_dt, hx, hy, hz, ox, oy, oz;
   Runner run;
};

// (input type, half-widths, odd flags) instantiated ahead of time.  The set covers the
// benchmark workloads (2D sigma 2; 2D sigma 3 orders 0..2; 3D sigma (1.5, 1.5, 3) orders
// (0,0,0)/(1,0,0); the structure tensor's sigma 1 gradients) and small-sigma configurations
// used by the parity tests.
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
   // (3D sigma 4, half-width 12 on every axis, runs faster as three fast line passes than on the
   // previous tile kernel, the warp-specialised one not fitting its ring: no entry.)
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

CUresult encode_source_map( CUtensorMap* out, CUtensorMapDataType dt, void const* ptr, cuuint64_t const* dims,
                            cuuint64_t const* strides, cuuint32_t const* box ) {
   return encode_tmap( out, dt, ptr, dims, strides, box );
}

cudaError_t launch_fused2d_ws( FusedKey const& key, FusedArgs& args, cudaStream_t stream ) {
   if( key.ndims != 2 || getenv( "DIPCU_NO_WS" )) { return cudaErrorNotSupported; }
   if( key.in_dt == DT_SFLOAT ) { return run2d_ws_bucket< float >( args, key.h, key.odd, stream ); }
   if( key.in_dt == DT_UINT16 ) { return run2d_ws_bucket< uint16_t >( args, key.h, key.odd, stream ); }
   return cudaErrorNotSupported;
}

cudaError_t launch_fused_adjoint2d( Adj2Params const& p, cudaStream_t stream ) {
   if( getenv( "DIPCU_NO_WS" )) { return cudaErrorNotSupported; }
   if( !p.x || p.x_dt == DT_SFLOAT ) { return run_adj2d_bucket< float >( p, stream ); }
   if( p.x_dt == DT_UINT16 ) { return run_adj2d_bucket< uint16_t >( p, stream ); }
   return cudaErrorNotSupported;
}

bool fused_available( FusedKey const& key ) {
   return find( key ) != nullptr;
}

cudaError_t launch_fused( FusedKey const& key, FusedArgs& args, cudaStream_t stream ) {
   Entry const* e = find( key );
   if( !e ) { return cudaErrorNotSupported; }
   return e->run( args, stream );
}

} // namespace dipcu
