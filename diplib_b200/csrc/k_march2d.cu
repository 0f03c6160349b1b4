// Launchers of the row-march 2D kernel (march2d.cuh): for single images (with an optional batch
// axis) and for the item lists of a batch plan.  Checks of the layouts and boundary conditions it
// takes, the two TMA maps per image, and the single-image work split (strips of 128 columns times
// row runs, sized so that the persistent grid's two CTAs per SM get whole waves of items).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdlib>
#include <map>
#include <mutex>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"
#include "march2d.cuh"

namespace dipcu {

int32_t* device_status_ptr();

namespace {

int sm_count() {
   static int n = 0;
   if( n == 0 ) {
      int dev = 0;
      cudaGetDevice( &dev );
      int v = 0;
      cudaDeviceGetAttribute( &v, cudaDevAttrMultiProcessorCount, dev );
      n = v > 0 ? v : 148;
   }
   return n;
}

template< typename TIn >
bool march2d_ready() {
   static std::mutex mu;
   static std::map< int, bool > ok;
   int dev = 0;
   cudaGetDevice( &dev );
   std::lock_guard< std::mutex > lock( mu );
   auto it = ok.find( dev );
   if( it != ok.end() ) { return it->second; }
   bool r = cudaFuncSetAttribute( march2d_kernel< TIn >, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  M2Smem::BYTES ) == cudaSuccess;
   ok[ dev ] = r;
   return r;
}

bool bc_marchable( int32_t bc, bool is_float ) {
   switch( bc ) {
      case BC_SYMMETRIC_MIRROR: case BC_PERIODIC: case BC_ZERO_ORDER_EXTRAPOLATE: case BC_ADD_ZEROS: return true;
      case BC_ASYMMETRIC_MIRROR: case BC_ASYMMETRIC_PERIODIC: return is_float;   // negated samples in the stage
      default: return false;
   }
}

// Row runs per strip for `units` = (batch x strips) strip columns of `ny` rows: the number of
// runs that minimises the estimated time (waves over the persistent grid times the rows a run's
// x phase processes, halo included).
int march2d_chunks( int64_t units, int64_t ny, int hy, int slots ) {
   int best = 1;
   double best_t = 1e300;
   int const max_c = static_cast< int >( ny < 4096 ? ny : 4096 );
   for( int c = 1; c <= max_c; ++c ) {
      int64_t const l = ( ny + c - 1 ) / c;
      if( c > 1 && l < 16 ) { break; }
      int64_t const items = units * (( ny + l - 1 ) / l );
      int64_t const waves = ( items + slots - 1 ) / slots;
      double const t = static_cast< double >( waves ) * static_cast< double >( l + 2 * hy + 8 );
      if( t < best_t * 0.999 ) { best_t = t; best = c; }
   }
   return best;
}

} // namespace

template< typename TIn >
bool march2d_image( M2Image& im, void const* src, int64_t nx, int64_t ny, int64_t ss1, int64_t nb, int64_t ssb,
                    float* dst, int64_t ds1, int64_t dsb, int32_t const bc[ 2 ], int32_t const h[ 2 ], int32_t const odd[ 2 ] ) {
   constexpr int esz = sizeof( TIn );
   constexpr int A = 16 / esz;
   if( h[ 0 ] > kM2MaxH || h[ 1 ] > kM2MaxH || h[ 0 ] < 0 || h[ 1 ] < 0 ) { return false; }
   if( nx < 1 || ny < 1 || nx > 0x7fffffff || ny > 0x7fffffff || nb < 1 || nb > 0x7fffffff ) { return false; }
   if( ss1 <= 0 || ( nb > 1 && ssb <= 0 )) { return false; }
   bool const is_float = std::is_same< TIn, float >::value;
   bool const tma_ok = ( reinterpret_cast< uintptr_t >( src ) & 15 ) == 0 && ( ss1 * esz ) % 16 == 0 &&
                       ( nb <= 1 || ( ssb * esz ) % 16 == 0 );
   // Rows TMA cannot address: float images take the per-thread copy path.
   if( !tma_ok && !( is_float && ( reinterpret_cast< uintptr_t >( src ) & 3 ) == 0 )) { return false; }
   if( !bc_marchable( bc[ 0 ], is_float ) || !bc_marchable( bc[ 1 ], is_float )) { return false; }
   im = M2Image{};
   im.tma = tma_ok ? 1 : 0;
   im.lead = ( h[ 0 ] + A - 1 ) / A * A;
   if( im.lead < A ) { im.lead = A; }
   im.bw = kM2TX + 2 * im.lead;
   if( im.bw > kM2MaxBW ) { return false; }
   CUtensorMapDataType dt = esz == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
   cuuint64_t dims[ 4 ] = { static_cast< cuuint64_t >( nx ), static_cast< cuuint64_t >( ny ), 1,
                            static_cast< cuuint64_t >( nb ) };
   cuuint64_t strides[ 3 ] = { static_cast< cuuint64_t >( ss1 * esz ), static_cast< cuuint64_t >( ss1 * esz * ny ),
                               static_cast< cuuint64_t >(( nb > 1 ? ssb : ss1 * ny ) * esz ) };
   cuuint32_t box[ 4 ] = { static_cast< cuuint32_t >( im.bw ), static_cast< cuuint32_t >( kM2R ), 1, 1 };
   if( im.tma ) {
      if( encode_source_map( &im.tmap, dt, src, dims, strides, box ) != CUDA_SUCCESS ) { return false; }
      box[ 1 ] = 1;
      if( encode_source_map( &im.tmap1, dt, src, dims, strides, box ) != CUDA_SUCCESS ) { return false; }
   }
   im.src = src;
   im.ss1 = ss1;
   im.ssb = ssb;
   im.dst = dst;
   im.ds1 = ds1;
   im.dsb = dsb;
   im.vec_out = (( reinterpret_cast< uintptr_t >( dst ) & 7 ) == 0 && ds1 % 2 == 0 && ( nb <= 1 || dsb % 2 == 0 )) ? 1 : 0;
   im.nx = static_cast< int32_t >( nx );
   im.ny = static_cast< int32_t >( ny );
   for( int i = 0; i < 2; ++i ) {
      im.bc[ i ] = bc[ i ];
      im.h[ i ] = h[ i ];
      im.odd[ i ] = odd[ i ];
   }
   return true;
}

template bool march2d_image< float >( M2Image&, void const*, int64_t, int64_t, int64_t, int64_t, int64_t, float*, int64_t,
                                      int64_t, int32_t const*, int32_t const*, int32_t const* );

int march2d_slots() {
   return 2 * sm_count();
}

namespace {

template< typename TIn >
cudaError_t run_march2d( FusedArgs const& f, int32_t const h[ 2 ], int32_t const odd[ 2 ], cudaStream_t stream ) {
   if( !march2d_ready< TIn >()) { return cudaErrorNotSupported; }
   M2Args a{};
   if( !march2d_image< TIn >( a.img0, f.src, f.n[ 0 ], f.n[ 1 ], f.ss[ 1 ], f.nb, f.sb, f.dst, f.ds[ 1 ], f.db, f.bc, h, odd )) {
      return cudaErrorNotSupported;
   }
   for( int ax = 0; ax < 2; ++ax ) {
      for( int k = 0; k <= h[ ax ]; ++k ) { a.w0[ ax ][ k ] = f.w[ ax ][ k ]; }
   }
   a.status = device_status_ptr();
   if( !a.status ) { return cudaErrorUnknown; }
   a.nb = static_cast< int32_t >( f.nb );
   a.strips = static_cast< int32_t >(( f.n[ 0 ] + kM2TX - 1 ) / kM2TX );
   int const slots = march2d_slots();
   a.chunks = march2d_chunks( static_cast< int64_t >( a.strips ) * a.nb, f.n[ 1 ], h[ 1 ], slots );
   a.lchunk = static_cast< int32_t >(( f.n[ 1 ] + a.chunks - 1 ) / a.chunks );
   a.chunks = static_cast< int32_t >(( f.n[ 1 ] + a.lchunk - 1 ) / a.lchunk );
   int64_t const items = static_cast< int64_t >( a.nb ) * a.strips * a.chunks;
   if( items > 0x7fffffff ) { return cudaErrorNotSupported; }
   int const grid = static_cast< int >( items < slots ? items : slots );
   march2d_kernel< TIn ><<< grid, kM2NT, M2Smem::BYTES, stream >>>( a ); count_launch();
   return cudaGetLastError();
}

} // namespace

cudaError_t launch_march2d_items( M2Image const* d_images, int nimages, M2Item const* d_items, int nitems, int32_t* counter,
                                  int stall, cudaStream_t stream ) {
   if( nitems <= 0 ) { return cudaSuccess; }
   if( !march2d_ready< float >()) { return cudaErrorNotSupported; }
   M2Args a{};
   a.images = d_images;
   a.nimages = nimages;
   a.items = d_items;
   a.nitems = nitems;
   a.queue = counter;
   a.stall_copies = stall ? 1 : 0;
   a.wait_limit = stall ? 20000u : 0u;       // a stalled copy is given up on after ~10 ms, not seconds
   a.status = device_status_ptr();
   if( !a.status ) { return cudaErrorUnknown; }
   int const slots = march2d_slots();
   int const grid = nitems < slots ? nitems : slots;
   march2d_kernel< float ><<< grid, kM2NT, M2Smem::BYTES, stream >>>( a ); count_launch();
   return cudaGetLastError();
}

cudaError_t launch_march2d( FusedKey const& key, FusedArgs& args, cudaStream_t stream ) {
   if( key.ndims != 2 || getenv( "DIPCU_NO_MARCH" )) { return cudaErrorNotSupported; }
   int32_t h[ 2 ] = { key.h[ 0 ], key.h[ 1 ] };
   int32_t odd[ 2 ] = { key.odd[ 0 ], key.odd[ 1 ] };
   if( key.in_dt == DT_SFLOAT ) { return run_march2d< float >( args, h, odd, stream ); }
   if( key.in_dt == DT_UINT16 ) { return run_march2d< uint16_t >( args, h, odd, stream ); }
   return cudaErrorNotSupported;
}

} // namespace dipcu
