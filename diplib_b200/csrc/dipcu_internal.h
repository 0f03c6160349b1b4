// Internal interfaces between the C-ABI layer (api.cpp) and the kernel launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dipcu.h"

namespace dipcu {

constexpr int kLineMaxHalf = 2048;  // longest half-width the line kernel accepts
constexpr int kFusedMaxTaps = 65;   // per-axis tap capacity of the fused kernels' parameters

// One pass of the line kernel (K2).
struct LinePass {
   void const* src;
   void* dst;
   int32_t src_dt, dst_dt;
   int32_t ndims, axis;
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t src_strides[ DIPCU_MAX_DIMS ];
   int64_t dst_strides[ DIPCU_MAX_DIMS ];
   int64_t h;
   int32_t odd, bc;
   bool compute_double;
   double const* taps;  // h + 1 host values, centre first
};
cudaError_t launch_line_pass( LinePass const& p, cudaStream_t stream );

struct ConvertArgs {
   void const* src;
   void* dst;
   int32_t src_dt, dst_dt, ndims;
   int64_t total;
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t sst[ DIPCU_MAX_DIMS ], dstst[ DIPCU_MAX_DIMS ];
};
cudaError_t launch_convert( ConvertArgs const& a, bool compute_double, cudaStream_t stream );

// Fused multi-axis tile kernels (K1).  The image is viewed as up to 3 filtered axes
// x (unit stride in both images), y, z, plus at most one unfiltered "batch" axis.
struct FusedArgs {
   void const* src;
   float* dst;
   int64_t n[ 3 ];          // sizes of x, y, z (z = 1 for 2D)
   int64_t ss[ 3 ];         // source strides of x (must be 1), y, z
   int64_t ds[ 3 ];         // destination strides
   int64_t nb, sb, db;      // batch axis size and strides
   int32_t bc[ 3 ];
   int32_t tiles_x, tiles_y, zchunks, lz;
   float w[ 3 ][ kFusedMaxTaps ];  // per axis, centre tap first
};

struct FusedKey {
   int32_t ndims;          // 2 or 3
   int32_t in_dt;          // DT_SFLOAT / DT_UINT16 / DT_UINT8 / DT_SINT16
   int32_t h[ 3 ];
   int32_t odd[ 3 ];
};

// Returns cudaErrorNotSupported if no fused kernel exists for `key`.
cudaError_t launch_fused( FusedKey const& key, FusedArgs& args, cudaStream_t stream );

// Records `msg` as this thread's dipcu_last_error_message() and returns `code`.
int record_error( int code, char const* msg );
bool fused_available( FusedKey const& key );

} // namespace dipcu
