// Internal interfaces between the C-ABI layer (api.cpp) and the kernel launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/dipcu.h"

namespace dipcu {

constexpr int kLineMaxHalf = 2048;  // longest half-width the line kernel accepts
constexpr int kFusedMaxTaps = 65;   // per-axis tap capacity of the fused kernels' parameters
constexpr int kFoldMaxHalf = 100;   // longest half-width the adjoint's halo fold accepts
constexpr int kFoldMaxEntries = 1000;

// One coefficient of the boundary extension: halo position j (line coordinate, outside [0, n))
// takes c * sample i.  The adjoint folds the halo gradient back along these entries.
struct FoldEntry {
   int32_t j, i;
   double c;
};

// One pass of the line kernel (K2).
struct LinePass {
   void const* src;
   void* dst;
   int32_t src_dt, dst_dt;
   int32_t ndims, axis;
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t src_strides[ DIPCU_MAX_DIMS ];
   int64_t dst_strides[ DIPCU_MAX_DIMS ];
   int64_t h;           // border: the boundary extension on both sides (the half-width in mode 0)
   int32_t odd, bc;
   bool compute_double;
   double const* taps;  // mode 0: h + 1 host values, centre first
   // mode 0: symmetric or antisymmetric taps (the Gaussian); mode 1: a general filter,
   // out[i] = sum_{j=-lo}^{hi} full[j + lo] x[i + j] (lo + hi + 1 <= kGeneralMaxTaps host values);
   // mode 2: the rectangular uniform filter of `usize` samples, window [i - usize/2, i + (usize+1)/2),
   // as a running sum in the order of dip::Uniform's line filter (src/linear/uniform.cpp:41-62).
   int32_t mode = 0;
   int64_t lo = 0, hi = 0, usize = 0;
   double const* full = nullptr;
};
constexpr int kGeneralMaxTaps = 256;
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

// 4D tiled TMA map (no swizzle, no interleave, zero fill) of a device buffer; cached per
// (pointer, layout, box).
CUresult encode_source_map( CUtensorMap* out, CUtensorMapDataType dt, void const* ptr, cuuint64_t const* dims,
                            cuuint64_t const* strides, cuuint32_t const* box );

struct FusedKey {
   int32_t ndims;          // 2 or 3
   int32_t in_dt;          // DT_SFLOAT / DT_UINT16 / DT_UINT8 / DT_SINT16
   int32_t h[ 3 ];
   int32_t odd[ 3 ];
};

// Returns cudaErrorNotSupported if no fused kernel exists for `key`.
cudaError_t launch_fused( FusedKey const& key, FusedArgs& args, cudaStream_t stream );

bool fused_available( FusedKey const& key );

// Fused 2D adjoint (input gradient and both sigma gradients) of the Gaussian FIR.
struct Adj2Params {
   float const* gy;                   // dL/d(out), float, x stride 1
   int64_t gys1, gyb;                 // row and batch strides
   void const* x;                     // the forward input (nullptr: no sigma gradients)
   int32_t x_dt;
   int64_t xs1, xb;
   float* gx;                         // dL/d(in), float, x stride 1 (nullptr: not wanted)
   int64_t gxs1, gxb;
   double* dsig[ 2 ];                 // dL/dsigma of the x and y axes (device; accumulated)
   int64_t n[ 2 ], nb;
   int32_t bc[ 2 ], h[ 2 ], odd[ 2 ];
   double const* taps[ 2 ];           // h + 1 taps, centre first
   double const* dtaps[ 2 ];          // their sigma derivatives (may be nullptr without sigma)
};
// cudaErrorNotSupported when the fused kernel does not apply (the caller runs the pass-by-pass
// adjoint instead).
cudaError_t launch_fused_adjoint2d( Adj2Params const& p, cudaStream_t stream );

// Warp-per-tile 2D kernel (any half-widths up to 12, float or uint16 input, the x-y boundary
// conditions it handles); cudaErrorNotSupported when it does not apply.
cudaError_t launch_fused2d_ws( FusedKey const& key, FusedArgs& args, cudaStream_t stream );

// Row-march 2D kernel (march2d.cuh: half-widths up to 32 on both axes, float or uint16 input,
// the index-mapping boundary conditions and "add zeros"); cudaErrorNotSupported when it does not
// apply.
cudaError_t launch_march2d( FusedKey const& key, FusedArgs& args, cudaStream_t stream );

// Adjoint halo fold along one axis (k_backward.cu).
struct FoldPass {
   void const* g;            // gradient w.r.t. the forward pass output (compute type)
   void* xb;                 // gradient w.r.t. the forward pass input (compute type), correlation part
   int32_t ndims, axis;
   int64_t sizes[ DIPCU_MAX_DIMS ];
   int64_t gst[ DIPCU_MAX_DIMS ], xst[ DIPCU_MAX_DIMS ];
   int64_t h;
   int32_t odd;
   bool compute_double;
   double const* taps;       // h + 1 forward taps, centre first
   FoldEntry const* entries;
   int32_t nentries;
};
cudaError_t launch_fold( FoldPass const& p, cudaStream_t stream );
// atomically adds <src, dst> (both of the compute type, layouts as in ConvertArgs) to *out.
cudaError_t launch_dot( ConvertArgs const& a, bool compute_double, double* out, cudaStream_t stream );

// Records `msg` as this thread's dipcu_last_error_message() and returns `code`.
int record_error( int code, char const* msg );

// Counts one kernel launch of this library (host side: a launch captured into a CUDA graph counts
// once, at capture).  Every launch site calls it right after its <<< >>> statement.
void count_launch();

// Per-axis filter as dip::GaussFIR builds it (src/linear/gauss.cpp:255-284); modes 1 and 2 (a
// general filter, the rectangular uniform filter) as LinePass describes them.
struct AxisFilter {
   bool process = false;
   int64_t h = 0;
   int32_t odd = 0;
   int32_t bc = 0;
   std::vector< double > taps;  // centre first, rounded to the compute precision
   int32_t mode = 0;
   int64_t lo = 0, hi = 0, usize = 0;
   std::vector< double > full;  // mode 1: lo + hi + 1 taps, rounded to the compute precision
};

// Checks an (in, out) image pair: forged, same sizes, valid types, non-overlapping.
int check_pair( dipcu_image_desc const* in, dipcu_image_desc const* out );

// dip::GaussFIR's per-axis set-up (sigma <= 0 / size-1 axes skipped, order and BC checks,
// weights in the precision of the computation).  `dtaps` (optional) receives d(taps)/d(sigma).
int build_filters( dipcu_image_desc const* in, double const* sigmas, uint32_t const* orders, int32_t const* bcs,
                   double truncation, std::vector< AxisFilter >& f, std::vector< std::vector< double >>* dtaps );

// Framework::Separable's pass order: processed axes by input stride, stable.
std::vector< int > pass_order( dipcu_image_desc const* in, std::vector< AxisFilter > const& f );

// Several GaussFIR outputs of `in` (sizes and boundary conditions shared, `ncomp` order vectors of
// ndims entries) from one read of it, by the multi-output tile kernel (multi_deriv.cu).  `mode`:
// 0 the components (nout = ncomp), 1 their symmetric products in DIPlib's symmetric-matrix order
// (nout = ncomp (ncomp + 1) / 2), 2 their sum, 3 the square root of their sum of squares (nout = 1).
// Returns -1 when the kernel does not take the case (2D/3D float computation, index-mapping or
// "add zeros" boundary conditions on filtered axes, half-widths up to 8, up to 6 components).
int multi_gauss_fir( dipcu_image_desc const* in, dipcu_image_desc const* outs, int nout, uint32_t const* orders, int ncomp,
                     int mode, double const* sigmas, int32_t const* bcs, double truncation, cudaStream_t stream );

// Copies `in` to `out` with the type conversion (no axis filtered).
int run_convert( dipcu_image_desc const* in, dipcu_image_desc const* out, cudaStream_t stream );

// Scratch images (each numel(in) samples of the compute type) run_line_passes needs for
// `passes` line passes: 0 for one pass, 1 when `out` has the compute type or for two passes, else 2.
int line_pass_scratch_images( int passes, bool out_is_buf );

// The line-kernel pass chain of Framework::Separable (in -> out -> out ...) along `order`, with
// the intermediates in the caller's scratch images (normal strides).
int run_line_passes( dipcu_image_desc const* in, dipcu_image_desc const* out, std::vector< AxisFilter > const& f,
                     std::vector< int > const& order, bool compute_double, void* const scratch[ 2 ], cudaStream_t stream );

// Runs the separable filter `f` from `in` to `out` (fused tile kernel when possible, else the
// line-kernel pass chain), computing in double when `compute_double`.
int run_filters( dipcu_image_desc const* in, dipcu_image_desc const* out, std::vector< AxisFilter > const& f,
                 bool compute_double, cudaStream_t stream );

} // namespace dipcu
