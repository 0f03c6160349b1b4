/*
 * dipcu -- B200 (sm_100a) implementation of DIPlib's Gaussian FIR filtering path.
 *
 * C-ABI of libdipcu.so.  Plain pointers and sizes only.  Every image argument is a
 * `dipcu_image_desc` whose `data` is a DEVICE pointer to the image origin; sizes and strides
 * follow dip::Image (include/diplib/library/image.h:268+ in DIPlib): DIPlib axis order (x first),
 * strides in samples (they may be negative).  Per-axis parameter arrays have exactly `ndims`
 * entries (the caller has already broadcast them the way dip::ArrayUseParameter does).
 *
 * All entry points are asynchronous on `stream` (a cudaStream_t; NULL = the legacy default
 * stream), return a dipcu_status, and record a message retrievable with
 * dipcu_last_error_message() (thread-local).  None of them synchronises the device.
 */
#ifndef DIPCU_H
#define DIPCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DIPCU_MAX_DIMS 8

/* Sample types: DIPlib's real types (include/diplib/library/datatype.h).  The codes are this
 * library's own (dip::DataType's internal enumerator order differs); a DIPlib caller converts with a
 * switch, as DipTypeToDipcu in INTEGRATION.md does. */
typedef enum {
   DIPCU_BIN = 0, DIPCU_UINT8 = 1, DIPCU_UINT16 = 2, DIPCU_UINT32 = 3, DIPCU_UINT64 = 4,
   DIPCU_SINT8 = 5, DIPCU_SINT16 = 6, DIPCU_SINT32 = 7, DIPCU_SINT64 = 8,
   DIPCU_SFLOAT = 9, DIPCU_DFLOAT = 10
} dipcu_dtype;

/* dip::BoundaryCondition enumerators, same values (include/diplib/boundary.h:65-80). */
typedef enum {
   DIPCU_BC_SYMMETRIC_MIRROR = 0, DIPCU_BC_ASYMMETRIC_MIRROR = 1, DIPCU_BC_ANTISYMMETRIC_REFLECT = 2,
   DIPCU_BC_PERIODIC = 3, DIPCU_BC_ASYMMETRIC_PERIODIC = 4, DIPCU_BC_ADD_ZEROS = 5,
   DIPCU_BC_ADD_MAX_VALUE = 6, DIPCU_BC_ADD_MIN_VALUE = 7, DIPCU_BC_ZERO_ORDER_EXTRAPOLATE = 8,
   DIPCU_BC_FIRST_ORDER_EXTRAPOLATE = 9, DIPCU_BC_SECOND_ORDER_EXTRAPOLATE = 10,
   DIPCU_BC_THIRD_ORDER_EXTRAPOLATE = 11, DIPCU_BC_ALREADY_EXPANDED = 12
} dipcu_bc;

typedef enum {
   DIPCU_OK = 0,
   DIPCU_ERR_INVALID_ARG = 1,       /* bad pointer, size, stride, dimensionality or parameter */
   DIPCU_ERR_UNSUPPORTED_DTYPE = 2, /* e.g. complex data (dip::E::DATA_TYPE_NOT_SUPPORTED) */
   DIPCU_ERR_UNSUPPORTED_BC = 3,    /* unknown value, or "already expanded" */
   DIPCU_ERR_ORDER_GT_3 = 4,        /* "Gaussian FIR filter not implemented for order > 3" */
   DIPCU_ERR_CUDA = 5,              /* a CUDA runtime call failed */
   DIPCU_ERR_TIMEOUT = 6,           /* a bounded device-side wait gave up */
   DIPCU_ERR_SIZES_DONT_MATCH = 7,  /* in/out size mismatch (dip::E::SIZES_DONT_MATCH) */
   DIPCU_ERR_KERNEL_TOO_LARGE = 8   /* kernel half-width beyond the supported maximum */
} dipcu_status;

typedef struct {
   void* data;                        /* device pointer to the origin sample */
   int32_t dtype;                     /* dipcu_dtype */
   int32_t ndims;                     /* 1 .. DIPCU_MAX_DIMS */
   int64_t sizes[ DIPCU_MAX_DIMS ];   /* DIPlib order, x first */
   int64_t strides[ DIPCU_MAX_DIMS ]; /* in samples */
} dipcu_image_desc;

/* ---- Forward filter ---------------------------------------------------------------------- */

/* The body of dip::GaussFIR (src/linear/gauss.cpp:238-286 in DIPlib) and the path below it:
 * dip::SeparableConvolution (src/linear/convolution.cpp:319-421) driven by
 * dip::Framework::Separable (src/library/framework_separable.cpp:35-431).
 *
 * `in`: any real sample type.  `out`: same sizes; its type is normally the one DIPlib picks
 * (dip::DataType::SuggestFlex: sfloat, or dfloat for 32/64-bit integer and dfloat input);
 * another type reproduces DIPlib's protected-output path (computation in the flex type,
 * clamp_cast on the final write).  `out` must not overlap `in` (DIPlib strips an overlapping
 * output first; the C++ layer above does the same).
 * `sigmas[d] <= 0` or `sizes[d] == 1` leaves axis d unfiltered; `orders[d]` in 0..3;
 * `bcs[d]` a dipcu_bc; `truncation <= 0` means 3.
 * Replaces the per-line, host-pointer callback Framework::SeparableLineFilter
 * (include/diplib/framework.h:654-669) with fused device kernels. */
int dipcu_gauss_fir( dipcu_image_desc const* in, dipcu_image_desc const* out,
                     double const* sigmas, uint32_t const* orders, int32_t const* bcs,
                     double truncation, void* stream );

/* The same filter for callers that cannot allocate device memory while they run: code whose GPU
 * memory is all handed out by another allocator (a framework's caching allocator, or a pool
 * reserved at start-up) so that the process must not grow its footprint behind that allocator's
 * back, and long-running pipelines that must not fail for lack of memory once started.  No
 * counterpart in DIPlib (whose CPU filter allocates its line buffers per thread).
 *
 * Allocates nothing: the pass intermediates live in a static device array of 32 MiB that the
 * library holds on every GPU it is used on until the process exits.  Images are limited to
 * 4 Mi samples when the filter computes in float and 2 Mi samples when it computes in double
 * (32/64-bit integer or dfloat input); larger images return DIPCU_ERR_INVALID_ARG.  Runs the
 * line kernel pass by pass.  All calls share the array: calls whose work overlaps on the GPU race
 * and give wrong results, so order them on one stream.  Every call outside stream capture looks up
 * the array's address on its device; a call under capture reuses the one found by the device's
 * last call outside capture, so make one call on a device (after any device reset) before
 * capturing one.  Arguments, checks and results are those of dipcu_gauss_fir. */
int dipcu_gauss_fir_noalloc( dipcu_image_desc const* in, dipcu_image_desc const* out,
                             double const* sigmas, uint32_t const* orders, int32_t const* bcs,
                             double truncation, void* stream );

/* ---- Other separable filters -------------------------------------------------------------- */

/* A real 1D filter as dip::OneDimensionalFilter holds it (include/diplib/linear.h:84-92 in DIPlib):
 * `size` weights (HOST memory), the origin (-1: the centre), and the symmetry: DIPCU_SYM_GENERAL
 * ("general" or ""), _EVEN ("even", and "conj" for a real filter: `weights` is the left half
 * with the centre last), _ODD ("odd"), _D_EVEN ("d-even", "d-conj"), _D_ODD ("d-odd"). */
typedef enum {
   DIPCU_SYM_GENERAL = 0, DIPCU_SYM_EVEN = 1, DIPCU_SYM_ODD = 2, DIPCU_SYM_D_EVEN = 3, DIPCU_SYM_D_ODD = 4
} dipcu_symmetry;

typedef struct {
   double const* weights;
   int64_t size;
   int64_t origin;
   int32_t symmetry;                  /* dipcu_symmetry */
} dipcu_filter_1d;

/* dip::SeparableConvolution for real filters (src/linear/convolution.cpp:319-421 in DIPlib):
 * `nfilters` is 1 (the filter is used along every axis) or in->ndims; `bcs` has ndims entries;
 * `process` (optional, ndims flags) selects the axes.  Output and computation types as
 * dipcu_gauss_fir (dip::DataType::SuggestFlex; another `out` type is the protected-output path).
 * An axis of size 1, or whose filter is empty or a single unit weight, is not filtered.  Filters up
 * to 256 weights after the symmetry's expansion (DIPCU_ERR_KERNEL_TOO_LARGE beyond).  Errors:
 * "Symmetry string not recognized" and "Origin outside of filter" (DIPCU_ERR_INVALID_ARG), as the
 * reference.  Intermediates of the pass chain are stream-ordered allocations. */
int dipcu_separable_convolution( dipcu_image_desc const* in, dipcu_image_desc const* out, dipcu_filter_1d const* filters,
                                 int nfilters, int32_t const* bcs, uint8_t const* process, void* stream );

/* Several Gaussian derivatives of one image from one read of it: the components of dip::Gradient,
 * dip::Hessian and dip::Laplace (src/linear/derivative.cpp:142-172, 330-418 in DIPlib), which the
 * reference computes as one dip::GaussFIR call each.  `orders` holds ncomp order vectors of ndims
 * entries; sigmas, boundary conditions and truncation are shared (ndims values each) and each
 * component equals dipcu_gauss_fir with its orders.  `mode` 0 writes the components (nout =
 * ncomp), 1 their symmetric products g_i g_j in DIPlib's symmetric-matrix order (diagonal first,
 * then the upper triangle column by column; nout = ncomp (ncomp + 1) / 2; dip::StructureTensor's
 * products), 2 their sum (dip::Laplace), 3 the square root of their sum of squares
 * (dip::GradientMagnitude); nout = 1 for modes 2 and 3.  `outs` are nout output images of the
 * input's sizes, any type (clamp_cast on the write).  Taken: 2D and 3D images whose computation
 * type is sfloat, index-mapping or "add zeros" boundary conditions on the filtered axes,
 * half-widths up to 8, up to 6 components (dipcu_gauss_fir_multi_supported says so, without
 * recording an error); other cases are DIPCU_ERR_INVALID_ARG. */
int dipcu_gauss_fir_multi( dipcu_image_desc const* in, dipcu_image_desc const* outs, int nout, uint32_t const* orders,
                           int ncomp, int32_t mode, double const* sigmas, int32_t const* bcs, double truncation, void* stream );
int dipcu_gauss_fir_multi_supported( dipcu_image_desc const* in, uint32_t const* orders, int ncomp, double const* sigmas,
                                     int32_t const* bcs, double truncation );

/* dip::GaussIIR (src/linear/gaussiir.cpp:725-790, include/diplib/linear.h:407-428 in DIPlib): the
 * recursive Gaussian (derivative) filter of van Vliet, Young and Verbeek, orders 0-4 per axis,
 * computed in dfloat like the reference (intermediates of the pass chain in dfloat, output
 * clamp_cast to `out`'s type, normally dip::DataType::SuggestFlex of the input).  `filter_orders`:
 * the recursion order per axis (1-5; NULL: the reference's default, order + 3 and 5 above order 2);
 * `design`: DIPCU_IIR_DISCRETE_TIME_FIT ("discrete time fit", the reference's default) or
 * DIPCU_IIR_FORWARD_BACKWARD ("forward backward").  Every boundary condition but "already
 * expanded".  Scan lines and the intermediate are stream-ordered allocations. */
#define DIPCU_IIR_DISCRETE_TIME_FIT 0
#define DIPCU_IIR_FORWARD_BACKWARD 1
int dipcu_gauss_iir( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sigmas,
                     uint32_t const* orders, int32_t const* bcs, uint32_t const* filter_orders, int32_t design,
                     double truncation, void* stream );

/* dip::GaussFT with spatial input and output (src/linear/gauss.cpp:397-487 in DIPlib): the
 * Gaussian (derivative) filter computed by multiplication in the Fourier domain.  `sigmas` and
 * `orders` hold ndims values (a negative sigma means no smoothing; an axis of size 1 is not
 * filtered; any derivative order).  With nbcs == ndims the image is first extended by those
 * boundary conditions to 5-smooth transform sizes that hold twice the half Gaussian size on each
 * side (as dip::Gauss does, which passes "default", i.e. mirror, when given none); with nbcs == 0
 * the transform covers exactly the image (periodic).  Extension supports the index-mapping
 * conditions and "add zeros" (DIPCU_ERR_UNSUPPORTED_BC otherwise).  Images of 1 to 3 dimensions.
 * Computation in dip::DataType::SuggestComplex of the input (double for 32/64-bit integers and
 * dfloat, else float); output type as dipcu_gauss_fir.  The transforms are cuFFT's; the outputs
 * follow the reference's own transform, including its treatment of odd transform lengths. */
int dipcu_gauss_ft( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sigmas, uint32_t const* orders,
                    double truncation, int32_t const* bcs, int nbcs, void* stream );

/* dip::Uniform with a rectangular kernel (src/linear/uniform.cpp:68-86, 147-163 in DIPlib): `sizes`
 * holds the kernel's per-axis sizes (ndims values; a size above 1 is truncated to an integer, as
 * dip::Kernel::Sizes does, others leave the axis unfiltered); the mean over the window
 * [i - size/2, i + (size+1)/2) of the boundary-extended line, computed as the reference's running
 * sum (same operation order).  Types as dipcu_gauss_fir. */
int dipcu_uniform( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* sizes, int32_t const* bcs,
                   void* stream );

/* ---- Backward (adjoint) ------------------------------------------------------------------- */

/* Gradients of dipcu_gauss_fir (no DIPlib counterpart; DIPlib has no derivatives of its filters).
 * `grad_out`: dL/d(out), of the filter's computation type (sfloat, or dfloat for 32/64-bit
 * integer and dfloat input).  `grad_in` (optional, same type): receives dL/d(in), the adjoint of
 * the forward pass by pass -- zero-padded correlation with the flipped kernel, then the halo
 * gradients folded back through the boundary extension (every boundary condition; half-widths up to
 * 100).  `grad_sigma` (optional, DEVICE array of ndims doubles): receives dL/d(sigma_d) for each
 * filtered axis (0 elsewhere), from the analytic derivative of the normalised discrete kernel
 * with its length held fixed; needs `in`.  Recomputes what it needs from `in`; allocates its
 * intermediates with cudaMallocAsync on `stream`. */
int dipcu_gauss_fir_backward( dipcu_image_desc const* grad_out, dipcu_image_desc const* in,
                              dipcu_image_desc const* grad_in, double* grad_sigma,
                              double const* sigmas, uint32_t const* orders, int32_t const* bcs,
                              double truncation, void* stream );

/* ---- Structure tensor ------------------------------------------------------------------------ */

/* dip::StructureTensor with the "gaussFIR" method, no mask (src/analysis/structure_tensor.cpp:33-59
 * in DIPlib; gradient as dip::Gradient, src/linear/derivative.cpp:142-172).  `in`: a 1D-3D
 * image of any non-binary type; the gradient runs along every axis of size > 1 and gradient sigma > 0
 * (dip::FindGradientDimensions, src/linear/derivative.cpp:120-138).  `out`: an image of
 * ndims + 1 dimensions, the input's sizes followed by the component axis of m(m+1)/2 entries
 * (m gradient axes) in DIPlib's symmetric-matrix order (diagonal first, then the upper triangle
 * column by column: xx, yy, zz, xy, xz, yz), of the flex type (sfloat, dfloat for 32/64-bit integer and dfloat input); any
 * strides, so DIPlib's own layout (component stride 1) and a planar one both work.
 * `grad_sigmas`, `tensor_sigmas`, `bcs`: one entry per input dimension (already broadcast, as
 * dip::ArrayUseParameter does).  The gradient images are scratch of the call (stream-ordered
 * allocations). */
int dipcu_structure_tensor( dipcu_image_desc const* in, dipcu_image_desc const* out, double const* grad_sigmas,
                            double const* tensor_sigmas, int32_t const* bcs, double truncation, void* stream );

/* Gradient of L = sum_c <grad_out_c, T_c> with respect to the input (no DIPlib counterpart).
 * `grad_out` has the layout of dipcu_structure_tensor's `out`; `grad_in` the input's sizes and the
 * flex type.  The gradient images are recomputed from `in`, never stored by the forward. */
int dipcu_structure_tensor_backward( dipcu_image_desc const* grad_out, dipcu_image_desc const* in,
                                     dipcu_image_desc const* grad_in, double const* grad_sigmas,
                                     double const* tensor_sigmas, int32_t const* bcs, double truncation,
                                     void* stream );

/* ---- Batched filter ------------------------------------------------------------------------ */

/* Many 2D sfloat images of uneven sizes, each with its own per-axis sigmas, orders (0..3) and
 * boundary conditions (the index-mapping ones and "add zeros"; half-widths up to 32).  Images
 * with both half-widths up to 12 and "mirror", "zero order", "add zeros", "asym mirror",
 * "periodic" or "asym periodic" along both axes run through grouped warp-per-tile launches (one per half-width bucket, per-image work
 * lists); the others through grouped line passes (along x into an intermediate the plan owns,
 * then along y; one launch per pass and per half-width bucket of that pass' axis, the y passes
 * after all x passes); the buckets run as parallel branches.  A persistent launch that pulls (image, tile) work items from a device queue remains
 * as the fallback (DIPCU_BATCH_NO_LINES routes the rest there).  No DIPlib counterpart (DIPlib
 * filters one image per call; this is dip::GaussFIR per image).
 * `sigmas`, `orders`, `bcs`: host arrays of 2 * count entries (x then y of each image).
 * Flags: DIPCU_BATCH_GRAPH captures the run (queue reset, on-device weights, all launches)
 * into a CUDA graph so that dipcu_batch_plan_run is one graph launch; DIPCU_BATCH_AUTOTUNE times
 * the persistent kernel's candidate tile shapes on this batch at creation (overwriting the outputs) and keeps the
 * fastest, remembered per batch signature.  The INJECT flags are test hooks: INVALID_IMAGE and
 * INVALID_TILE plant one impossible work item, which the kernels skip and report through
 * dipcu_device_status; STALLED_COPY makes the row-march launch announce its TMA copies without
 * issuing them, so that its bounded waits give up (after ~10 ms) and it reports DIPCU_ERR_TIMEOUT
 * with no copy in flight -- the context stays usable.
 * The plan allocates its tables and the line-pass intermediate at creation; runs allocate nothing.  The images must stay alive
 * while the plan is used.  The sigma table (dipcu_batch_plan_sigmas, device, 2 * count doubles)
 * may be rewritten between runs, as long as no kernel length changes. */
typedef struct dipcu_batch_plan dipcu_batch_plan;
#define DIPCU_BATCH_GRAPH 1
#define DIPCU_BATCH_AUTOTUNE 2
#define DIPCU_BATCH_INJECT_INVALID_IMAGE 256
#define DIPCU_BATCH_INJECT_INVALID_TILE 512
#define DIPCU_BATCH_INJECT_STALLED_COPY 1024
int dipcu_batch_plan_create( dipcu_image_desc const* ins, dipcu_image_desc const* outs, int count,
                             double const* sigmas, uint32_t const* orders, int32_t const* bcs, double truncation,
                             int flags, dipcu_batch_plan** plan );
int dipcu_batch_plan_run( dipcu_batch_plan* plan, void* stream );
/* Work items (all paths), chosen tile shape and persistent grid size of a plan. */
int dipcu_batch_plan_info( dipcu_batch_plan const* plan, int* nitems, int* tile_x, int* tile_y, int* grid );
/* Kernels one run launches (the weights kernel, the persistent tile kernel when it has items,
 * one grouped warp-per-tile launch per half-width bucket in use) and the work items the grouped
 * path takes.  No counterpart in the reference (plan introspection). */
int dipcu_batch_plan_launches( dipcu_batch_plan const* plan, int* kernels, int* grouped_items );
double* dipcu_batch_plan_sigmas( dipcu_batch_plan* plan );
int dipcu_batch_plan_destroy( dipcu_batch_plan* plan );

/* Reads (and with `clear`, resets) the device status word where kernels report a skipped invalid
 * work item (DIPCU_ERR_INVALID_ARG) or a timed-out wait (DIPCU_ERR_TIMEOUT).  Synchronises. */
int dipcu_device_status( int* status, int clear );

/* ---- Kernel weights ----------------------------------------------------------------------- */

/* Half-kernel length of dip::MakeHalfGaussian (src/linear/gauss.cpp:38-62): returns
 * 1 + HalfGaussianSize (at least 2 for order 3), 1 for sigma == 0, or -1 for order > 3.
 * `dt_double` selects the dfloat truncation limit (maximum_gauss_truncation<dfloat>). */
int dipcu_half_gaussian_length( double sigma, uint32_t order, double truncation, int dt_double );

/* On-device construction of the weights of dip::MakeHalfGaussian (src/linear/gauss.cpp:53-165)
 * for `count` (sigma, order) pairs read from DEVICE arrays.  Entry i writes its reversed half
 * kernel (centre tap first, as InternOneDimensionalFilter stores it, convolution.cpp:76-156)
 * to `weights + i * stride` as floats; with `dweights` non-NULL also d(weights)/d(sigma).
 * `lengths` (device, optional) receives each half-kernel length; entries longer than `stride`
 * are truncated and flagged with a negative length. */
int dipcu_make_gauss_weights( double const* sigmas, uint32_t const* orders, int count, double truncation,
                              float* weights, float* dweights, int32_t* lengths, int stride, void* stream );

/* ---- Utilities ----------------------------------------------------------------------------- */

/* dip::StringToBoundaryCondition (include/diplib/boundary.h:87-103): a dipcu_bc, or -1 when the
 * string is not recognised ("Boundary condition not recognized: " + bc). */
int dipcu_bc_from_string( char const* bc );

/* Message of the last failing call on this host thread ("" if none). */
char const* dipcu_last_error_message( void );

/* Library version string. */
char const* dipcu_version( void );

/* Kernel launches this library has issued since it was loaded, counted on the host: a launch
 * captured into a CUDA graph counts once, at capture, so a graph's replays launch the count that
 * its capture added. */
uint64_t dipcu_launch_count( void );

#ifdef __cplusplus
}
#endif

#endif /* DIPCU_H */
