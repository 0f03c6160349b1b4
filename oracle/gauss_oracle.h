/* Test infrastructure only: a plain-C restatement of DIPlib's Gaussian FIR path, used as the
 * parity oracle for the CUDA kernels.  It is never linked into or called by the product.
 *
 * Pinned against the reference itself: tests/test_oracle_pin.py compares every function here
 * with the same function of the unmodified DIPlib sources (oracle/_ref/libdipref.so, built by
 * oracle/Makefile) where that library exists, and tests/golden/ holds fixtures generated from
 * it (tests/golden/make_golden.py) for runs without the reference tree.
 *
 * Conventions follow DIPlib: sizes and strides are in DIPlib order (x first) and in samples.
 */
#ifndef GAUSS_ORACLE_H
#define GAUSS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Data type codes, identical to include/dipcu.h. */
enum {
   OR_BIN = 0, OR_UINT8 = 1, OR_UINT16 = 2, OR_UINT32 = 3, OR_UINT64 = 4,
   OR_SINT8 = 5, OR_SINT16 = 6, OR_SINT32 = 7, OR_SINT64 = 8, OR_SFLOAT = 9, OR_DFLOAT = 10
};

/* dip::BoundaryCondition enumerator values (include/diplib/boundary.h:65-80). */
enum {
   OR_BC_SYMMETRIC_MIRROR = 0, OR_BC_ASYMMETRIC_MIRROR, OR_BC_ANTISYMMETRIC_REFLECT, OR_BC_PERIODIC,
   OR_BC_ASYMMETRIC_PERIODIC, OR_BC_ADD_ZEROS, OR_BC_ADD_MAX_VALUE, OR_BC_ADD_MIN_VALUE,
   OR_BC_ZERO_ORDER_EXTRAPOLATE, OR_BC_FIRST_ORDER_EXTRAPOLATE, OR_BC_SECOND_ORDER_EXTRAPOLATE,
   OR_BC_THIRD_ORDER_EXTRAPOLATE, OR_BC_ALREADY_EXPANDED
};

/* Status codes. */
enum { OR_OK = 0, OR_ERR_ORDER = 1, OR_ERR_BC = 2, OR_ERR_DTYPE = 3, OR_ERR_ARG = 4 };

/* HalfGaussianSize, src/linear/gauss.cpp:38-51. */
size_t or_half_gaussian_size( double sigma, unsigned order, double truncation, int dt_double );

/* MakeHalfGaussian, src/linear/gauss.cpp:53-165: writes the half kernel (x=0 at the END) into
 * `out` (capacity `cap`), returns its length, or -1 for order > 3. */
int or_make_half_gaussian( double sigma, unsigned order, double truncation, int dt_double, double* out, int cap );

/* detail::ExpandBuffer, src/library/copy_buffer.cpp:359-813, for sfloat / dfloat buffers.
 * `buffer` points at the first of `pixels` samples (stride `stride`). */
int or_expand_buffer_f32( float* buffer, ptrdiff_t stride, size_t pixels, size_t left, size_t right, int bc );
int or_expand_buffer_f64( double* buffer, ptrdiff_t stride, size_t pixels, size_t left, size_t right, int bc );

/* dip::GaussFIR (src/linear/gauss.cpp:238-286) -> dip::SeparableConvolution
 * (src/linear/convolution.cpp:319-421) -> dip::Framework::Separable
 * (src/library/framework_separable.cpp:35-431), with the reference's per-pass float semantics.
 *
 * `in`: `ndims` dims, sizes `sizes`, strides `in_strides` (samples), type `in_dtype`.
 * `out`: same sizes, strides `out_strides`, type `out_dtype`.  `out_dtype` is normally the type
 * the reference chooses (sfloat, or dfloat for 32/64-bit integers and dfloat input); any other
 * type reproduces the reference's protected-output path (intermediate image + clamp_cast).
 * `sigmas`, `orders`, `bcs`: one entry per dimension (already broadcast).
 * Returns OR_OK or an error code. */
int or_gauss_fir( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                  void* out, int out_dtype, int64_t const* out_strides,
                  double const* sigmas, unsigned const* orders, int const* bcs, double truncation );

/* dip::SeparableConvolution with caller-supplied EVEN (odd[d] = 0) / ODD (odd[d] = 1) real filters:
 * taps[d] holds lens[d] values, the centre tap FIRST; taps[d] == NULL leaves axis d unfiltered. */
int or_separable_fir( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                      void* out, int out_dtype, int64_t const* out_strides,
                      double const* const* taps, int const* lens, int const* odd, int const* bcs );

/* Filter symmetry (dip::OneDimensionalFilter::symmetry: "general", "even", "odd", "d-even",
 * "d-odd"; "conj" and "d-conj" are "even" and "d-even" for real filters). */
enum { OR_SYM_GENERAL = 0, OR_SYM_EVEN = 1, OR_SYM_ODD = 2, OR_SYM_D_EVEN = 3, OR_SYM_D_ODD = 4 };

/* dip::SeparableConvolution (src/linear/convolution.cpp:319-421) with real filters as given to
 * DIPlib: per filter the data (lens[i] values, up to 4096), origin (-1: centre) and symmetry;
 * `nfilters` 1 (used on every axis) or ndims.  `process` (NULL: all axes). */
int or_separable_convolution( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                              void* out, int out_dtype, int64_t const* out_strides, int nfilters,
                              double const* const* data, int const* lens, long const* origins, int const* symmetries,
                              int const* bcs, int const* process );

/* dip::Uniform with a rectangular kernel (src/linear/uniform.cpp:33-86): per-axis filter sizes
 * (axes with size <= 1 unfiltered), running-sum line filter. */
int or_uniform_rect( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                     void* out, int out_dtype, int64_t const* out_strides, int64_t const* filter_sizes, int const* bcs );

/* Output/compute type rule: DataType::SuggestFlex, src/library/datatype.cpp:109-124. */
int or_suggest_flex( int dtype );

/* dip::GaussIIR (src/linear/gaussiir.cpp:725-790): recursive Gaussian (derivative) filter, orders
 * 0-4, computed in dfloat.  `filter_orders` NULL: the reference's defaults; `forward_backward` 0:
 * "discrete time fit", 1: "forward backward". */
int or_gauss_iir( void const* in, int in_dtype, int ndims, int64_t const* sizes, int64_t const* in_strides,
                  void* out, int out_dtype, int64_t const* out_strides, double const* sigmas, unsigned const* orders,
                  int const* bcs, unsigned const* filter_orders, int forward_backward, double truncation );

#ifdef __cplusplus
}
#endif

#endif
