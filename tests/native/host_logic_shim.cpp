// Test-only: exposes the __host__ __device__ helpers of diplib_b200/csrc/dipcu_common.cuh,
// compiled for the host, so that tests/test_host_logic.py can check them against the oracle on
// a machine without a GPU.  The same source is what the kernels run.
#include <stdint.h>

#include "dipcu_common.cuh"

extern "C" {

// Extends `n` float samples at `line` by `border` samples on each side into `out`
// (length n + 2 * border) with dipcu::bc_extend.
void hl_extend_f32( float const* line, int64_t n, int64_t border, int32_t bc, float* out ) {
   auto ld = [ & ]( int64_t i ) { return line[ i ]; };
   for( int64_t j = -border; j < n + border; ++j ) {
      out[ j + border ] = ( j >= 0 && j < n ) ? line[ j ] : dipcu::bc_extend< float >( j, n, bc, border, ld );
   }
}

int64_t hl_half_gaussian_length( double sigma, uint32_t order, double truncation, int dt_double ) {
   return dipcu::half_gaussian_length( sigma, order, truncation, dt_double != 0 );
}

// Reversed half kernel (centre first) in double, and its sigma derivative.
void hl_make_half_gaussian( double sigma, uint32_t order, int64_t len, double* w, double* dw ) {
   dipcu::make_half_gaussian< double >( sigma, order, len, w, dw );
}

// exp rounded to the nearest double (the device weights' exp), evaluated on the host.
double hl_exp_rn( double x ) {
   return dipcu::exp_rn( x );
}

} // extern "C"
