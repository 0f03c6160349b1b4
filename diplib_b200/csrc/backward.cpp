// dipcu_gauss_fir_backward: gradients of the Gaussian FIR with respect to its input and to each
// sigma.  No DIPlib counterpart; the forward it differentiates is dip::GaussFIR
// (src/linear/gauss.cpp:238-286), pass by pass as dip::Framework::Separable runs it
// (src/library/framework_separable.cpp:35-431): y = P_d ... P_1 x with P_a = C_a E_a.
//
//  * x_bar = P_1^T ... P_d^T y_bar, each P_a^T = E_a^T C_a^T evaluated as a zero-padded correlation
//    with the flipped taps (the line kernel with "add zeros"; odd kernels negate) followed by the
//    fold of the halo gradients through the boundary extension's coefficients.
//  * d L / d sigma_a = <y_bar, G_a'(x)>, with G_a' the forward filter whose axis-a taps are
//    replaced by their analytic sigma derivative (kernel length held fixed).  G_a'(x) is
//    recomputed here, never stored by the forward.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "dipcu_common.cuh"
#include "dipcu_internal.h"

namespace dipcu {

namespace {

// Coefficients of the boundary extension of a line of length n by h samples on both sides, for
// every halo position: z_j = sum_i c_ji x_i.  Evaluated with the forward's own bc_extend on unit
// vectors over the candidate sources (the mapped index and the two samples at each end).
int fold_entries( int64_t n, int64_t h, int32_t bc, std::vector< FoldEntry >& out ) {
   out.clear();
   for( int64_t j = -h; j < n + h; ++j ) {
      if( j == 0 ) { j = n; }                       // skip the interior
      if( j >= n + h ) { break; }
      int64_t cand[ 5 ];
      int nc = 0;
      bool neg = false;
      int64_t m = ( bc == BC_ADD_ZEROS || bc == BC_ADD_MAX_VALUE || bc == BC_ADD_MIN_VALUE ) ? -1
                  : bc_map_index( j, n, bc == BC_ANTISYMMETRIC_REFLECT ? BC_SYMMETRIC_MIRROR : bc, &neg );
      int64_t const extra[ 5 ] = { m, 0, 1, n - 2, n - 1 };
      for( int64_t c : extra ) {
         if( c < 0 || c >= n ) { continue; }
         bool dup = false;
         for( int k = 0; k < nc; ++k ) { dup |= cand[ k ] == c; }
         if( !dup ) { cand[ nc++ ] = c; }
      }
      for( int k = 0; k < nc; ++k ) {
         int64_t const i0 = cand[ k ];
         auto unit = [ & ]( int64_t i ) { return i == i0 ? 1.0 : 0.0; };
         auto zero = []( int64_t ) { return 0.0; };
         // Affine BCs ("add max"/"add min" are constants): subtract the value at x = 0.
         double c = bc_extend< double >( j, n, bc, h, unit ) - bc_extend< double >( j, n, bc, h, zero );
         if( c != 0.0 ) {
            if( out.size() >= static_cast< size_t >( kFoldMaxEntries )) { return -1; }
            out.push_back( FoldEntry{ static_cast< int32_t >( j ), static_cast< int32_t >( i0 ), c } );
         }
      }
   }
   return 0;
}

int fail_cuda( cudaError_t e, char const* where ) {
   std::string msg = std::string( where ) + ": " + cudaGetErrorString( e );
   return record_error( DIPCU_ERR_CUDA, msg.c_str() );
}

// The whole 2D backward in one kernel (input gradient and both sigma gradients) when the layout
// allows it: both processed axes filtered in float, x the axis of unit stride in grad_out,
// grad_in and in, at most one other axis of size > 1 (a batch).  Returns -1 when it does not
// apply, else the status.
int try_fused_adjoint( dipcu_image_desc const* grad_out, dipcu_image_desc const* in, dipcu_image_desc const* grad_in,
                       double* grad_sigma, std::vector< AxisFilter > const& f, std::vector< std::vector< double >> const& df,
                       std::vector< int > const& order, cudaStream_t stream ) {
   int const nd = grad_out->ndims;
   int ax = -1, ay = -1;
   for( int d : order ) {
      bool unit = grad_out->strides[ d ] == 1 && ( !grad_in || grad_in->strides[ d ] == 1 ) &&
                  ( !grad_sigma || ( in && in->strides[ d ] == 1 ));
      if( unit && ax < 0 ) { ax = d; }
   }
   if( ax < 0 ) { return -1; }
   for( int d : order ) { if( d != ax ) { ay = d; } }
   int batch = -1;
   for( int d = 0; d < nd; ++d ) {
      if( d == ax || d == ay || grad_out->sizes[ d ] == 1 ) { continue; }
      if( batch >= 0 ) { return -1; }
      batch = d;
   }
   if( grad_sigma && ( !in || !( in->dtype == DT_SFLOAT || in->dtype == DT_UINT16 ))) { return -1; }
   Adj2Params p{};
   p.gy = static_cast< float const* >( grad_out->data );
   p.gys1 = grad_out->strides[ ay ];
   p.gyb = batch >= 0 ? grad_out->strides[ batch ] : 0;
   p.x = grad_sigma ? in->data : nullptr;
   p.x_dt = grad_sigma ? in->dtype : DT_SFLOAT;
   p.xs1 = grad_sigma ? in->strides[ ay ] : 0;
   p.xb = ( grad_sigma && batch >= 0 ) ? in->strides[ batch ] : 0;
   p.gx = grad_in ? static_cast< float* >( grad_in->data ) : nullptr;
   p.gxs1 = grad_in ? grad_in->strides[ ay ] : 0;
   p.gxb = ( grad_in && batch >= 0 ) ? grad_in->strides[ batch ] : 0;
   p.n[ 0 ] = grad_out->sizes[ ax ];
   p.n[ 1 ] = grad_out->sizes[ ay ];
   p.nb = batch >= 0 ? grad_out->sizes[ batch ] : 1;
   int const axes[ 2 ] = { ax, ay };
   for( int i = 0; i < 2; ++i ) {
      AxisFilter const& af = f[ static_cast< size_t >( axes[ i ] ) ];
      p.bc[ i ] = af.bc;
      p.h[ i ] = static_cast< int32_t >( af.h );
      p.odd[ i ] = af.odd;
      p.taps[ i ] = af.taps.data();
      p.dtaps[ i ] = df[ static_cast< size_t >( axes[ i ] ) ].data();
   }
   if( grad_sigma ) {
      cudaError_t e = cudaMemsetAsync( grad_sigma, 0, sizeof( double ) * static_cast< size_t >( nd ), stream );
      if( e != cudaSuccess ) { return fail_cuda( e, "cudaMemsetAsync" ); }
      p.dsig[ 0 ] = grad_sigma + ax;
      p.dsig[ 1 ] = grad_sigma + ay;
   }
   cudaError_t e = launch_fused_adjoint2d( p, stream );
   if( e == cudaErrorNotSupported ) { return -1; }
   if( e != cudaSuccess ) { return fail_cuda( e, "fused2d_adj_kernel" ); }
   return DIPCU_OK;
}

} // namespace

} // namespace dipcu

using namespace dipcu;

extern "C" int dipcu_gauss_fir_backward( dipcu_image_desc const* grad_out, dipcu_image_desc const* in,
                                          dipcu_image_desc const* grad_in, double* grad_sigma,
                                          double const* sigmas, uint32_t const* orders, int32_t const* bcs,
                                          double truncation, void* stream_ ) {
   cudaStream_t stream = static_cast< cudaStream_t >( stream_ );
   if( !grad_out || !sigmas || !orders || !bcs ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "dipcu_gauss_fir_backward: null argument" );
   }
   if( grad_sigma && !in ) {
      return record_error( DIPCU_ERR_INVALID_ARG, "dipcu_gauss_fir_backward: the sigma gradient needs the input image" );
   }
   dipcu_image_desc const* ref = in ? in : grad_out;
   int32_t const cdt = in ? suggest_flex( in->dtype ) : grad_out->dtype;
   bool const cdouble = cdt == DT_DFLOAT;
   if( grad_out->dtype != cdt || ( grad_in && grad_in->dtype != cdt ) || ( cdt != DT_SFLOAT && cdt != DT_DFLOAT )) {
      return record_error( DIPCU_ERR_UNSUPPORTED_DTYPE,
                           "gradients must have the filter's computation type (sfloat, or dfloat for 32/64-bit integer and dfloat input)" );
   }
   if( in ) {
      if( int st = check_pair( in, grad_out )) { return st; }
   }
   if( grad_in ) {
      if( int st = check_pair( grad_out, grad_in )) { return st; }
   }
   std::vector< AxisFilter > f;
   std::vector< std::vector< double >> df;
   if( int st = build_filters( ref, sigmas, orders, bcs, truncation, f, &df )) { return st; }
   std::vector< int > order = pass_order( ref, f );
   int const nd = ref->ndims;
   int const P = static_cast< int >( order.size() );
   int64_t n = 1;
   for( int d = 0; d < nd; ++d ) { n *= ref->sizes[ d ]; }
   int64_t normal[ DIPCU_MAX_DIMS ];
   {
      int64_t s = 1;
      for( int d = 0; d < nd; ++d ) { normal[ d ] = s; s *= ref->sizes[ d ]; }
   }
   if( P == 2 && !cdouble && ( grad_in || grad_sigma )) {
      int st = try_fused_adjoint( grad_out, in, grad_in, grad_sigma, f, df, order, stream );
      if( st != -1 ) { return st; }
   }
   size_t const esz = cdouble ? 8 : 4;
   int const nscratch = ( grad_sigma && P > 0 ) ? 2 : ( P > 2 ? 2 : ( P > 1 ? 1 : 0 ));
   void* scratch[ 2 ] = { nullptr, nullptr };
   for( int i = 0; i < nscratch; ++i ) {
      cudaError_t e = cudaMallocAsync( &scratch[ i ], static_cast< size_t >( n ) * esz, stream );
      if( e != cudaSuccess ) {
         for( int k = 0; k < i; ++k ) { cudaFreeAsync( scratch[ k ], stream ); }
         return fail_cuda( e, "cudaMallocAsync (backward intermediate)" );
      }
   }
   int status = DIPCU_OK;
   auto done = [ & ]( int st ) {
      for( int i = 0; i < nscratch; ++i ) { cudaFreeAsync( scratch[ i ], stream ); }
      return st;
   };

   // ---- input gradient: the adjoint passes in reverse order.
   if( grad_in ) {
      if( P == 0 ) {
         dipcu_image_desc go = *grad_out;
         status = run_filters( &go, grad_in, f, cdouble, stream );   // identity copy
         if( status ) { return done( status ); }
      }
      void const* cur = grad_out->data;
      int64_t const* cur_st = grad_out->strides;
      for( int idx = P - 1; idx >= 0; --idx ) {
         int const ax = order[ idx ];
         AxisFilter const& af = f[ static_cast< size_t >( ax ) ];
         bool const last = idx == 0;
         void* dst = last ? grad_in->data : scratch[ ( P - 1 - idx ) % 2 ];
         int64_t const* dst_st = last ? grad_in->strides : normal;
         std::vector< double > flipped( af.taps );
         if( af.odd ) { for( auto& t : flipped ) { t = -t; } }
         LinePass lp{};
         lp.src = cur;
         lp.dst = dst;
         lp.src_dt = cdt;
         lp.dst_dt = cdt;
         lp.ndims = nd;
         lp.axis = ax;
         for( int d = 0; d < nd; ++d ) {
            lp.sizes[ d ] = ref->sizes[ d ];
            lp.src_strides[ d ] = cur_st[ d ];
            lp.dst_strides[ d ] = dst_st[ d ];
         }
         lp.h = af.h;
         lp.odd = af.odd;
         lp.bc = BC_ADD_ZEROS;
         lp.compute_double = cdouble;
         lp.taps = flipped.data();
         cudaError_t e = launch_line_pass( lp, stream );
         if( e != cudaSuccess ) { return done( fail_cuda( e, "line_pass_kernel (adjoint)" )); }
         std::vector< FoldEntry > entries;
         if( af.h > kFoldMaxHalf || fold_entries( ref->sizes[ ax ], af.h, af.bc, entries ) != 0 ) {
            return done( record_error( DIPCU_ERR_KERNEL_TOO_LARGE, "the backward supports kernel half-widths up to 100" ));
         }
         FoldPass fp{};
         fp.g = cur;
         fp.xb = dst;
         fp.ndims = nd;
         fp.axis = ax;
         for( int d = 0; d < nd; ++d ) {
            fp.sizes[ d ] = ref->sizes[ d ];
            fp.gst[ d ] = cur_st[ d ];
            fp.xst[ d ] = dst_st[ d ];
         }
         fp.h = af.h;
         fp.odd = af.odd;
         fp.compute_double = cdouble;
         fp.taps = af.taps.data();
         fp.entries = entries.data();
         fp.nentries = static_cast< int32_t >( entries.size() );
         e = launch_fold( fp, stream );
         if( e != cudaSuccess ) { return done( fail_cuda( e, "fold_kernel" )); }
         cur = dst;
         cur_st = dst_st;
      }
   }

   // ---- sigma gradients: <y_bar, G_a'(x)> per processed axis.
   if( grad_sigma ) {
      cudaError_t e = cudaMemsetAsync( grad_sigma, 0, sizeof( double ) * static_cast< size_t >( nd ), stream );
      if( e != cudaSuccess ) { return done( fail_cuda( e, "cudaMemsetAsync" )); }
      dipcu_image_desc tmp{};
      tmp.data = scratch[ 0 ];
      tmp.dtype = cdt;
      tmp.ndims = nd;
      for( int d = 0; d < nd; ++d ) { tmp.sizes[ d ] = ref->sizes[ d ]; tmp.strides[ d ] = normal[ d ]; }
      for( int ax : order ) {
         std::vector< AxisFilter > fd( f );
         fd[ static_cast< size_t >( ax ) ].taps = df[ static_cast< size_t >( ax ) ];
         status = run_filters( in, &tmp, fd, cdouble, stream );
         if( status ) { return done( status ); }
         ConvertArgs c{};
         c.src = tmp.data;
         c.dst = grad_out->data;
         c.src_dt = cdt;
         c.dst_dt = cdt;
         c.ndims = nd;
         c.total = n;
         for( int d = 0; d < nd; ++d ) {
            c.sizes[ d ] = ref->sizes[ d ];
            c.sst[ d ] = normal[ d ];
            c.dstst[ d ] = grad_out->strides[ d ];
         }
         e = launch_dot( c, cdouble, grad_sigma + ax, stream );
         if( e != cudaSuccess ) { return done( fail_cuda( e, "dot_kernel" )); }
      }
   }
   return done( DIPCU_OK );
}
