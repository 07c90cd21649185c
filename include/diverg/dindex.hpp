/**
 *  @file  diverg/dindex.hpp
 *  @brief util::create_distance_index with the reference's template signature.
 *
 *  The reference's include/diverg/dindex.hpp:46-189: the index
 *  A^dlo * (A + I)^(dup - dlo) of a range-CRS adjacency `ra`, here built on the
 *  B200 through the C ABI of include/dvg.h with every intermediate resident in
 *  device memory.  Requires dlo <= dup and dup != 0; where the reference
 *  aborts (DIVERG_ASSERT, exit 134) this throws std::runtime_error.  The
 *  configuration argument is ignored; `timer1` (when given) is reset before
 *  and read after the device build, measuring it without the host<->device
 *  copies as the reference's DIVERG_STATS timer does.
 */
#ifndef DIVERG_B200_DINDEX_HPP__
#define DIVERG_B200_DINDEX_HPP__

#include <chrono>
#include <stdexcept>

#include "range_sparse.hpp"

namespace diverg {
  /** A wall-clock stand-in for Kokkos::Timer (reset / seconds). */
  class Timer {
  public:
    Timer( ) : t0_( std::chrono::steady_clock::now() ) { }
    void reset( ) { t0_ = std::chrono::steady_clock::now(); }
    double seconds( ) const
    {
      return std::chrono::duration< double >( std::chrono::steady_clock::now() - t0_ ).count();
    }

  private:
    std::chrono::steady_clock::time_point t0_;
  };

  namespace util {
    template< typename TRCRSMatrix, typename TSparseConfig = DefaultSparseConfiguration, typename TTimer = Timer >
    inline TRCRSMatrix
    create_distance_index( TRCRSMatrix const& ra, unsigned int dlo, unsigned int dup, TSparseConfig = {},
                           TTimer* timer1_ptr = nullptr, TTimer* /* timer2_ptr */ = nullptr )
    {
      static_assert( crs_matrix::is_range_crs_matrix< TRCRSMatrix >::value, "matrix should be in Range CRS format." );
      detail::DeviceMatrix da, dd;
      detail::upload( ra, da );
      if ( timer1_ptr ) timer1_ptr->reset();
      detail::check( dvg_create_distance_index( detail::context(), da.get(), dlo, dup, dd.out() ) );
      return detail::download< TRCRSMatrix >( dd );
    }

    /** dindex.hpp:556-570 (dispatching to :435-469): two distance indices of
     *  the same graph merge into their union A + B, which the reference
     *  computes with range_spadd for in-core range matrices, as here on the
     *  device.  The result is a mutable (RangeDynamic) matrix. */
    template< typename TMutableCRSMatrix, typename TCRSMatrix >
    inline TMutableCRSMatrix
    merge_distance_index( TCRSMatrix& dindex1, TCRSMatrix& dindex2 )
    {
      static_assert( crs_matrix::is_range_crs_matrix< TCRSMatrix >::value
                         && crs_matrix::is_range_crs_matrix< TMutableCRSMatrix >::value,
                     "input and output distance indices must be in the same (Range) group" );
      if ( dindex1.numRows() != dindex2.numRows() || dindex1.numCols() != dindex2.numCols() )
        throw std::runtime_error( "diverg: merge_distance_index: the indices differ in shape" );
      detail::DeviceMatrix d1, d2, dm;
      detail::upload( dindex1, d1 );
      detail::upload( dindex2, d2 );
      detail::check( dvg_range_spadd( detail::context(), d1.get(), d2.get(), dm.out() ) );
      return detail::download< TMutableCRSMatrix >( dm );
    }
  }  // namespace util
}  // namespace diverg

#endif  // DIVERG_B200_DINDEX_HPP__
