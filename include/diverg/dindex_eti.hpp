/**
 *  @file  diverg/dindex_eti.hpp
 *  @brief The non-template distance-index entry points (reference ETI surface).
 *
 *  The reference's include/diverg/dindex_eti.hpp:44-53 and
 *  src/eti/dindex.cpp:23-40: create_distance_index for the <uint32_t,
 *  uint64_t> and <uint32_t, uint32_t> range-CRS matrices, here inline over
 *  libdvg.so (no Kokkos, no separate compiled library to link besides it).
 */
#ifndef DIVERG_B200_DINDEX_ETI_HPP__
#define DIVERG_B200_DINDEX_ETI_HPP__

#include <cstdint>

#include "dindex.hpp"

namespace diverg {
  namespace util {
    inline CRSMatrix< crs_matrix::RangeDynamic, bool, uint32_t, uint64_t >
    create_distance_index( CRSMatrix< crs_matrix::RangeDynamic, bool, uint32_t, uint64_t > const& ra,
                           unsigned int dmin, unsigned int dmax )
    {
      return create_distance_index( ra, dmin, dmax, DefaultSparseConfiguration{} );
    }

    inline CRSMatrix< crs_matrix::RangeDynamic, bool, uint32_t, uint32_t >
    create_distance_index( CRSMatrix< crs_matrix::RangeDynamic, bool, uint32_t, uint32_t > const& ra,
                           unsigned int dmin, unsigned int dmax )
    {
      return create_distance_index( ra, dmin, dmax, DefaultSparseConfiguration{} );
    }
  }  // namespace util
}  // namespace diverg

#endif  // DIVERG_B200_DINDEX_ETI_HPP__
