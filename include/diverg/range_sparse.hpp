/**
 *  @file  diverg/range_sparse.hpp
 *  @brief Range SpGEMM / SpAdd / power / identity with the reference's API.
 *
 *  The host-container entry points of the reference's
 *  include/diverg/range_sparse.hpp -- range_spgemm (:2325-2332), range_spadd
 *  (:470-477), range_power (:2362-2368) and create_range_identity_matrix
 *  (:95-110) -- computed on the B200 through the C ABI of include/dvg.h:
 *  inputs are copied to the device, the product runs there, and the result
 *  comes back by value, as the reference's ETI wrappers do.  The sparse
 *  configuration argument is accepted and ignored: the device plan is chosen
 *  by libdvg.so.
 */
#ifndef DIVERG_B200_RANGE_SPARSE_HPP__
#define DIVERG_B200_RANGE_SPARSE_HPP__

#include <type_traits>

#include <dvg.h>

#include "crs_matrix.hpp"
#include "runtime.hpp"

namespace diverg {
  /** Stand-ins for the reference's compile-time configuration tags
   *  (range_sparse_base.hpp:480-498); they carry no behaviour here. */
  struct DefaultSparseConfiguration { };
  struct DefaultExecutionSpace { };

  namespace detail {
    /** A device matrix owned for the duration of a call. */
    class DeviceMatrix {
    public:
      explicit DeviceMatrix( dvg_matrix* m = nullptr ) : m_( m ) { }
      ~DeviceMatrix() { if ( m_ ) dvg_matrix_free( context(), m_ ); }
      DeviceMatrix( DeviceMatrix const& ) = delete;
      DeviceMatrix& operator=( DeviceMatrix const& ) = delete;
      dvg_matrix* get( ) const { return m_; }
      dvg_matrix** out( ) { return &m_; }

    private:
      dvg_matrix* m_;
    };

    template< typename TRCRSMatrix >
    inline void
    upload( TRCRSMatrix const& m, DeviceMatrix& d )
    {
      typedef typename TRCRSMatrix::size_type size_type;
      if ( std::is_same< size_type, uint32_t >::value ) {
        check( dvg_matrix_upload_u32( context(), m.numRows(), m.numCols(),
                                      reinterpret_cast< const uint32_t* >( m.get_rowmap().data() ),
                                      m.get_entries().data(), m.nnz(), d.out() ) );
      }
      else {
        check( dvg_matrix_upload( context(), m.numRows(), m.numCols(),
                                  reinterpret_cast< const uint64_t* >( m.get_rowmap().data() ),
                                  m.get_entries().data(), m.nnz(), d.out() ) );
      }
    }

    template< typename TRCRSMatrix >
    inline TRCRSMatrix
    download( DeviceMatrix const& d )
    {
      typedef typename TRCRSMatrix::size_type size_type;
      uint32_t nrows = 0, ncols = 0;
      uint64_t nentries = 0, nnz = 0;
      check( dvg_matrix_info( d.get(), &nrows, &ncols, &nentries, &nnz ) );
      typename TRCRSMatrix::entries_type entries( nentries );
      typename TRCRSMatrix::rowmap_type rowmap( size_t( nrows ) + 1 );
      if ( std::is_same< size_type, uint32_t >::value ) {
        check( dvg_matrix_download_u32( context(), d.get(), reinterpret_cast< uint32_t* >( rowmap.data() ),
                                        entries.data() ) );
      }
      else {
        check( dvg_matrix_download( context(), d.get(), reinterpret_cast< uint64_t* >( rowmap.data() ),
                                    entries.data() ) );
      }
      return TRCRSMatrix( ncols, std::move( entries ), std::move( rowmap ), static_cast< size_type >( nnz ) );
    }
  }  // namespace detail

  /** range_sparse.hpp:95-110 */
  template< typename TRCRSMatrix, typename TExecSpace = DefaultExecutionSpace >
  inline TRCRSMatrix
  create_range_identity_matrix( typename TRCRSMatrix::ordinal_type n, TExecSpace = {} )
  {
    detail::DeviceMatrix d;
    detail::check( dvg_range_identity( detail::context(), n, d.out() ) );
    return detail::download< TRCRSMatrix >( d );
  }

  /** range_sparse.hpp:470-477 */
  template< typename TRCRSMatrix, typename TExecSpace = DefaultExecutionSpace >
  inline TRCRSMatrix
  range_spadd( TRCRSMatrix const& a, TRCRSMatrix const& b, TExecSpace = {} )
  {
    detail::DeviceMatrix da, db, dc;
    detail::upload( a, da );
    detail::upload( b, db );
    detail::check( dvg_range_spadd( detail::context(), da.get(), db.get(), dc.out() ) );
    return detail::download< TRCRSMatrix >( dc );
  }

  /** range_sparse.hpp:2325-2332 */
  template< typename TRCRSMatrix, typename TSparseConfig = DefaultSparseConfiguration >
  inline TRCRSMatrix
  range_spgemm( TRCRSMatrix const& a, TRCRSMatrix const& b, TSparseConfig = {} )
  {
    detail::DeviceMatrix da, db, dc;
    detail::upload( a, da );
    detail::upload( b, db );
    detail::check( dvg_range_spgemm( detail::context(), da.get(), db.get(), dc.out() ) );
    return detail::download< TRCRSMatrix >( dc );
  }

  /** range_sparse.hpp:2362-2368 */
  template< typename TRCRSMatrix, typename TSparseConfig = DefaultSparseConfiguration >
  inline TRCRSMatrix
  range_power( TRCRSMatrix const& a, unsigned int k, TSparseConfig = {} )
  {
    detail::DeviceMatrix da, dc;
    detail::upload( a, da );
    detail::check( dvg_range_power( detail::context(), da.get(), k, dc.out() ) );
    return detail::download< TRCRSMatrix >( dc );
  }
}  // namespace diverg

#endif  // DIVERG_B200_RANGE_SPARSE_HPP__
