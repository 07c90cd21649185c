/**
 *  @file  diverg/crs_matrix.hpp
 *  @brief Range-CRS host container with the reference's interface.
 *
 *  CRSMatrix< crs_matrix::RangeDynamic, bool, uint32_t, TSize > with the
 *  members of the reference's include/diverg/crs_matrix.hpp:1873-2004 (class)
 *  and :1138-1519 (base): numRows, numCols, nnz, rowMap, entry, get_entries,
 *  get_rowmap, operator()(i, j), at(i, j), serialize, load, size_in_bytes.
 *  Storage is the same pair of std::vectors (entries: flattened inclusive
 *  [start, end] column ranges; rowmap: entry offsets, two per range), so the
 *  host-side behaviour and the on-disk bytes are those of the reference.
 *  The B200 path computes on the RangeDynamic spec with uint32_t columns.
 *  CRSMatrix< crs_matrix::RangeCompressed, ... > (crs_matrix.hpp:1050-1133,
 *  :2245-2386 there) stores a built matrix immutably as Elias-delta coded
 *  entries and rowmap (diverg/enc_vector.hpp) and answers the same queries.
 */
#ifndef DIVERG_B200_CRS_MATRIX_HPP__
#define DIVERG_B200_CRS_MATRIX_HPP__

#include <cstdint>
#include <istream>
#include <ostream>
#include <stdexcept>
#include <type_traits>
#include <utility>
#include <vector>

#include "diverg/enc_vector.hpp"

namespace diverg {
  namespace crs_matrix {
    struct RangeDynamic { };
    struct RangeCompressed { };
    struct RangeGroup { };
    struct BasicGroup { };

    /** crs_matrix.hpp:149-169: membership in a row's flattened ranges. */
    template< typename TIter, typename TOrdinal >
    inline bool
    binary_search( TIter begin, TIter end, TOrdinal key, RangeGroup )
    {
      auto first = begin;
      auto len = end - first;
      while ( len > 0 ) {
        auto half = len / 2;
        auto middle = first + half;
        if ( *middle < key ) {
          first = middle + 1;
          len = len - half - 1;
        }
        else len = half;
      }
      if ( ( first - begin ) % 2 ) --first;
      return first != end && *first <= key;
    }

    /** crs_matrix.hpp:175-189 */
    template< typename TSize, typename TEntries >
    inline TSize
    nnz( TEntries const& entries, RangeGroup )
    {
      TSize c = 0;
      for ( std::size_t i = 0; i + 1 < entries.size(); i += 2 ) c += entries[ i + 1 ] - entries[ i ] + 1;
      return c;
    }
  }  // namespace crs_matrix

  template< typename TSpec, typename TValue = bool, typename TOrdinal = uint32_t, typename TSize = uint64_t >
  class CRSMatrix;

  template< typename TOrdinal, typename TSize >
  class CRSMatrix< crs_matrix::RangeDynamic, bool, TOrdinal, TSize > {
    static_assert( std::is_same< TOrdinal, uint32_t >::value, "the B200 path uses uint32_t columns" );
    static_assert( std::is_same< TSize, uint64_t >::value || std::is_same< TSize, uint32_t >::value,
                   "the size type is uint64_t or uint32_t" );

  public:
    typedef crs_matrix::RangeDynamic spec_type;
    typedef bool value_type;
    typedef TOrdinal ordinal_type;
    typedef TSize size_type;
    typedef std::vector< TOrdinal > entries_type;
    typedef std::vector< TSize > rowmap_type;

    CRSMatrix( ) : num_cols( 0 ), m_nnz( 0 ), rowmap( 1, 0 ) { }

    /** crs_matrix.hpp:1894-1902: a zero nnz is recounted from the entries. */
    CRSMatrix( ordinal_type ncols, entries_type e_entries, rowmap_type e_rowmap, size_type e_nnz = 0 )
      : num_cols( ncols ), m_nnz( e_nnz ), entries( std::move( e_entries ) ), rowmap( std::move( e_rowmap ) )
    {
      if ( this->m_nnz == 0 ) this->m_nnz = crs_matrix::nnz< size_type >( this->entries, crs_matrix::RangeGroup{} );
    }

    inline ordinal_type numCols( ) const { return this->num_cols; }
    inline ordinal_type numRows( ) const { return static_cast< ordinal_type >( this->rowmap.size() - 1 ); }
    inline size_type nnz( ) const { return this->m_nnz; }
    inline ordinal_type entry( size_type i ) const { return this->entries[ i ]; }
    inline size_type rowMap( ordinal_type i ) const { return this->rowmap[ i ]; }
    inline entries_type const& get_entries( ) const { return this->entries; }
    inline entries_type& get_entries( ) { return this->entries; }
    inline rowmap_type const& get_rowmap( ) const { return this->rowmap; }
    inline rowmap_type& get_rowmap( ) { return this->rowmap; }

    /** crs_matrix.hpp:1197-1218 */
    inline value_type
    operator()( ordinal_type i, ordinal_type j ) const
    {
      return crs_matrix::binary_search( this->entries.begin() + this->rowmap[ i ],
                                        this->entries.begin() + this->rowmap[ i + 1 ], j,
                                        crs_matrix::RangeGroup{} );
    }

    /** crs_matrix.hpp:1222-1230 */
    inline value_type
    at( ordinal_type i, ordinal_type j ) const
    {
      if ( i >= this->numRows() || j >= this->numCols() ) throw std::runtime_error( "index out of range" );
      return ( *this )( i, j );
    }

    /** crs_matrix.hpp:893-898 */
    inline size_type
    size_in_bytes( ) const
    {
      return this->entries.size() * sizeof( TOrdinal ) + this->rowmap.size() * sizeof( TSize )
             + sizeof( TOrdinal ) + sizeof( TSize );
    }

    inline void
    clear( )
    {
      this->entries.clear();
      this->rowmap.assign( 1, 0 );
      this->num_cols = 0;
      this->m_nnz = 0;
    }

    /** crs_matrix.hpp:1392-1400 and :1986-1991: entries, rowmap (each a uint64
     *  count then the raw elements), ncols and nnz as uint64. */
    inline void
    serialize( std::ostream& out ) const
    {
      write_vector( out, this->entries );
      write_vector( out, this->rowmap );
      write_pod( out, static_cast< uint64_t >( this->num_cols ) );
      write_pod( out, static_cast< uint64_t >( this->m_nnz ) );
    }

    /** crs_matrix.hpp:1402-1409 and :1993-2000 */
    inline void
    load( std::istream& in )
    {
      read_vector( in, this->entries );
      read_vector( in, this->rowmap );
      uint64_t ncols = 0, dnnz = 0;
      read_pod( in, ncols );
      read_pod( in, dnnz );
      this->num_cols = static_cast< ordinal_type >( ncols );
      this->m_nnz = static_cast< size_type >( dnnz );
    }

  private:
    template< typename T >
    static void write_pod( std::ostream& out, T const& v ) { out.write( reinterpret_cast< const char* >( &v ), sizeof( T ) ); }
    template< typename T >
    static void read_pod( std::istream& in, T& v ) { in.read( reinterpret_cast< char* >( &v ), sizeof( T ) ); }
    template< typename T >
    static void
    write_vector( std::ostream& out, std::vector< T > const& v )
    {
      write_pod( out, static_cast< uint64_t >( v.size() ) );
      if ( !v.empty() ) out.write( reinterpret_cast< const char* >( v.data() ), sizeof( T ) * v.size() );
    }
    template< typename T >
    static void
    read_vector( std::istream& in, std::vector< T >& v )
    {
      uint64_t n = 0;
      read_pod( in, n );
      v.resize( n );
      if ( n ) in.read( reinterpret_cast< char* >( v.data() ), sizeof( T ) * n );
    }

    ordinal_type num_cols;
    size_type m_nnz;
    entries_type entries;
    rowmap_type rowmap;
  };

  /** The immutable, compressed form of a range-CRS matrix: entries and rowmap
   *  Elias-delta coded (crs_matrix.hpp:1050-1133: sdsl::enc_vector over
   *  elias_delta), built from a RangeDynamic matrix and read with the same
   *  queries (crs_matrix.hpp:2245-2386).  A row's entries are decoded from the
   *  nearest sample before them; modifying the matrix is not offered, as in
   *  the reference ("A Compressed Range CRS cannot be modified"). */
  template< typename TOrdinal, typename TSize >
  class CRSMatrix< crs_matrix::RangeCompressed, bool, TOrdinal, TSize > {
    static_assert( std::is_same< TOrdinal, uint32_t >::value, "the B200 path uses uint32_t columns" );

  public:
    typedef crs_matrix::RangeCompressed spec_type;
    typedef bool value_type;
    typedef TOrdinal ordinal_type;
    typedef TSize size_type;
    typedef EliasDeltaVector entries_type;
    typedef EliasDeltaVector rowmap_type;
    typedef CRSMatrix< crs_matrix::RangeDynamic, bool, TOrdinal, TSize > mutable_type;

    CRSMatrix( ) : num_cols( 0 ), m_nnz( 0 ), rowmap( std::vector< uint64_t >( 1, 0 ) ) { }

    /** Compresses a built matrix (crs_matrix.hpp:2263-2270: by way of the mutable spec). */
    explicit CRSMatrix( mutable_type const& m )
      : num_cols( m.numCols() ), m_nnz( m.nnz() ), entries( m.get_entries() ), rowmap( m.get_rowmap() )
    { }

    inline ordinal_type numCols( ) const { return this->num_cols; }
    inline ordinal_type numRows( ) const { return static_cast< ordinal_type >( this->rowmap.size() - 1 ); }
    inline size_type nnz( ) const { return this->m_nnz; }
    inline size_type rowMap( ordinal_type i ) const { return static_cast< size_type >( this->rowmap[ i ] ); }
    inline ordinal_type entry( size_type k ) const { return static_cast< ordinal_type >( this->entries[ k ] ); }

    /** Row i's flattened ranges. */
    inline std::vector< ordinal_type >
    row( ordinal_type i ) const
    {
      std::vector< ordinal_type > out;
      this->entries.decode( this->rowMap( i ), this->rowMap( i + 1 ), out );
      return out;
    }

    /** crs_matrix.hpp:1197-1218 over the decoded row. */
    inline value_type
    operator()( ordinal_type i, ordinal_type j ) const
    {
      const std::vector< ordinal_type > r = this->row( i );
      return crs_matrix::binary_search( r.begin(), r.end(), j, crs_matrix::RangeGroup{} );
    }

    inline value_type
    at( ordinal_type i, ordinal_type j ) const
    {
      if ( i >= this->numRows() || j >= this->numCols() ) throw std::runtime_error( "index out of range" );
      return ( *this )( i, j );
    }

    /** crs_matrix.hpp:1127-1132: the coded vectors and the two scalars. */
    inline size_type
    size_in_bytes( ) const
    {
      return static_cast< size_type >( this->entries.size_in_bytes() + this->rowmap.size_in_bytes()
                                       + sizeof( TOrdinal ) + sizeof( TSize ) );
    }

    /** The matrix decoded back into its mutable form. */
    inline mutable_type
    decompress( ) const
    {
      typename mutable_type::entries_type e;
      typename mutable_type::rowmap_type r;
      this->entries.decode( 0, this->entries.size(), e );
      this->rowmap.decode( 0, this->rowmap.size(), r );
      return mutable_type( this->num_cols, std::move( e ), std::move( r ), this->m_nnz );
    }

    /** The two coded vectors (entries, then rowmap), then ncols and nnz as
     *  uint64, in the order of crs_matrix.hpp:1392-1409 and :1986-2000; the
     *  coded vectors are this library's own layout, not sdsl's. */
    inline void
    serialize( std::ostream& out ) const
    {
      this->entries.serialize( out );
      this->rowmap.serialize( out );
      const uint64_t nc = this->num_cols, nz = this->m_nnz;
      out.write( reinterpret_cast< const char* >( &nc ), sizeof( nc ) );
      out.write( reinterpret_cast< const char* >( &nz ), sizeof( nz ) );
    }

    inline void
    load( std::istream& in )
    {
      this->entries.load( in );
      this->rowmap.load( in );
      uint64_t nc = 0, nz = 0;
      in.read( reinterpret_cast< char* >( &nc ), sizeof( nc ) );
      in.read( reinterpret_cast< char* >( &nz ), sizeof( nz ) );
      if ( !in || this->rowmap.size() == 0 ) throw std::runtime_error( "RangeCompressed: malformed stream" );
      this->num_cols = static_cast< ordinal_type >( nc );
      this->m_nnz = static_cast< size_type >( nz );
    }

  private:
    ordinal_type num_cols;
    size_type m_nnz;
    entries_type entries;
    rowmap_type rowmap;
  };

  template< typename TOrdinal = uint32_t, typename TSize = uint64_t >
  using RangeCompressedCRSMatrix = CRSMatrix< crs_matrix::RangeCompressed, bool, TOrdinal, TSize >;

  namespace crs_matrix {
    template< typename T > struct is_range_crs_matrix : std::false_type { };
    template< typename TOrdinal, typename TSize >
    struct is_range_crs_matrix< CRSMatrix< RangeDynamic, bool, TOrdinal, TSize > > : std::true_type { };
    template< typename TOrdinal, typename TSize >
    struct is_range_crs_matrix< CRSMatrix< RangeCompressed, bool, TOrdinal, TSize > > : std::true_type { };
  }  // namespace crs_matrix
}  // namespace diverg

#endif  // DIVERG_B200_CRS_MATRIX_HPP__
