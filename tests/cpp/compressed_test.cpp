// The compressed range-CRS container (CRSMatrix<RangeCompressed>) against its
// mutable source: sizes, row pointers, entries, membership, decompression and
// its serialised form, on seeded random matrices, edge cases and the
// reference-layout fixture given as argv[1].  Prints "ok" and exits 0, or
// names the first mismatch and exits 1.
#include <cstdint>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "diverg/crs_matrix.hpp"

using Dyn = diverg::CRSMatrix< diverg::crs_matrix::RangeDynamic, bool, uint32_t, uint64_t >;
using Cmp = diverg::CRSMatrix< diverg::crs_matrix::RangeCompressed, bool, uint32_t, uint64_t >;

static uint64_t state = 42;
static uint64_t next( )
{
  state = state * 6364136223846793005ull + 1442695040888963407ull;
  return state >> 17;
}

static int fail( std::string const& what )
{
  std::cout << "mismatch: " << what << std::endl;
  return 1;
}

// rows of up to max_ranges sorted disjoint ranges in [0, ncols)
static Dyn random_matrix( uint32_t nrows, uint32_t ncols, uint32_t max_ranges, uint32_t max_len )
{
  std::vector< uint32_t > e;
  std::vector< uint64_t > r( 1, 0 );
  for ( uint32_t i = 0; i < nrows; ++i ) {
    const uint32_t k = max_ranges ? uint32_t( next() % ( max_ranges + 1 ) ) : 0;
    uint64_t c = next() % ( ncols / 4 + 1 );
    for ( uint32_t q = 0; q < k && c < ncols; ++q ) {
      const uint64_t len = next() % max_len;
      const uint64_t hi = std::min< uint64_t >( ncols - 1, c + len );
      e.push_back( uint32_t( c ) );
      e.push_back( uint32_t( hi ) );
      c = hi + 2 + next() % 50;
    }
    r.push_back( e.size() );
  }
  return Dyn( ncols, e, r );
}

static int check( Dyn const& d, std::string const& name, bool full )
{
  const Cmp c( d );
  if ( c.numRows() != d.numRows() || c.numCols() != d.numCols() || c.nnz() != d.nnz() ) return fail( name + ": sizes" );
  for ( uint32_t i = 0; i <= d.numRows(); ++i )
    if ( c.rowMap( i ) != d.rowMap( i ) ) return fail( name + ": rowmap " + std::to_string( i ) );
  const uint64_t ne = d.get_entries().size();
  for ( uint64_t k = 0; k < ne; k += full ? 1 : 97 )
    if ( c.entry( k ) != d.entry( k ) ) return fail( name + ": entry " + std::to_string( k ) );
  const uint32_t nr = d.numRows(), ncol = d.numCols();
  if ( nr && ncol ) {
    for ( int q = 0; q < 20000; ++q ) {
      const uint32_t i = uint32_t( next() % nr ), j = uint32_t( next() % ncol );
      if ( c( i, j ) != d( i, j ) ) return fail( name + ": membership" );
    }
    for ( uint32_t i = 0; i < nr; i += full ? 1 : 131 ) {  // every range end and the column after it
      for ( uint64_t k = d.rowMap( i ); k < d.rowMap( i + 1 ); ++k ) {
        const uint32_t j = d.entry( k );
        if ( c( i, j ) != d( i, j ) ) return fail( name + ": membership at a bound" );
        if ( j + 1 < ncol && c( i, j + 1 ) != d( i, j + 1 ) ) return fail( name + ": membership past a bound" );
      }
    }
  }
  const Dyn back = c.decompress();
  if ( back.get_entries() != d.get_entries() || back.get_rowmap() != d.get_rowmap() || back.nnz() != d.nnz()
       || back.numCols() != d.numCols() )
    return fail( name + ": decompress" );
  std::stringstream ss;
  c.serialize( ss );
  Cmp l;
  l.load( ss );
  const Dyn back2 = l.decompress();
  if ( back2.get_entries() != d.get_entries() || back2.get_rowmap() != d.get_rowmap() || l.nnz() != d.nnz() )
    return fail( name + ": serialize and load" );
  return 0;
}

int main( int argc, char** argv )
{
  int bad = 0;
  bad |= check( Dyn( 7, {}, std::vector< uint64_t >( 1, 0 ) ), "no rows", true );
  bad |= check( Dyn( 9, {}, std::vector< uint64_t >( 6, 0 ) ), "empty rows", true );
  bad |= check( random_matrix( 300, 1000, 4, 20 ), "small", true );
  bad |= check( random_matrix( 20000, 4000000, 30, 5000 ), "wide rows", false );
  {  // columns near the top of uint32_t, and rows that restart far below the last
    std::vector< uint32_t > e = { 4294967290u, 4294967293u, 0u, 0u, 5u, 4294967292u, 3u, 3u };
    std::vector< uint64_t > r = { 0, 2, 4, 6, 8 };
    bad |= check( Dyn( 4294967294u, e, r ), "extreme columns", true );
  }
  {  // an index-like matrix: one range a row near the diagonal compresses well
    std::vector< uint32_t > e;
    std::vector< uint64_t > r( 1, 0 );
    for ( uint32_t i = 0; i < 200000; ++i ) {
      e.push_back( i + 400 + uint32_t( next() % 4 ) );
      e.push_back( i + 600 + uint32_t( next() % 4 ) );
      r.push_back( e.size() );
    }
    const Dyn d( 201000, e, r );
    bad |= check( d, "index-like", false );
    const Cmp c( d );
    if ( c.size_in_bytes() * 3 > d.size_in_bytes() ) bad |= fail( "index-like: compressed to more than a third" );
  }
  if ( argc > 1 ) {  // the reference-layout fixture: compress, decompress, same bytes
    std::ifstream f( argv[ 1 ], std::ios::binary );
    Dyn d;
    d.load( f );
    bad |= check( d, "fixture", true );
    std::stringstream a, b;
    d.serialize( a );
    Cmp( d ).decompress().serialize( b );
    if ( a.str() != b.str() ) bad |= fail( "fixture: bytes after a round trip" );
  }
  if ( !bad ) std::cout << "ok" << std::endl;
  return bad;
}
