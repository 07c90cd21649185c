/**
 *    @file  enc_vector.hpp
 *   @brief  An immutable integer vector stored as Elias-delta codes of the
 *           differences of consecutive elements, with sampled absolute values
 *           for random access.
 *
 *  The storage of the reference's RangeCompressed range-CRS matrices
 *  (crs_matrix.hpp:1050-1133 in cartoonist/diverg: sdsl::enc_vector over
 *  sdsl::coder::elias_delta for entries and rowmap) restated on its published
 *  method: every element but each 128th is the Elias-delta code of its
 *  difference to the element before it; each 128th element is kept whole
 *  together with the bit position of the next code, so element i costs one
 *  sample read and at most 127 code reads.  Differences are signed (the
 *  entries of a range CRS restart in every row) and enter the code zig-zag
 *  mapped, plus one (Elias-delta codes integers >= 1).  The bit layout and the
 *  serialised form are this library's own: sdsl's is a third-party format
 *  that is not reproduced.
 */
#ifndef DIVERG_B200_ENC_VECTOR_HPP__
#define DIVERG_B200_ENC_VECTOR_HPP__

#include <cstdint>
#include <istream>
#include <ostream>
#include <stdexcept>
#include <vector>

namespace diverg {
  class EliasDeltaVector {
  public:
    static constexpr uint64_t sample_every = 128;

    EliasDeltaVector( ) : n( 0 ), nbits( 0 ) { }

    template< typename TVector >
    explicit EliasDeltaVector( TVector const& v ) : n( 0 ), nbits( 0 )
    {
      this->n = v.size();
      uint64_t prev = 0;
      for ( uint64_t i = 0; i < this->n; ++i ) {
        const uint64_t x = static_cast< uint64_t >( v[ i ] );
        if ( i % sample_every == 0 ) {
          this->samples.push_back( x );
          this->ptrs.push_back( this->nbits );
        }
        else {
          this->put_code( zigzag( static_cast< int64_t >( x - prev ) ) + 1 );
        }
        prev = x;
      }
    }

    inline uint64_t size( ) const { return this->n; }
    inline bool empty( ) const { return this->n == 0; }

    /** Element i. */
    inline uint64_t
    operator[]( uint64_t i ) const
    {
      const uint64_t s = i / sample_every;
      uint64_t x = this->samples[ s ];
      uint64_t pos = this->ptrs[ s ];
      for ( uint64_t k = s * sample_every + 1; k <= i; ++k ) x += unzigzag( this->get_code( pos ) - 1 );
      return x;
    }

    /** Elements [begin, end) into out (one sample read, then the codes). */
    template< typename T >
    inline void
    decode( uint64_t begin, uint64_t end, std::vector< T >& out ) const
    {
      out.clear();
      if ( begin >= end ) return;
      out.reserve( end - begin );
      const uint64_t s = begin / sample_every;
      uint64_t x = this->samples[ s ];
      uint64_t pos = this->ptrs[ s ];
      for ( uint64_t k = s * sample_every; k < end; ++k ) {
        if ( k % sample_every == 0 ) {
          x = this->samples[ k / sample_every ];
          pos = this->ptrs[ k / sample_every ];
        }
        else {
          x += unzigzag( this->get_code( pos ) - 1 );
        }
        if ( k >= begin ) out.push_back( static_cast< T >( x ) );
      }
    }

    /** Bytes held: samples, code pointers and the code stream. */
    inline uint64_t
    size_in_bytes( ) const
    {
      return sizeof( uint64_t ) * ( this->samples.size() + this->ptrs.size() + this->words.size() + 2 );
    }

    /** n, bits, then samples, pointers and code words (each a uint64 count
     *  and the raw little-endian words). */
    inline void
    serialize( std::ostream& out ) const
    {
      write_pod( out, this->n );
      write_pod( out, this->nbits );
      write_vec( out, this->samples );
      write_vec( out, this->ptrs );
      write_vec( out, this->words );
    }

    inline void
    load( std::istream& in )
    {
      read_pod( in, this->n );
      read_pod( in, this->nbits );
      read_vec( in, this->samples );
      read_vec( in, this->ptrs );
      read_vec( in, this->words );
      if ( !in || this->samples.size() != ( this->n + sample_every - 1 ) / sample_every
           || this->ptrs.size() != this->samples.size() || this->words.size() != ( this->nbits + 63 ) / 64 )
        throw std::runtime_error( "EliasDeltaVector: malformed stream" );
    }

  private:
    static inline uint64_t zigzag( int64_t d ) { return ( static_cast< uint64_t >( d ) << 1 ) ^ static_cast< uint64_t >( d >> 63 ); }
    static inline int64_t unzigzag( uint64_t z ) { return static_cast< int64_t >( z >> 1 ) ^ -static_cast< int64_t >( z & 1 ); }

    static inline unsigned bit_length( uint64_t x )
    {
      unsigned l = 0;
      while ( x ) { ++l; x >>= 1; }
      return l;
    }

    /** Appends the `len` low bits of v, most significant first. */
    inline void
    put_bits( uint64_t v, unsigned len )
    {
      for ( unsigned k = len; k > 0; --k ) {
        const uint64_t bit = ( v >> ( k - 1 ) ) & 1u;
        if ( this->nbits % 64 == 0 ) this->words.push_back( 0 );
        if ( bit ) this->words.back() |= uint64_t( 1 ) << ( 63 - this->nbits % 64 );
        ++this->nbits;
      }
    }

    inline uint64_t
    get_bit( uint64_t pos ) const
    {
      return ( this->words[ pos / 64 ] >> ( 63 - pos % 64 ) ) & 1u;
    }

    inline uint64_t
    get_bits( uint64_t& pos, unsigned len ) const
    {
      uint64_t v = 0;
      for ( unsigned k = 0; k < len; ++k ) v = ( v << 1 ) | this->get_bit( pos++ );
      return v;
    }

    /** Elias delta: (L - 1) zeros, N in L bits, then the N - 1 bits of x
     *  below its leading one, where N = bits of x and L = bits of N. */
    inline void
    put_code( uint64_t x )
    {
      const unsigned nb = bit_length( x ), lb = bit_length( nb );
      this->put_bits( 0, lb - 1 );
      this->put_bits( nb, lb );
      this->put_bits( x, nb - 1 );
    }

    inline uint64_t
    get_code( uint64_t& pos ) const
    {
      unsigned zeros = 0;
      while ( this->get_bit( pos ) == 0 ) {
        ++zeros;
        ++pos;
        if ( zeros > 6 ) throw std::runtime_error( "EliasDeltaVector: malformed code" );
      }
      const unsigned nb = static_cast< unsigned >( this->get_bits( pos, zeros + 1 ) );
      if ( nb == 0 || nb > 64 ) throw std::runtime_error( "EliasDeltaVector: malformed code" );
      const uint64_t low = this->get_bits( pos, nb - 1 );
      return nb == 64 ? ( uint64_t( 1 ) << 63 ) | low : ( uint64_t( 1 ) << ( nb - 1 ) ) | low;
    }

    template< typename T >
    static void write_pod( std::ostream& out, T const& v ) { out.write( reinterpret_cast< const char* >( &v ), sizeof( T ) ); }
    template< typename T >
    static void read_pod( std::istream& in, T& v ) { in.read( reinterpret_cast< char* >( &v ), sizeof( T ) ); }
    static void
    write_vec( std::ostream& out, std::vector< uint64_t > const& v )
    {
      write_pod( out, static_cast< uint64_t >( v.size() ) );
      if ( !v.empty() ) out.write( reinterpret_cast< const char* >( v.data() ), sizeof( uint64_t ) * v.size() );
    }
    static void
    read_vec( std::istream& in, std::vector< uint64_t >& v )
    {
      uint64_t c = 0;
      read_pod( in, c );
      if ( !in || c > ( uint64_t( 1 ) << 40 ) ) throw std::runtime_error( "EliasDeltaVector: malformed stream" );
      v.resize( c );
      if ( c ) in.read( reinterpret_cast< char* >( v.data() ), sizeof( uint64_t ) * c );
    }

    uint64_t n;
    uint64_t nbits;
    std::vector< uint64_t > samples;  // element i * sample_every
    std::vector< uint64_t > ptrs;     // bit position of the code of element i * sample_every + 1
    std::vector< uint64_t > words;    // the codes, bit 0 the most significant bit of word 0
  };
}  // namespace diverg

#endif  // DIVERG_B200_ENC_VECTOR_HPP__
