/**
 *  @file  diverg/gfa.hpp
 *  @brief A sequence graph read from GFA 1 or GFA 2 text, with the part of
 *         gum's SeqGraph interface that util::range_adjacency_matrix walks.
 *
 *  The reference loads graphs with gum (gum::util::load_gfa over GFAKluge,
 *  benchmark/src/rcrs_benchmark.hpp:292-376) and then orders the nodes
 *  ("native": the file's order; "topological"; others).  gum is a third-party
 *  library absent here; this reader follows the GFA specifications: segments
 *  (GFA 1 `S name seq [LN:i:len]`, GFA 2 `S sid slen seq`) give the nodes and
 *  their lengths, links (GFA 1 `L from + to + overlap`) and edges (GFA 2
 *  `E eid sid1+ sid2+ ...`) the forward edges.  Node ids are the segment names
 *  when all are positive integers, else 1, 2, ... in file order.  Ordering
 *  "native" ranks nodes in file order; "topological" ranks them by Kahn's
 *  algorithm taking the lowest native rank first, and ranks the nodes of
 *  cycles after, in native order (a semi-topological order, as gum applies
 *  to graphs that are not DAGs).  Edges between opposite strands are not
 *  representable in the forward range adjacency and are rejected.
 */
#ifndef DIVERG_B200_GFA_HPP__
#define DIVERG_B200_GFA_HPP__

#include <algorithm>
#include <cstdint>
#include <istream>
#include <queue>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace diverg {
  namespace gfa {
    class Graph {
    public:
      typedef uint64_t id_type;
      typedef uint64_t rank_type;
      typedef uint8_t linktype_type;

      inline rank_type get_node_count( ) const { return this->ids.size(); }
      inline id_type rank_to_id( rank_type rank ) const { return this->ids.at( rank - 1 ); }
      inline rank_type id_to_rank( id_type id ) const { return this->rank_of.at( id ); }
      inline uint64_t node_length( id_type id ) const { return this->len.at( this->id_to_rank( id ) - 1 ); }

      /** f(rank, id) for ranks from `from` on, while f returns true. */
      template< typename F >
      inline void
      for_each_node( F f, rank_type from = 1 ) const
      {
        for ( rank_type r = from; r <= this->ids.size(); ++r )
          if ( !f( r, this->ids[ r - 1 ] ) ) return;
      }

      /** f(to_id, linktype) for the edges out of node id, while f returns true. */
      template< typename F >
      inline void
      for_each_edges_out( id_type id, F f ) const
      {
        for ( id_type to : this->out.at( this->id_to_rank( id ) - 1 ) )
          if ( !f( to, linktype_type( 0 ) ) ) return;
      }

      std::vector< id_type > ids;                       // id of rank r at r - 1
      std::vector< uint64_t > len;                      // length of the node of rank r at r - 1
      std::vector< std::vector< id_type > > out;        // successors (ids) of the node of rank r at r - 1
      std::unordered_map< id_type, rank_type > rank_of;
    };

    /** Reads GFA 1 or 2 text; ordering "native" or "topological". */
    inline Graph
    load( std::istream& in, std::string const& ordering = "native" )
    {
      if ( ordering != "native" && ordering != "topological" )
        throw std::runtime_error( "gfa: unknown ordering '" + ordering + "'" );
      std::vector< std::string > names;
      std::vector< uint64_t > lens;
      std::vector< std::pair< std::string, std::string > > links;
      std::unordered_map< std::string, uint64_t > index;
      std::string line;
      auto strand = []( std::string const& s, bool gfa2 ) {
        if ( gfa2 ) {
          if ( s.empty() || ( s.back() != '+' && s.back() != '-' ) ) throw std::runtime_error( "gfa: bad segment reference " + s );
          if ( s.back() == '-' ) throw std::runtime_error( "gfa: reverse-strand edges are not supported" );
          return s.substr( 0, s.size() - 1 );
        }
        return s;
      };
      while ( std::getline( in, line ) ) {
        if ( !line.empty() && line.back() == '\r' ) line.pop_back();
        std::vector< std::string > f;
        std::stringstream ss( line );
        std::string tok;
        while ( std::getline( ss, tok, '\t' ) ) f.push_back( tok );
        if ( f.empty() ) continue;
        if ( f[ 0 ] == "S" ) {
          if ( f.size() < 3 ) throw std::runtime_error( "gfa: short S line" );
          uint64_t l = 0;
          bool gfa2 = f.size() >= 4 && !f[ 2 ].empty() && std::all_of( f[ 2 ].begin(), f[ 2 ].end(), ::isdigit )
                      && f[ 3 ].find( ':' ) == std::string::npos;
          if ( gfa2 ) {
            l = std::stoull( f[ 2 ] );
          }
          else if ( f[ 2 ] != "*" ) {
            l = f[ 2 ].size();
          }
          else {
            for ( std::size_t k = 3; k < f.size(); ++k )
              if ( f[ k ].rfind( "LN:i:", 0 ) == 0 ) l = std::stoull( f[ k ].substr( 5 ) );
          }
          if ( index.count( f[ 1 ] ) ) throw std::runtime_error( "gfa: segment " + f[ 1 ] + " defined twice" );
          index[ f[ 1 ] ] = names.size();
          names.push_back( f[ 1 ] );
          lens.push_back( l );
        }
        else if ( f[ 0 ] == "L" ) {
          if ( f.size() < 5 ) throw std::runtime_error( "gfa: short L line" );
          if ( f[ 2 ] != "+" || f[ 4 ] != "+" ) throw std::runtime_error( "gfa: reverse-strand edges are not supported" );
          links.emplace_back( f[ 1 ], f[ 3 ] );
        }
        else if ( f[ 0 ] == "E" ) {
          if ( f.size() < 4 ) throw std::runtime_error( "gfa: short E line" );
          links.emplace_back( strand( f[ 2 ], true ), strand( f[ 3 ], true ) );
        }
      }
      const uint64_t n = names.size();
      bool numeric = true;
      for ( auto const& s : names )
        if ( s.empty() || !std::all_of( s.begin(), s.end(), ::isdigit ) || std::stoull( s ) == 0 ) numeric = false;
      std::vector< uint64_t > id( n );
      for ( uint64_t k = 0; k < n; ++k ) id[ k ] = numeric ? std::stoull( names[ k ] ) : k + 1;
      std::vector< std::vector< uint64_t > > succ( n );  // by file position
      for ( auto const& e : links ) {
        auto a = index.find( e.first ), b = index.find( e.second );
        if ( a == index.end() || b == index.end() ) throw std::runtime_error( "gfa: edge to an unknown segment" );
        succ[ a->second ].push_back( b->second );
      }
      // ranks: file order, or Kahn's order taking the lowest file position first
      std::vector< uint64_t > order;
      if ( ordering == "native" ) {
        for ( uint64_t k = 0; k < n; ++k ) order.push_back( k );
      }
      else {
        std::vector< uint64_t > indeg( n, 0 );
        for ( uint64_t k = 0; k < n; ++k )
          for ( uint64_t t : succ[ k ] ) ++indeg[ t ];
        std::priority_queue< uint64_t, std::vector< uint64_t >, std::greater< uint64_t > > ready;
        for ( uint64_t k = 0; k < n; ++k )
          if ( indeg[ k ] == 0 ) ready.push( k );
        std::vector< char > done( n, 0 );
        while ( !ready.empty() ) {
          const uint64_t k = ready.top();
          ready.pop();
          order.push_back( k );
          done[ k ] = 1;
          for ( uint64_t t : succ[ k ] )
            if ( --indeg[ t ] == 0 ) ready.push( t );
        }
        for ( uint64_t k = 0; k < n; ++k )
          if ( !done[ k ] ) order.push_back( k );
      }
      Graph g;
      g.ids.resize( n );
      g.len.resize( n );
      g.out.resize( n );
      for ( uint64_t r = 0; r < n; ++r ) {
        const uint64_t k = order[ r ];
        g.ids[ r ] = id[ k ];
        g.len[ r ] = lens[ k ];
        g.rank_of[ id[ k ] ] = r + 1;
        for ( uint64_t t : succ[ k ] ) g.out[ r ].push_back( id[ t ] );
      }
      return g;
    }
  }  // namespace gfa
}  // namespace diverg

#endif  // DIVERG_B200_GFA_HPP__
