/**
 *  @file  diverg/adjacency.hpp
 *  @brief util::range_adjacency_matrix with the reference's template signature.
 *
 *  The reference's include/diverg/adjacency.hpp:249-265: the range-CRS
 *  adjacency matrix of the nodes of ranks [lower, upper) of a sequence graph
 *  (upper = 0: through the last node), built here on the B200 through
 *  dvg_adjacency_from_graph (include/dvg.h).  The graph type is any class with
 *  the part of gum's SeqGraph interface the reference's adjacency_matrix
 *  walks (adjacency.hpp:170-228): the id_type / rank_type / linktype_type
 *  typedefs, get_node_count(), rank_to_id(rank), id_to_rank(id),
 *  node_length(id), for_each_node(f(rank, id) -> bool, from_rank) and
 *  for_each_edges_out(id, f(to_id, linktype) -> bool).  A gum graph works as
 *  is.  The walk collects node lengths in rank order and the edges out of
 *  the range's nodes on the host; the matrix is built and converted to
 *  ranges on the device and returned by value.  Errors throw
 *  std::runtime_error (an edge leaving [lower, upper) included, where the
 *  reference's result is undefined).
 */
#ifndef DIVERG_B200_ADJACENCY_HPP__
#define DIVERG_B200_ADJACENCY_HPP__

#include <cstdint>
#include <vector>

#include "range_sparse.hpp"

namespace diverg {
  namespace util {
    template< typename TRangeCRSMatrix, class TGraph >
    inline TRangeCRSMatrix
    range_adjacency_matrix( TGraph const& graph, typename TGraph::rank_type lower = 1,
                            typename TGraph::rank_type upper = 0 )
    {
      static_assert( crs_matrix::is_range_crs_matrix< TRangeCRSMatrix >::value,
                     "output matrix should be in Range CRS format." );
      typedef typename TGraph::rank_type rank_type;
      typedef typename TGraph::id_type id_type;
      typedef typename TGraph::linktype_type linktype_type;

      const rank_type nnodes = graph.get_node_count();
      if ( upper == 0 ) upper = nnodes + 1;
      std::vector< uint32_t > node_len( nnodes );
      std::vector< uint32_t > edges;
      graph.for_each_node(
          [&]( rank_type rank, id_type id ) {
            node_len[ rank - 1 ] = static_cast< uint32_t >( graph.node_length( id ) );
            if ( rank >= lower && rank < upper ) {
              graph.for_each_edges_out( id, [&]( id_type to, linktype_type ) {
                edges.push_back( static_cast< uint32_t >( rank ) );
                edges.push_back( static_cast< uint32_t >( graph.id_to_rank( to ) ) );
                return true;
              } );
            }
            return true;
          },
          1 );
      detail::DeviceMatrix d;
      detail::check( dvg_adjacency_from_graph( detail::context(), static_cast< uint32_t >( nnodes ),
                                               node_len.data(), edges.size() / 2, edges.data(),
                                               static_cast< uint32_t >( lower ),
                                               static_cast< uint32_t >( upper ), d.out() ) );
      return detail::download< TRangeCRSMatrix >( d );
    }
  }  // namespace util
}  // namespace diverg

#endif  // DIVERG_B200_ADJACENCY_HPP__
