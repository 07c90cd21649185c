// Reads a GFA file with include/diverg/gfa.hpp and prints the graph as the
// adjacency builder walks it: one line "n <nodes>", then "v <rank> <id> <len>"
// per node and "e <from rank> <to rank>" per edge, in rank order.
#include <fstream>
#include <iostream>

#include "diverg/gfa.hpp"

int main( int argc, char** argv )
{
  if ( argc < 3 ) return 2;
  std::ifstream in( argv[ 1 ] );
  try {
    const diverg::gfa::Graph g = diverg::gfa::load( in, argv[ 2 ] );
    std::cout << "n " << g.get_node_count() << "\n";
    g.for_each_node( [&]( uint64_t rank, uint64_t id ) {
      std::cout << "v " << rank << " " << id << " " << g.node_length( id ) << "\n";
      g.for_each_edges_out( id, [&]( uint64_t to, uint8_t ) {
        std::cout << "e " << rank << " " << g.id_to_rank( to ) << "\n";
        return true;
      } );
      return true;
    } );
  } catch ( std::exception const& e ) {
    std::cout << "error " << e.what() << "\n";
    return 1;
  }
  return 0;
}
