#ifndef UMAPPP_NEIGHBOR_LIST_HPP
#define UMAPPP_NEIGHBOR_LIST_HPP

/**
 * @file NeighborList.hpp
 * @brief Nearest-neighbour input (drop-in for libscran/umappp
 * include/umappp/NeighborList.hpp:28-29): for each observation, its neighbours
 * as (index, distance) pairs, unique, sorted by increasing distance, no self.
 */

#include <utility>
#include <vector>

namespace umappp {

template <typename Index_, typename Float_>
using NeighborList = std::vector<std::vector<std::pair<Index_, Float_> > >;

}  // namespace umappp

#endif
