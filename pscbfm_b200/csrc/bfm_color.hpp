/*
 * bfm_color.hpp -- species colouring of forests on the device (bfm_color.cu).
 */
#pragma once
#include <cstdint>
#include <vector>

namespace bfm {

/* The reference's colouring (graphColoring with uniform rebalancing) of a
 * bond graph that is a forest, with its depth-first walk replaced by a
 * parity union-find on the current GPU.  nbr8 holds 8 slots per node.
 * Returns false, leaving `color` untouched, when the graph is not a forest
 * (the caller then colours on the host). */
bool color_forest_device(uint32_t n, const uint8_t *deg, const uint32_t *nbr8, bool uniform, std::vector<uint32_t> &color);

} // namespace bfm
