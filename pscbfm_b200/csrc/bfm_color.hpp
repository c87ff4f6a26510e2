/*
 * bfm_color.hpp -- species colouring on the device (bfm_color.cu).
 */
#pragma once
#include <cstdint>
#include <vector>

namespace bfm {

/* The reference's colouring (graphColoring with uniform rebalancing) of a
 * bond graph, with its depth-first walk replaced on every tree component by
 * a parity union-find on the current GPU; components with a cycle are
 * walked on the host.  nbr8 holds 8 slots per node.  Returns 1 when every
 * component was coloured on the device, 2 when components with a cycle went
 * to the host walk, 0 (leaving `color` untouched) when the union-find did
 * not converge and the caller must colour on the host. */
int color_graph_device(uint32_t n, const uint8_t *deg, const uint32_t *nbr8, bool uniform, std::vector<uint32_t> &color);

} // namespace bfm
