// Node partition of the FEM block for the persistent PCG's CTAs (host code).
//
// Each CTA of the Schur PCG owns a contiguous range of block rows.  How many of
// a CTA's blocks reach rows of other CTAs decides how much it must read from
// its neighbours every SpMV (its vector window) and, for the block-local
// preconditioner, how much of D its own diagonal block captures.  The mesh's own
// node numbering is arbitrary (the vehicle tire mesh: mean |i - j| of 1,089 over
// an edge within a 3,548-node tire), so the analysis renumbers the FEM nodes:
// the nodes are split into compact parts of balanced weight, and numbered part
// by part (by original index inside a part), so that part k is the contiguous
// row range of CTA k.
//
// The partition is graph growing on the node adjacency of D, in the spirit of
// the "bubble" methods (Diekmann, Preis, Schlimbach, Walshaw 2000): seeds spread
// by farthest-point sampling (breadth-first distance), parts grown one node at
// a time, always the lightest part taking the next node of its breadth-first
// front, then sweeps that let weight flow from heavy parts to lighter
// neighbours.  (Lloyd-style rounds that re-seed each part at its most interior
// node and grow again measured no better on the vehicle tire mesh: 16.0 % of
// the blocks cross parts either way.)  Connected components are partitioned
// separately, with parts in proportion to their weight.  Deterministic.
#pragma once
#include <vector>

namespace hsc {

// adjacency: CSR over n nodes (symmetric, no self loops); weight: per node
// (> 0).  Returns part[i] in [0, nparts) for every node.
std::vector<int> partition_nodes(int n, const std::vector<int>& adj_ptr, const std::vector<int>& adj,
                                 const std::vector<double>& weight, int nparts);

}  // namespace hsc
