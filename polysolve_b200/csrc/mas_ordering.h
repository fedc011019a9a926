// Subdomain ordering: which 32 block rows form each MAS bank.
//
// The reference partitions the block graph with KaMinPar into parts of at most 32 nodes
// (mas_utils/GraphPartition.cpp:176-289, MASSolver.cu:223-242) and sorts nodes by part. Here the
// ordering is a permutation of block rows into padded ids (bank * 32 + lane):
//   * "morton":  Morton (Z-order) of the block rows' positions, quantised at the mean point
//                spacing, chunked into banks of 32;
//   * "graph":   recursive bisection by BFS distance from a pseudo-peripheral node (no
//                coordinates needed), leaves of at most 32 nodes;
//   * "natural": the given order, chunked into banks of 32.
// In "morton" and "graph", block rows without off-diagonal blocks (e.g. Dirichlet identity rows)
// go to their own trailing banks: they are isolated graph nodes and would otherwise split the
// subdomains they land in.
#pragma once

#include <cstdint>
#include <vector>

namespace pmas
{
    // 1 for block rows with no off-diagonal block.
    std::vector<uint8_t> isolated_blocks(int n, const int *outer, const int *inner, int bd);

    // padded[V] and the bank count.
    std::vector<int> morton_padded(const double *xyz, int V, const std::vector<uint8_t> &isolated, int *banks);
    std::vector<int> graph_padded(int n, const int *outer, const int *inner, int bd,
                                  const std::vector<uint8_t> &isolated, int *banks);
    std::vector<int> natural_padded(int V, int *banks);

    // 64-bit FNV-1a style hash of a CSC pattern (n, outer, inner), OpenMP-parallel. The same pass
    // checks the pattern: *valid (if given) is false unless outer runs from 0 to nnz without
    // decreasing and every row index lies in [0, n). Row order inside a column is free.
    // threads: OpenMP threads of the pass (0: all).
    uint64_t pattern_hash(int n, const int *outer, const int *inner, long long nnz, bool *valid = nullptr,
                          int threads = 0);
} // namespace pmas
