/*
 * nwgraph_gen.h -- seeded synthetic graph builder (host C ABI).
 *
 * Not part of the drop-in boundary: the reference has no RMAT generator
 * (its GAP generator submodule, bench/gapbs-reference, is not vendored), so
 * this builds the CSR that the reference's CPU page_rank and the GPU engine
 * both consume. The CSR layout is NWGraph's adjacency<1>
 * (include/nwgraph/adjacency.hpp:86-195): row_ptr = indices_ (n+1 uint32),
 * col = std::get<0>(to_be_indexed_) (nnz uint32), row i = in-neighbours of i.
 * All generated graphs are symmetric simple graphs with rows sorted ascending.
 */
#ifndef NWGRAPH_GEN_H
#define NWGRAPH_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nwgen_csr {
  uint64_t  n;
  uint64_t  nnz;
  uint32_t* row_ptr; /* n+1, malloc'd */
  uint32_t* col;     /* nnz, malloc'd */
} nwgen_csr;

/* RMAT with 2^scale vertices and round(edge_factor * 2^scale) samples,
 * quadrant probabilities a, b, c (d = 1-a-b-c), symmetrised and deduplicated.
 * nthreads <= 0 uses every hardware thread; the result does not depend on it.
 * Returns 0, -1 bad arguments, -2 out of memory, -3 nnz overflows uint32. */
int nwgen_rmat(int scale, double edge_factor, double a, double b, double c, uint64_t seed, int nthreads,
               nwgen_csr* out);

/* floor(sqrt(n_target))^2-vertex 4-neighbour grid. */
int nwgen_grid(uint64_t n_target, nwgen_csr* out);

/* CSR (adjacency<1>: row = destination) from a directed edge list; with
 * symmetrize != 0 self-loops are dropped and reverse edges added. Rows are
 * sorted and duplicates dropped either way. */
int nwgen_from_edges(const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n, int symmetrize, int nthreads,
                     nwgen_csr* out);

void nwgen_free(nwgen_csr* g);

#ifdef __cplusplus
}
#endif
#endif
