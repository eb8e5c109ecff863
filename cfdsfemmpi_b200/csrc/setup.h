// Host-side set-up of the nodal-block matrix structure (no CUDA).
//
// Builds, deterministically from the mesh alone:
//   * the node graph (nodes sharing an element), sorted per node: the block
//     sparsity of the BSR matrix.  With Dirichlet rows/columns deleted, its
//     scalar expansion equals the free-dof pattern the reference inserts into
//     PETSc (src/base/StabFEM2.cpp:192-227);
//   * the element -> block slot map: for element e and local nodes (i, j) the
//     index of block (conn[e][i], conn[e][j]); the first writer of every block
//     in colour order is marked by storing -slot-1;
//   * a greedy element colouring (elements that share a node differ), visited
//     in element-id order;
//   * the free-dof numbering of the reference (node-major, skipping
//     prescribed (node, dof) pairs, StabFEM2.cpp:57-81) and the Dirichlet sets.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace cfdgpu {

struct Topology {
  int nNode = 0, nElem = 0, npe = 0, ndof = 0;
  std::vector<int32_t> rowptr;       // nNode+1
  std::vector<int32_t> colidx;       // nnzb
  std::vector<int32_t> slot;         // nElem*npe*npe
  std::vector<int32_t> color;        // nElem
  std::vector<int32_t> color_ptr;    // ncolors+1
  std::vector<int32_t> color_elems;  // nElem, grouped by colour, ascending id inside a colour
  int ncolors = 0;
  std::vector<int32_t> dofmap;       // nNode*ndof -> free index or -1
  int nfree = 0;
  std::vector<int32_t> fixed_dofs;   // sorted distinct prescribed dofs
  // Dirichlet list in input order (node*ndof+dof, value)
  std::vector<int32_t> dbc_index;
  std::vector<double> dbc_value;
  // per distinct prescribed dof: how many list entries name it (the reference
  // adds solnApplied once per entry, StabFEM2.cpp:719-730)
  std::vector<int32_t> dbc_mult;
  std::vector<uint8_t> fixmask;      // per node: bit d set when dof d is prescribed
  int64_t nnzb() const { return (int64_t)colidx.size(); }
};

// Block ILU(k) structure of a block-Jacobi preconditioner on the BSR pattern
// (PETSc PCBJACOBI with sub-PC ILU(levels), input/petsc_options_gmres.dat:2-5):
// nodes are cut into nblocks contiguous ranges (nNode/nblocks nodes each, the
// first nNode%nblocks ranges one longer), couplings between ranges are
// dropped, and each range gets the level-of-fill pattern of ILU(levels) in
// natural node order, lev(i,j) = min over pivots p of lev(i,p) + lev(p,j) + 1
// with the blocks of A at level 0.  A node whose dofs are all prescribed has
// an identity row and column in the BSR matrix and no row in the
// reference's free-dof system: it keeps only its diagonal block and takes no
// part in any other row, so the block factors equal the scalar ILU(levels)
// of the free-dof matrix in exact arithmetic.  levels = -1 keeps all fill:
// the complete LU of each range (one range: -pc_type lu).
struct IluPattern {
  int levels = 0, nblocks = 1;
  std::vector<int32_t> rowptr;   // nNode+1
  std::vector<int32_t> colidx;   // sorted per row
  std::vector<int32_t> diag;     // position of the diagonal block of each row
  std::vector<int32_t> aslot;    // per block of A: its position in the factors, or -1
  std::vector<int32_t> blk;      // nblocks+1 node offsets
  // factor row i is node perm[i] (empty: the identity).  ILU(k) keeps the
  // natural order, as PETSc's ILU does; the complete factorisation of one
  // block (-pc_type lu) uses a reverse Cuthill-McKee order of the node graph,
  // which bounds its fill by the graph's bandwidth (a direct solve's result
  // does not depend on the order beyond rounding)
  std::vector<int32_t> perm, iperm;
  // update map of the numeric factorisation: for a strictly lower block q =
  // (i, p), umap[uoff[q] + k] is the position in row i of the k-th block
  // right of the diagonal in row p, or -1 when row i's pattern drops it
  std::vector<int64_t> uoff;     // nnzb (meaningful for strictly lower blocks)
  std::vector<int32_t> umap;
  // rows sorted by level of the lower DAG (factorisation and lower solve:
  // level(i) = 1 + max level of the strictly lower blocks' columns) and of
  // the upper DAG (upper solve), row order inside a level
  std::vector<int32_t> lorder, uorder;
  int nlev_l = 0, nlev_u = 0;
  int maxw_l = 0, maxw_u = 0;    // rows in the widest level of each DAG
  // chains of the triangular solves: maximal runs of consecutive rows in
  // which each row depends on its neighbour (row i on i-1 in the lower solve,
  // on i+1 in the upper solve), at most ILU_CHAIN_MAX rows.  A chain is solved
  // in order by one warp, so the dependency along it never goes through
  // memory.  lchain/uchain: nchains x {first row, one past the last row};
  // lchain_order/uchain_order: chain ids sorted by the level of the chain
  // DAG (a chain's inputs lie in chains of lower levels).
  std::vector<int32_t> lchain, uchain, lchain_order, uchain_order;
  int lchain_levels = 0, uchain_levels = 0, lchain_maxw = 0, uchain_maxw = 0;
  int64_t nnzb() const { return (int64_t)colidx.size(); }
};

constexpr int ILU_CHAIN_MAX = 128;

std::string build_ilu_pattern(const Topology &t, int levels, int nblocks, IluPattern &f);

// Returns "" on success, else an error message.
std::string build_topology(int nNode, int nElem, int npe, int ndof, const int32_t *conn, int nDBC,
                           const int32_t *dbc_node, const int32_t *dbc_dof, const double *dbc_value,
                           Topology &t);

}  // namespace cfdgpu
