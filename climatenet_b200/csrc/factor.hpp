// factor.hpp — one-time sparse Cholesky factorisation of the global-step
// matrix M + dt^2 A^T A and its device layout.
//
// Replaces Eigen::SimplicialLLT::compute (include/physics/SimulationSpeed.hpp:102,
// src/physics/SimulationSpeed.cpp:53).  The matrix is constant for the whole run
// (the reference never refactorises in the shipped path), so the factor is
// computed once on the host in FP64 and then re-laid out for the device
// triangular sweeps:
//
//  * ordering: nested dissection by recursive coordinate bisection of the rest
//    positions with vertex separators taken from the matrix graph;
//  * supernodes = the nested-dissection tree nodes (leaf domains and
//    separators), each a dense column block [c0, c0+ns) with row set R_s;
//  * numeric factorisation: multifrontal, supernode by supernode in postorder;
//  * partitioned inverse: per supernode W_s = [D_s^-1 ; L_Rs D_s^-1] where D_s
//    is the diagonal block.  The forward sweep is then y_s = D^-1 b_s,
//    b_R -= (L_R D^-1) b_s and the backward sweep x_s = W_s^T [y_s ; -x_R]:
//    both are plain matrix-vector products with no dependency inside a
//    supernode, so a supernode can be split across any number of warps.
//  * W_s is stored twice: row-major (forward, one warp group per row) and
//    column-major (backward, one warp group per column); each sweep reads its
//    copy exactly once with coalesced loads.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "model.hpp"

namespace pdfb {

struct Factor {
  int N = 0;
  std::vector<int> perm, iperm;  // perm[k] = vertex at pivot position k
  int n_sn = 0;
  std::vector<int> sn_c0, sn_ns, sn_nr, sn_parent, sn_level;
  std::vector<int64_t> sn_roff;  // offset into rows
  std::vector<int> rows;         // R_s, permuted indices, ascending
  std::vector<int64_t> sn_woff;  // offset of W_s (same for both copies)
  std::vector<double> Wr, Wc;    // packed W_s, row-major / column-major
  int n_levels = 0;
  int64_t nnz_w = 0;             // sum ns(ns+1)/2 + nr ns
  int64_t nnz_l_true = 0;        // structural nnz of L (diagonal included)
  double factor_ms = 0;
};

// Returns false (and sets err) if the matrix is not positive definite.
bool factorize(const Model& m, double dt, int leaf_size, Factor& f, std::string& err);

// W column offset inside a supernode: column j starts at colstart(j).
inline int64_t w_colstart(int64_t j, int64_t ns, int64_t nr) { return j * (ns + nr) - j * (j - 1) / 2; }
// W row offset: rows i < ns start at i(i+1)/2, rows ns+r at ns(ns+1)/2 + r ns.
inline int64_t w_rowstart(int64_t i, int64_t ns) {
  return i < ns ? i * (i + 1) / 2 : ns * (ns + 1) / 2 + (i - ns) * ns;
}

}  // namespace pdfb
