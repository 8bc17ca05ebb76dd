// sparse_lu.h -- symbolic analysis for the batched sparse LU of the Newton
// matrix P = I - c J over the fixed reactor Jacobian pattern.
//
// The reference factors P with SuperLU (MMD on A'A, MC64 row scaling, static
// diagonal pivots, applications/cfd_plugin/interfaces/superlu_manager
// superlu_manager.cpp:5-19, :66-155) on the CPU and with cuSolverRf on the
// GPU after a host symbolic factorization (cusolver_rf_manager.cu:109-234).
// Here the symbolic work is done once per mechanism on the host: a
// minimum-degree ordering of the symmetric structure of the species block
// with the (dense) temperature variable last, symbolic fill, and the tables a
// warp uses for left-looking numeric factorization and column-oriented
// triangular solves.  Pivots are static (diagonal of the permuted matrix).
#pragma once
#include <vector>

#include "mech.h"

namespace zrk {

struct LUSymbolic {
  int n = 0, nnz = 0;                // factor size and stored entries (L+U)
  std::vector<int> perm, iperm;      // new index -> old, old -> new
  std::vector<int> col_ptr, row_idx; // CSC of L+U in permuted order, rows ascending
  std::vector<int> diag_pos;         // storage index of (j, j)
  std::vector<int> jac_to_lu;        // Jacobian nonzero -> LU storage index
  std::vector<int> diag_of_orig;     // original variable -> LU storage index of its diagonal
  long flops = 0;                    // multiply-adds of one numeric factorization
};

LUSymbolic analyze_lu(const JacPattern &p);

}  // namespace zrk
