// devmech.h -- mechanism tables laid out for the sm_100a kinetics kernels.
//
// One reaction record per reaction drives the rate-constant phase: each
// record carries the forward Arrhenius triple, the reverse rule (explicit
// REV triple or equilibrium constant), the third-body / falloff index and the
// reactant / product species, so one work item computes both steps of a
// reaction (rate_const.cpp:539-582 ordering: Arrhenius, Keq, third body,
// falloff; then perf_net.cpp:190-274 limiter and concentration products).
// Species-production and Jacobian phases use gather lists (per species and
// per Jacobian nonzero) so every sum is deterministic and atomic-free.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "mech.h"

namespace zrk {

constexpr int kMaxSide = 6;  // max species per reaction side (CHEMKIN limit)

enum RxnFlags : int {
  kRevKeq = 1,       // reverse step from the equilibrium constant
  kRevArr = 2,       // reverse step from explicit REV parameters
  kThirdBody = 4,
  kFalloff = 8,
  kPlog = 16,        // forward rate from the PLOG table (aux: PLOG index)
};

struct alignas(16) RxnRec {
  double lnA, n, Ta;        // forward (converted units)
  double lnA_r, n_r, Ta_r;  // explicit reverse, or dn in lnA_r for Keq
  int fwd, rev;             // step indices (rev = -1: irreversible)
  int flags, aux;           // aux: third-body or falloff list index
  int nr, np;
  short r[kMaxSide], p[kMaxSide];
};
static_assert(sizeof(RxnRec) % 16 == 0, "RxnRec alignment");

// Plain-pointer view of the device tables (all device addresses).
struct DevMech {
  int nsp, nrxn, nstep, nnz;
  int max_list;  // unused by kernels, kept for diagnostics
  const double *mw, *inv_mw, *ru_inv_mw, *thermo;  // thermo: [nsp*16]
  const RxnRec *rxn;
  const int *tb_ptr, *tb_spc;
  const double *tb_alpha;
  const int *fo_ptr, *fo_spc_eff, *fo_type, *fo_spc;
  const double *fo_alpha, *fo_par;
  // PLOG reactions: distinct pressures per reaction (plog_pt_ptr), Arrhenius
  // lines per pressure (plog_ln_ptr); see MechTables
  const int *plog_pt_ptr, *plog_ln_ptr;
  const double *plog_p, *plog_lnp, *plog_lnA, *plog_sgn, *plog_n, *plog_Ta;
  // species production gather lists (step indices in ascending step order)
  const int *sd_ptr, *sd_step, *sc_ptr, *sc_step;
  // Jacobian pattern and per-nonzero gather lists
  const int *col_ptr, *row_idx, *last_row;
  const int *nzd_ptr, *nzd_step, *nzc_ptr, *nzc_step;
  // Species-column Jacobian entries as one flat list in column-major order
  // without each column's temperature row (nj items; column j holds items
  // [jf_ptr[j], jf_ptr[j+1]), and item f is nonzero f + j of the compressed
  // columns): per item {row, n_des | n_cre << 16}, its destruction then
  // creation step indices from jt[jt_ptr[f]], and the cumulative work
  // estimate jcost[f] (3 + n_des + n_cre per item) that splits the list into
  // equal shares for the thread groups of the rates kernel.
  int nj;
  const int2 *jw;
  const unsigned short *jt;
  const int *jt_ptr, *jcost, *jf_ptr;
  // row-wise view of the Jacobian pattern: row i has entries jr_kk[p] (index
  // into the compressed-column values) in columns jr_col[p], p in
  // [jr_ptr[i], jr_ptr[i+1])
  const int *jr_ptr, *jr_kk, *jr_col;
  // work lists sorted by decreasing estimated cost, for snake-order
  // assignment to thread groups: reactions, species (production gathers),
  // species Jacobian columns
  const int *rxn_order, *spc_order, *col_order;
  // the reaction records in rxn_order order (position p holds reaction
  // rxn_order[p]): one load instead of two dependent ones per work item
  const RxnRec *rxn_by_cost;
  // The tables the rates kernel reads form the first hot_bytes bytes of the
  // allocation at base (16-byte aligned), so a CTA can stage them in shared
  // memory and address them at a fixed offset from their global copies.
  const unsigned char *base;
  int hot_bytes;
};

// Host-side builder; owns the device allocation.
class DeviceMechanism {
 public:
  DeviceMechanism(const MechTables &t, const JacPattern &p);
  ~DeviceMechanism();
  DeviceMechanism(const DeviceMechanism &) = delete;
  DeviceMechanism &operator=(const DeviceMechanism &) = delete;
  const DevMech &view() const { return view_; }
  size_t bytes() const { return bytes_; }
  // host copies of the gather lists (for tests / cost models)
  int n_terms() const { return n_terms_; }

 private:
  void *blob_ = nullptr;
  size_t bytes_ = 0;
  int n_terms_ = 0;
  DevMech view_{};
};

}  // namespace zrk
