// mech.h -- mechanism tables for the sm_100a kinetics path.
//
// The product's own CHEMKIN-II loader builds the tables the kinetics kernels
// read, in Zero-RK's indexing so results line up species-for-species and
// step-for-step with zerork::mechanism:
//   species order      : SPECIES section order           (src/zerork/mechanism.cpp:117-138)
//   step order         : fwd[,rev] per reaction           (src/zerork/info_net.cpp:46-97)
//   reactant/products  : expanded integer stoichiometry   (src/zerork/info_net.cpp:176-330)
//   Arrhenius params   : unit conversion + 1e-6 merge     (src/zerork/rate_const.cpp:226-332)
//   Keq / third body / falloff lists                      (src/zerork/rate_const.cpp:334-537)
#pragma once
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace zrk {

enum FalloffKind { kLindemann = 0, kTroe3 = 1, kTroe4 = 2, kSRI = 3 };

struct MechTables {
  int nsp = 0, nrxn = 0, nstep = 0;
  std::vector<std::string> species;
  std::vector<std::string> elements;
  std::vector<double> mw;      // [nsp] kg/kmol
  std::vector<double> thermo;  // [nsp*16] Tmid, 7 low, 7 high, pad
  std::vector<int> step_rxn, step_dir;
  std::vector<int> reac_ptr, reac_spc, prod_ptr, prod_spc;
  std::vector<int> arr_step;
  std::vector<double> arr_lnA, arr_n, arr_Ta;
  std::vector<int> keq_step, keq_fwd;
  std::vector<double> keq_dn;
  std::vector<int> tb_fwd, tb_rev, tb_ptr, tb_spc;
  std::vector<double> tb_alpha;
  std::vector<int> fo_fwd, fo_rev, fo_type, fo_spc, fo_ptr, fo_eff_spc;
  std::vector<double> fo_alpha, fo_par;  // fo_par: 8 per falloff reaction
  // PLOG reactions (src/zerork/plog_reaction.cpp, rate_const.cpp:1146-1201):
  // forward step, distinct pressure points (Pa, ascending, with their logs)
  // [plog_pt_ptr[j], plog_pt_ptr[j+1]), and per point the Arrhenius lines
  // [plog_ln_ptr[q], plog_ln_ptr[q+1]) summed with the sign of their A
  std::vector<int> plog_step, plog_pt_ptr, plog_ln_ptr;
  std::vector<double> plog_p, plog_lnp, plog_lnA, plog_sgn, plog_n, plog_Ta;
  std::vector<int> rxn_reversible, rxn_third_body, rxn_falloff, rxn_plog;

  int tot_reac() const { return (int)reac_spc.size(); }
  int tot_prod() const { return (int)prod_spc.size(); }
};

// Parse CHEMKIN mechanism + thermo files. Throws zrk::ParseError.
struct ParseError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
MechTables load_chemkin(const std::string &mech_file, const std::string &therm_file);

// Fixed Jacobian sparsity over n = nsp+1 variables (species, temperature),
// compressed-column, rows ascending: reactor_nvector_serial.cpp:122-281.
// Term lists map each (step, concentration column) pair to its nonzero.
struct JacPattern {
  int n = 0, nnz = 0;
  std::vector<int> col_ptr, row_idx, last_row;
  std::vector<int> des_conc, des_step, des_nz;
  std::vector<int> cre_conc, cre_step, cre_nz;
};
JacPattern build_jac_pattern(const MechTables &t);

}  // namespace zrk
