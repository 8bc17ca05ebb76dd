// devmech.cpp -- pack MechTables + JacPattern into one device allocation.
#include "devmech.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

namespace zrk {
namespace {

const double kRu = 8.314462618e3;

struct Blob {
  std::vector<unsigned char> bytes;
  template <class T>
  size_t add(const std::vector<T> &v, size_t align = 256) {
    size_t off = (bytes.size() + align - 1) & ~(align - 1);
    bytes.resize(off + std::max<size_t>(v.size() * sizeof(T), 16), 0);
    if (!v.empty()) std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
    return off;
  }
};

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

DeviceMechanism::DeviceMechanism(const MechTables &t, const JacPattern &p) {
  const int ns = t.nsp;
  std::vector<double> inv_mw(ns), ru_inv_mw(ns);
  for (int j = 0; j < ns; ++j) {
    inv_mw[j] = 1.0 / t.mw[j];          // mechanism.cpp:135 invMolWt
    ru_inv_mw[j] = kRu / t.mw[j];       // mechanism.cpp:136 RuInvMolWt
  }
  // reaction records
  std::vector<RxnRec> rec(t.nrxn);
  std::vector<int> arr_of_step(t.nstep, -1);
  for (size_t k = 0; k < t.arr_step.size(); ++k) arr_of_step[t.arr_step[k]] = (int)k;
  std::vector<int> plog_of_step(t.nstep, -1);
  for (size_t k = 0; k < t.plog_step.size(); ++k) plog_of_step[t.plog_step[k]] = (int)k;
  std::vector<int> step_of_fwd(t.nrxn, -1), step_of_rev(t.nrxn, -1);
  for (int s = 0; s < t.nstep; ++s) {
    if (t.step_dir[s] == 1) step_of_fwd[t.step_rxn[s]] = s;
    else step_of_rev[t.step_rxn[s]] = s;
  }
  for (int j = 0; j < t.nrxn; ++j) {
    RxnRec &R = rec[j];
    std::memset(&R, 0, sizeof(R));
    R.fwd = step_of_fwd[j];
    R.rev = step_of_rev[j];
    R.aux = -1;
    int a = arr_of_step[R.fwd];
    if (a >= 0) {
      R.lnA = t.arr_lnA[a];
      R.n = t.arr_n[a];
      R.Ta = t.arr_Ta[a];
    } else if (plog_of_step[R.fwd] >= 0) {
      R.flags |= kPlog;
      R.aux = plog_of_step[R.fwd];
    } else {
      throw std::runtime_error("forward step without Arrhenius or PLOG parameters");
    }
    if (R.rev >= 0) {
      int b = arr_of_step[R.rev];
      if (b >= 0) {
        R.flags |= kRevArr;
        R.lnA_r = t.arr_lnA[b];
        R.n_r = t.arr_n[b];
        R.Ta_r = t.arr_Ta[b];
      } else {
        R.flags |= kRevKeq;
      }
    }
    R.nr = t.reac_ptr[R.fwd + 1] - t.reac_ptr[R.fwd];
    R.np = t.prod_ptr[R.fwd + 1] - t.prod_ptr[R.fwd];
    if (R.nr > kMaxSide || R.np > kMaxSide)
      throw std::runtime_error("reaction " + std::to_string(j) + " has more than 6 species on a side");
    for (int k = 0; k < R.nr; ++k) R.r[k] = (short)t.reac_spc[t.reac_ptr[R.fwd] + k];
    for (int k = 0; k < R.np; ++k) R.p[k] = (short)t.prod_spc[t.prod_ptr[R.fwd] + k];
  }
  for (size_t k = 0; k < t.keq_step.size(); ++k) {
    int j = t.step_rxn[t.keq_fwd[k]];
    rec[j].lnA_r = t.keq_dn[k];  // dn stored in the reverse slot
  }
  for (size_t k = 0; k < t.tb_fwd.size(); ++k) {
    int j = t.step_rxn[t.tb_fwd[k]];
    rec[j].flags |= kThirdBody;
    rec[j].aux = (int)k;
  }
  for (size_t k = 0; k < t.fo_fwd.size(); ++k) {
    int j = t.step_rxn[t.fo_fwd[k]];
    rec[j].flags |= kFalloff;
    rec[j].aux = (int)k;
  }
  // species gather lists, ascending step order (perf_net.cpp:257-267 sum order)
  std::vector<std::vector<int>> sd(ns), sc(ns);
  for (int s = 0; s < t.nstep; ++s) {
    for (int k = t.reac_ptr[s]; k < t.reac_ptr[s + 1]; ++k) sd[t.reac_spc[k]].push_back(s);
    for (int k = t.prod_ptr[s]; k < t.prod_ptr[s + 1]; ++k) sc[t.prod_spc[k]].push_back(s);
  }
  std::vector<int> sd_ptr(1, 0), sd_step, sc_ptr(1, 0), sc_step;
  for (int j = 0; j < ns; ++j) {
    sd_step.insert(sd_step.end(), sd[j].begin(), sd[j].end());
    sd_ptr.push_back((int)sd_step.size());
    sc_step.insert(sc_step.end(), sc[j].begin(), sc[j].end());
    sc_ptr.push_back((int)sc_step.size());
  }
  // Jacobian per-nonzero gather lists, in term-list order
  // (reactor_nvector_serial.cpp:659-673: all destruction terms, then creation)
  std::vector<std::vector<int>> nzd(p.nnz), nzc(p.nnz);
  for (size_t q = 0; q < p.des_nz.size(); ++q) nzd[p.des_nz[q]].push_back(p.des_step[q]);
  for (size_t q = 0; q < p.cre_nz.size(); ++q) nzc[p.cre_nz[q]].push_back(p.cre_step[q]);
  std::vector<int> nzd_ptr(1, 0), nzd_step, nzc_ptr(1, 0), nzc_step;
  for (int k = 0; k < p.nnz; ++k) {
    nzd_step.insert(nzd_step.end(), nzd[k].begin(), nzd[k].end());
    nzd_ptr.push_back((int)nzd_step.size());
    nzc_step.insert(nzc_step.end(), nzc[k].begin(), nzc[k].end());
    nzc_ptr.push_back((int)nzc_step.size());
  }
  n_terms_ = (int)(nzd_step.size() + nzc_step.size());
  // flat species-column list for the rates kernel's Jacobian phase
  std::vector<int2> jw;
  std::vector<unsigned short> jt;
  std::vector<int> jt_ptr(1, 0), jcost(1, 0), jf_ptr(1, 0);
  for (int j = 0; j < ns; ++j) {
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1] - 1; ++k) {  // the last entry is the T row
      const int nd = nzd_ptr[k + 1] - nzd_ptr[k], nc = nzc_ptr[k + 1] - nzc_ptr[k];
      if (nd > 0xffff || nc > 0xffff || t.nstep > 0xffff)
        throw std::runtime_error("mechanism too large for 16-bit Jacobian term lists");
      jw.push_back(make_int2(p.row_idx[k], nd | (nc << 16)));
      for (int q = nzd_ptr[k]; q < nzd_ptr[k + 1]; ++q) jt.push_back((unsigned short)nzd_step[q]);
      for (int q = nzc_ptr[k]; q < nzc_ptr[k + 1]; ++q) jt.push_back((unsigned short)nzc_step[q]);
      jt_ptr.push_back((int)jt.size());
      jcost.push_back(jcost.back() + 3 + nd + nc);
    }
    jf_ptr.push_back((int)jw.size());
  }
  std::vector<std::vector<std::pair<int, int>>> rows(p.n);
  for (int j = 0; j < p.n; ++j)
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) rows[p.row_idx[k]].push_back({k, j});
  std::vector<int> jr_ptr(1, 0), jr_kk, jr_col;
  for (int i = 0; i < p.n; ++i) {
    for (auto &e : rows[i]) {
      jr_kk.push_back(e.first);
      jr_col.push_back(e.second);
    }
    jr_ptr.push_back((int)jr_kk.size());
  }

  // cost-sorted work lists (stable: ties keep index order)
  auto sorted_by = [](std::vector<double> cost) {
    std::vector<int> idx(cost.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    return idx;
  };
  std::vector<double> rc(t.nrxn), sc2(ns), cc(ns);
  for (int j = 0; j < t.nrxn; ++j) {
    const RxnRec &R = rec[j];
    double c = 1.0 + 0.1 * (R.nr + R.np);
    if (R.flags & (kRevKeq | kRevArr)) c += 1.0;
    if (R.flags & kThirdBody) c += 0.5 + 0.1 * (t.tb_ptr[R.aux + 1] - t.tb_ptr[R.aux]);
    if (R.flags & kFalloff) c += 3.0 + 0.1 * (t.fo_ptr[R.aux + 1] - t.fo_ptr[R.aux]);
    if (R.flags & kPlog) {
      const int q0 = t.plog_pt_ptr[R.aux], q1 = t.plog_pt_ptr[R.aux + 1];
      c += 2.0 + 0.5 * (t.plog_ln_ptr[q1] - t.plog_ln_ptr[q0]);
    }
    rc[j] = c;
  }
  for (int k = 0; k < ns; ++k) {
    sc2[k] = (sd_ptr[k + 1] - sd_ptr[k]) + (sc_ptr[k + 1] - sc_ptr[k]);
    double w = 0.0;
    for (int kk = p.col_ptr[k]; kk < p.col_ptr[k + 1]; ++kk)
      w += 1.0 + (nzd_ptr[kk + 1] - nzd_ptr[kk]) + (nzc_ptr[kk + 1] - nzc_ptr[kk]);
    cc[k] = w;
  }
  const std::vector<int> rxn_order = sorted_by(rc), spc_order = sorted_by(sc2), col_order = sorted_by(cc);

  // The tables of the rates kernel first, 16-byte aligned and contiguous:
  // the kernel may stage [blob, blob + hot_bytes) in shared memory.
  std::vector<RxnRec> rec_by_cost;
  for (int p : rxn_order) rec_by_cost.push_back(rec[p]);
  Blob b;
  const size_t h = 16;
  size_t o_rbc = b.add(rec_by_cost, h);
  size_t o_mw = b.add(t.mw, h), o_imw = b.add(inv_mw, h), o_rimw = b.add(ru_inv_mw, h),
         o_th = b.add(t.thermo, h);
  size_t o_tbp = b.add(t.tb_ptr, h), o_tbs = b.add(t.tb_spc, h), o_tba = b.add(t.tb_alpha, h);
  size_t o_fop = b.add(t.fo_ptr, h), o_foe = b.add(t.fo_eff_spc, h), o_fot = b.add(t.fo_type, h),
         o_fos = b.add(t.fo_spc, h), o_foa = b.add(t.fo_alpha, h), o_fopar = b.add(t.fo_par, h);
  size_t o_plpp = b.add(t.plog_pt_ptr, h), o_pllp = b.add(t.plog_ln_ptr, h), o_plp = b.add(t.plog_p, h),
         o_pllnp = b.add(t.plog_lnp, h), o_pla = b.add(t.plog_lnA, h), o_pls = b.add(t.plog_sgn, h),
         o_pln = b.add(t.plog_n, h), o_plt = b.add(t.plog_Ta, h);
  size_t o_sdp = b.add(sd_ptr, h), o_sds = b.add(sd_step, h), o_scp = b.add(sc_ptr, h),
         o_scs = b.add(sc_step, h);
  size_t o_so = b.add(spc_order, h);
  size_t o_cp = b.add(p.col_ptr, h), o_ri = b.add(p.row_idx, h);
  size_t o_jw = b.add(jw, h), o_jt = b.add(jt, h), o_jtp = b.add(jt_ptr, h), o_jc = b.add(jcost, h),
         o_jf = b.add(jf_ptr, h);
  const size_t hot = (b.bytes.size() + 15) & ~size_t(15);
  size_t o_rec = b.add(rec);
  size_t o_lr = b.add(p.last_row);
  size_t o_ndp = b.add(nzd_ptr), o_nds = b.add(nzd_step), o_ncp = b.add(nzc_ptr), o_ncs = b.add(nzc_step);
  size_t o_jrp = b.add(jr_ptr), o_jrk = b.add(jr_kk), o_jrc = b.add(jr_col);
  size_t o_ro = b.add(rxn_order), o_co = b.add(col_order);
  bytes_ = b.bytes.size();
  check(cudaMalloc(&blob_, bytes_), "cudaMalloc(mechanism tables)");
  check(cudaMemcpy(blob_, b.bytes.data(), bytes_, cudaMemcpyHostToDevice), "cudaMemcpy(mechanism tables)");
  auto P = [&](size_t off) { return (const void *)((const unsigned char *)blob_ + off); };
  view_.base = (const unsigned char *)blob_;
  view_.hot_bytes = (int)hot;
  view_.nsp = ns;
  view_.nrxn = t.nrxn;
  view_.nstep = t.nstep;
  view_.nnz = p.nnz;
  view_.mw = (const double *)P(o_mw);
  view_.inv_mw = (const double *)P(o_imw);
  view_.ru_inv_mw = (const double *)P(o_rimw);
  view_.thermo = (const double *)P(o_th);
  view_.rxn = (const RxnRec *)P(o_rec);
  view_.tb_ptr = (const int *)P(o_tbp);
  view_.tb_spc = (const int *)P(o_tbs);
  view_.tb_alpha = (const double *)P(o_tba);
  view_.fo_ptr = (const int *)P(o_fop);
  view_.fo_spc_eff = (const int *)P(o_foe);
  view_.fo_type = (const int *)P(o_fot);
  view_.fo_spc = (const int *)P(o_fos);
  view_.fo_alpha = (const double *)P(o_foa);
  view_.fo_par = (const double *)P(o_fopar);
  view_.plog_pt_ptr = (const int *)P(o_plpp);
  view_.plog_ln_ptr = (const int *)P(o_pllp);
  view_.plog_p = (const double *)P(o_plp);
  view_.plog_lnp = (const double *)P(o_pllnp);
  view_.plog_lnA = (const double *)P(o_pla);
  view_.plog_sgn = (const double *)P(o_pls);
  view_.plog_n = (const double *)P(o_pln);
  view_.plog_Ta = (const double *)P(o_plt);
  view_.sd_ptr = (const int *)P(o_sdp);
  view_.sd_step = (const int *)P(o_sds);
  view_.sc_ptr = (const int *)P(o_scp);
  view_.sc_step = (const int *)P(o_scs);
  view_.col_ptr = (const int *)P(o_cp);
  view_.row_idx = (const int *)P(o_ri);
  view_.last_row = (const int *)P(o_lr);
  view_.nzd_ptr = (const int *)P(o_ndp);
  view_.nzd_step = (const int *)P(o_nds);
  view_.nzc_ptr = (const int *)P(o_ncp);
  view_.nzc_step = (const int *)P(o_ncs);
  view_.nj = (int)jw.size();
  view_.jw = (const int2 *)P(o_jw);
  view_.jt = (const unsigned short *)P(o_jt);
  view_.jt_ptr = (const int *)P(o_jtp);
  view_.jcost = (const int *)P(o_jc);
  view_.jf_ptr = (const int *)P(o_jf);
  view_.jr_ptr = (const int *)P(o_jrp);
  view_.jr_kk = (const int *)P(o_jrk);
  view_.jr_col = (const int *)P(o_jrc);
  view_.rxn_order = (const int *)P(o_ro);
  view_.spc_order = (const int *)P(o_so);
  view_.col_order = (const int *)P(o_co);
  view_.rxn_by_cost = (const RxnRec *)P(o_rbc);
}

DeviceMechanism::~DeviceMechanism() {
  if (blob_) cudaFree(blob_);
}

}  // namespace zrk
