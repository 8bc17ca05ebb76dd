/*
 * zerork_b200_mechanism.h -- C++ mirror of zerork::mechanism and
 * zerork::mechanism_cuda (src/zerork/mechanism.h:20-285,
 * src/zerork/mechanism_cuda.h:9-45) over the C ABI of zerork_b200.h, so code
 * written against the reference's classes relinks with the same method
 * names, argument order and array conventions.
 *
 * Rates run on the GPU (one state per call for the host methods, n states for
 * the _mr_dev methods); the small thermodynamic helpers (concentrations,
 * internal energy, heat capacity) are host arithmetic on the loaded tables,
 * as in the reference.  Errors throw std::runtime_error carrying
 * zrk_last_error() (the reference aborts instead).  A mechanism is not
 * thread-safe, like the reference's, which keeps mutable workspaces.
 */
#ifndef ZERORK_B200_MECHANISM_H
#define ZERORK_B200_MECHANISM_H

#ifdef __cplusplus
#include <stdexcept>
#include <string>
#include <vector>

#include "zerork_b200.h"

namespace zerork_b200 {

class mechanism {
 public:
  /* mechanism(mechFileName, thermFileName, convertFileName, verbosity)
   * (mechanism.h:23-27): parses and uploads the tables to the current
   * device.  convertFileName (the reference's parser log) and verbosity
   * are accepted and ignored. */
  mechanism(const char *mechFileName, const char *thermFileName,
            const char *convertFileName = nullptr, int verbosity = 0) {
    (void)convertFileName;
    (void)verbosity;
    check(zrk_mech_create(mechFileName, thermFileName, &m_));
    int ns = 0, nr = 0, nst = 0, nnz = 0;
    check(zrk_mech_sizes(m_, &ns, &nr, &nst, &nnz));
    nsp_ = ns;
    nrxn_ = nr;
    nstep_ = nst;
    mw_ = table("mw");
    thermo_ = table("thermo");
    for (int j = 0; j < nsp_; ++j) inv_mw_.push_back(1.0 / mw_[j]);
    for (int j = 0; j < nsp_; ++j) ru_inv_mw_.push_back(kRu * inv_mw_[j]);
  }
  virtual ~mechanism() {
    if (m_) zrk_mech_free(m_);
  }
  mechanism(const mechanism &) = delete;
  mechanism &operator=(const mechanism &) = delete;

  int getNumSpecies() const { return nsp_; }
  int getNumReactions() const { return nrxn_; }
  int getNumSteps() const { return nstep_; }
  const char *getSpeciesName(int idx) const { return zrk_mech_species_name(m_, idx); }
  double getGasConstant() const { return kRu; }
  void getMolWtSpc(double mwOut[]) const {
    for (int j = 0; j < nsp_; ++j) mwOut[j] = mw_[j];
  }

  /* c[j] = (1/v) W_j^-1 y[j] (mechanism.cpp:323-329) */
  void getCfromVY(const double v, const double y[], double c[]) const {
    const double dens = 1.0 / v;
    for (int j = 0; j < nsp_; ++j) c[j] = dens * inv_mw_[j] * y[j];
  }
  /* 1 / sum(y_j / W_j) */
  double getMolWtMixFromY(const double y[]) const {
    double s = 0.0;
    for (int j = 0; j < nsp_; ++j) s += y[j] * inv_mw_[j];
    return 1.0 / s;
  }
  double getDensityFromTPY(const double T, const double P, const double y[]) const {
    return P * getMolWtMixFromY(y) / (kRu * T);
  }
  /* NASA-7 h/RT - 1 (mechanism.cpp:381-386, nasa_poly.cpp:78-117) */
  void getIntEnergy_RT(const double T, double u_RT[]) const {
    const double invT = 1.0 / T;
    double m0 = T, m1 = T * m0, m2 = T * m1, m3 = T * m2;
    m0 *= 0.50000000000000000000;
    m1 *= 0.33333333333333333333;
    m2 *= 0.25000000000000000000;
    m3 *= 0.20000000000000000000;
    for (int j = 0; j < nsp_; ++j) {
      const double *c = &thermo_[16 * j];
      const int o = (T < c[0]) ? 1 : 8;
      u_RT[j] = c[o] + c[o + 1] * m0 + c[o + 2] * m1 + c[o + 3] * m2 + c[o + 4] * m3 +
                c[o + 5] * invT - 1.0;
    }
  }
  /* mass c_v of the mixture, species c_v in cvSpc (mechanism.cpp:428-441) */
  double getMassCvFromTY(const double T, const double y[], double cvSpc[]) const {
    double cv = 0.0;
    for (int j = 0; j < nsp_; ++j) {
      const double *c = &thermo_[16 * j];
      const int o = (T < c[0]) ? 1 : 8;
      cvSpc[j] = c[o] + T * (c[o + 1] + T * (c[o + 2] + T * (c[o + 3] + T * c[o + 4])));
      cvSpc[j] -= 1.0;
      cvSpc[j] *= ru_inv_mw_[j];
      cv += cvSpc[j] * y[j];
    }
    return cv;
  }
  double getMassCvFromTY(const double T, const double y[]) const {
    std::vector<double> cv(nsp_);
    return getMassCvFromTY(T, y, cv.data());
  }

  /* getReactionRates (mechanism.h:114, perf_net.cpp:126-188): one state,
   * no limiter */
  void getReactionRates(const double T, const double C[], double netOut[], double createOut[],
                        double destroyOut[], double stepOut[]) {
    check(zrk_rates_tc_host(m_, 1, &T, C, nullptr, netOut, createOut, destroyOut, stepOut));
  }
  /* getNetReactionRates (mechanism.h:124) */
  void getNetReactionRates(const double T, const double C[], double netOut[]) {
    check(zrk_rates_tc_host(m_, 1, &T, C, nullptr, netOut, nullptr, nullptr, nullptr));
  }
  /* getReactionRatesLimiter (mechanism.h:143, perf_net.cpp:190-274) */
  void getReactionRatesLimiter(const double T, const double C[], const double step_limiter[],
                               double netOut[], double createOut[], double destroyOut[],
                               double stepOut[]) {
    check(zrk_rates_tc_host(m_, 1, &T, C, step_limiter, netOut, createOut, destroyOut, stepOut));
  }

  zrk_mech_t handle() const { return m_; }

 protected:
  static constexpr double kRu = 8.314462618e3;  // src/zerork/constants.h:10
  static void check(int rc) {
    if (rc != ZRK_OK) throw std::runtime_error(std::string("zerork_b200: ") + zrk_last_error());
  }
  std::vector<double> table(const char *name) const {
    long count = 0;
    int is_double = 0;
    check(zrk_mech_table(m_, name, nullptr, 0, &count, &is_double));
    std::vector<double> v(count);
    check(zrk_mech_table(m_, name, v.data(), count, &count, &is_double));
    return v;
  }
  zrk_mech_t m_ = nullptr;
  int nsp_ = 0, nrxn_ = 0, nstep_ = 0;
  std::vector<double> mw_, inv_mw_, ru_inv_mw_, thermo_;
};

/* mechanism_cuda (mechanism_cuda.h:9-45): the multi-reactor device entry
 * points, arrays species-major with nReactors as leading dimension
 * (C_dev[j * nReactors + k]), on the default stream. */
class mechanism_cuda : public mechanism {
 public:
  mechanism_cuda(const char *mechFileName, const char *thermFileName,
                 const char *convertFileName, int verbosity, int nReactorsMax)
      : mechanism(mechFileName, thermFileName, convertFileName, verbosity),
        n_max_(nReactorsMax) {}
  void getReactionRates_CUDA_mr_dev(const int nReactors, const double T_dev[], const double C_dev[],
                                    double netOut_dev[], double createOut_dev[],
                                    double destroyOut_dev[], double stepOut_dev[]) {
    check_n(nReactors);
    check(zrk_rates_tc_dev(m_, nReactors, nReactors, T_dev, C_dev, nullptr, netOut_dev,
                           createOut_dev, destroyOut_dev, stepOut_dev, nullptr));
  }
  void getReactionRatesLimiter_CUDA_mr_dev(const int nReactors, const double T_dev[],
                                           const double C_dev[], const double stepLimiter_dev[],
                                           double netOut_dev[], double createOut_dev[],
                                           double destroyOut_dev[], double stepOut_dev[]) {
    check_n(nReactors);
    check(zrk_rates_tc_dev(m_, nReactors, nReactors, T_dev, C_dev, stepLimiter_dev, netOut_dev,
                           createOut_dev, destroyOut_dev, stepOut_dev, nullptr));
  }
  int nReactorsMax() { return n_max_; }

 private:
  /* the reference asserts nReactors <= nReactorsMax (mechanism_cuda.cu:154) */
  void check_n(int n) const {
    if (n < 0 || n > n_max_)
      throw std::runtime_error("zerork_b200: nReactors outside [0, nReactorsMax]");
  }
  int n_max_;
};

}  // namespace zerork_b200

#endif  // __cplusplus
#endif  // ZERORK_B200_MECHANISM_H
