// CPU ORACLE — test infrastructure only.  Not part of the engine: only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg load this library, as the
// checker and as the timed CPU baseline.
//
// A plain C++ restatement of C++QED v2.120's MCWF path, written against the same
// cqg_system_desc the GPU engine consumes.  It keeps the reference's algorithm and
// cost structure on purpose:
//   - Tridiagonal::apply slice by slice over dummy axes, diagonals in index order
//     (quantumoperator/Tridiagonal.tcc:220-263), terms in system order
//     (BinarySystem.cc:194-207, Composite.tcc:178-197), interaction-picture
//     propagation cumulative and shared by every trajectory (Tridiagonal.tcc:153-163);
//   - Boost.Odeint controlled_runge_kutta<runge_kutta_cash_karp54> (Boost 1.75, not
//     vendored in the reference): the published Cash-Karp tableau, the default error
//     checker err = max|xerr_i| / (eps_abs + eps_rel (|x_i| + |dt| |dxdt_i|)) and the
//     default step adjuster (decrease: max(0.9 err^-1/3, 0.2); increase if err < 0.5:
//     0.9 max(err, 5^-5)^-1/5), called as make_controlled(epsRel, epsAbs, ...) so the
//     user's epsRel lands in the absolute slot (ODE.h:199-214);
//   - ode_engine::Base::step (ODE.h:234-262);
//   - MCWF_Trajectory::step / coherentTimeDevelopment / manageTimeStep / performJump
//     (MCWF_Trajectory.h:250-374) with pcg64{seed, prngStream+i} and
//     std::uniform_real_distribution<double> (MCWF_Trajectory.h:161,191,208,223-226);
//   - Ensemble::advance serial over trajectories and the density-operator average
//     rho = (1/N) sum |psi><psi| at every stream (StochasticTrajectory.h:220-245,
//     MCWF_Trajectory.h:406-420);
//   - Master::step (Master.h:153-208);
//   - trajectory::run's dc / Dt / NDt loops (Trajectory.h:462-610).
// The pcg64 engine is the pcg-cpp one vendored with pyarrow (arrow_vendored::pcg64).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <memory>
#include <thread>
#include <vector>

#include "cqg.h"
#include "cqg_model.h"
#include "pcg/pcg_random.hpp"

namespace {

using dcomp = std::complex<double>;
using CVec = std::vector<dcomp>;
using pcg64 = arrow_vendored::pcg64;

thread_local std::string oracleError;

dcomp C(const cqg_complex& c) { return dcomp(c.re, c.im); }

size_t pow3(int r) {
  size_t p = 1;
  for (int i = 0; i < r; ++i) p *= 3;
  return p;
}

////////////////////////////////////////////////////////////////////////////////
// System wrapper with the reference's mutable interaction-picture caches
////////////////////////////////////////////////////////////////////////////////

struct Term {  // one Tridiagonal placed on axes
  int rank;
  int axes[CQG_MAX_RANK];
  long k[CQG_MAX_RANK];
  std::vector<CVec> orig, cur, freq;  // 3^rank; cur is propagated cumulatively
  double tCurrent = 0;
};

struct Jump {
  Term J;
  int rateAxis;
  std::vector<double> weights;  // empty: special
};

struct Obs {
  Term op;
  bool dense = false;
  CVec mat;
  int denseAxis = 0;
  int colRe, colIm;
};

struct System {
  int rank;
  long dims[CQG_MAX_RANK];
  long strides[CQG_MAX_RANK];
  size_t D;
  std::vector<Term> ham;
  bool hasH, hasLi, hasEx;
  std::vector<CVec> exact;  // per axis
  std::vector<double> exactT;  // FreeExact caches: t_ of the last update per axis
  std::vector<CVec> exactDiag;
  std::vector<Jump> jumps;
  std::vector<Obs> obs;
  int nAvr;
  double fmax;

  Term makeTerm(const cqg_tridiagonal& t) const {
    Term r;
    r.rank = t.rank;
    for (int a = 0; a < t.rank; ++a) {
      r.axes[a] = t.axes[a];
      r.k[a] = long(t.differences[a]);
    }
    const size_t L = pow3(t.rank);
    r.orig.resize(L);
    r.freq.resize(L);
    for (size_t j = 0; j < L; ++j) {
      size_t sz = 1, rem = j;
      std::vector<int> dig(t.rank);
      for (int a = t.rank - 1; a >= 0; --a) {
        dig[a] = int(rem % 3);
        rem /= 3;
      }
      for (int a = 0; a < t.rank; ++a) sz *= dig[a] == 0 ? dims[t.axes[a]] : dims[t.axes[a]] - r.k[a];
      if (t.diagonals && t.diagonals[j]) {
        r.orig[j].resize(sz);
        for (size_t i = 0; i < sz; ++i) r.orig[j][i] = C(t.diagonals[j][i]);
      }
      if (t.freqs && t.freqs[j]) {
        r.freq[j].resize(sz);
        for (size_t i = 0; i < sz; ++i) r.freq[j][i] = C(t.freqs[j][i]);
      }
    }
    r.cur = r.orig;
    return r;
  }

  explicit System(const cqg_system_desc& d) {
    rank = d.rank;
    D = 1;
    for (int a = rank - 1; a >= 0; --a) {
      dims[a] = long(d.dims[a]);
      strides[a] = long(D);
      D *= size_t(d.dims[a]);
    }
    for (int i = 0; i < d.n_ham; ++i) ham.push_back(makeTerm(d.ham[i]));
    hasH = d.has_hamiltonian != 0;
    exact.resize(rank);
    exactDiag.resize(rank);
    exactT.assign(rank, 0.);
    hasEx = false;
    for (int a = 0; a < rank; ++a)
      if (d.exact[a]) {
        hasEx = true;
        exact[a].resize(dims[a]);
        exactDiag[a].assign(dims[a], dcomp(0, 0));  // FreeExact diagonal_ starts zero, t_ = 0
        for (long n = 0; n < dims[a]; ++n) exact[a][n] = C(d.exact[a][n]);
      }
    for (int i = 0; i < d.n_jumps; ++i) {
      Jump j;
      j.J = makeTerm(d.jumps[i].op);
      j.rateAxis = d.jumps[i].rate_axis;
      if (d.jumps[i].rate_weights)
        j.weights.assign(d.jumps[i].rate_weights, d.jumps[i].rate_weights + dims[j.rateAxis]);
      jumps.push_back(j);
    }
    hasLi = d.n_jumps > 0;
    for (int i = 0; i < d.n_obs; ++i) {
      Obs o;
      const auto& co = d.obs[i];
      if (co.dense) {
        o.dense = true;
        o.denseAxis = co.dense_axis;
        const long N = dims[co.dense_axis];
        o.mat.resize(N * N);
        for (long k = 0; k < N * N; ++k) o.mat[k] = C(co.dense[k]);
      } else
        o.op = makeTerm(co.op);
      o.colRe = co.col_re;
      o.colIm = co.col_im;
      obs.push_back(o);
    }
    nAvr = d.n_avr;
    fmax = d.highest_frequency;
  }
};

// Tridiagonal::propagate (Tridiagonal.tcc:153-163): cumulative, diagonal 0 left out
void propagate(Term& t, double tau) {
  if (double dt = tau - t.tCurrent) {
    for (size_t i = 1; i < t.cur.size(); ++i)
      if (!t.cur[i].empty() && !t.freq[i].empty())
        for (size_t n = 0; n < t.cur[i].size(); ++n) t.cur[i][n] *= std::exp(dt * t.freq[i][n]);
  }
  t.tCurrent = tau;
}

// Iterates the dummy axes (those not in `t`) of a rank-R C-order array and calls
// f(base offset) for every slice.
template <typename F>
void forEachSlice(const System& s, const int* axes, int r, F&& f) {
  bool retained[CQG_MAX_RANK] = {};
  for (int a = 0; a < r; ++a) retained[axes[a]] = true;
  long idx[CQG_MAX_RANK] = {};
  while (true) {
    long base = 0;
    for (int a = 0; a < s.rank; ++a) base += idx[a] * s.strides[a];
    f(base);
    int a = s.rank - 1;
    for (; a >= 0; --a) {
      if (retained[a]) continue;
      if (++idx[a] < s.dims[a]) break;
      idx[a] = 0;
    }
    if (a < 0) break;
  }
}

// Tridiagonal<R>::apply on every slice: dpsi(out range) += d_j(box) * psi(in range)
void applyTerm(const System& s, const Term& t, const std::vector<CVec>& diags, const dcomp* psi, dcomp* dpsi) {
  const size_t L = diags.size();
  forEachSlice(s, t.axes, t.rank, [&](long base) {
    for (size_t j = 0; j < L; ++j) {
      const CVec& d = diags[j];
      if (d.empty()) continue;
      int dig[CQG_MAX_RANK];
      long ext[CQG_MAX_RANK], outOff = 0, inOff = 0;
      size_t rem = j;
      for (int a = t.rank - 1; a >= 0; --a) {
        dig[a] = int(rem % 3);
        rem /= 3;
      }
      for (int a = 0; a < t.rank; ++a) {
        const long N = s.dims[t.axes[a]], K = t.k[a];
        ext[a] = dig[a] == 0 ? N : N - K;
        if (dig[a] == 1) outOff += K * s.strides[t.axes[a]];
        if (dig[a] == 2) inOff += K * s.strides[t.axes[a]];
      }
      long m[CQG_MAX_RANK] = {};
      for (size_t c = 0; c < d.size(); ++c) {
        long off = 0;
        for (int a = 0; a < t.rank; ++a) off += m[a] * s.strides[t.axes[a]];
        dpsi[base + off + outOff] += d[c] * psi[base + off + inOff];
        for (int a = t.rank - 1; a >= 0; --a) {
          if (++m[a] < ext[a]) break;
          m[a] = 0;
        }
      }
    }
  });
}

// structure::Hamiltonian::addContribution for the whole system, OneTime = t - t0
void addContribution(System& s, double t, const dcomp* psi, dcomp* dpsi, double t0) {
  for (auto& term : s.ham) {
    bool td = false;
    for (auto& f : term.freq) td |= !f.empty();
    if (td) propagate(term, t - t0);
    applyTerm(s, term, td ? term.cur : term.orig, psi, dpsi);
  }
}

// Exact::actWithU per free in axis order (BinarySystem.cc:173-180): FreeExact::actWithU_v
// updates its diagonal when the OneTime argument changed, then multiplies.
void actWithU(System& s, double t, dcomp* psi, double t0) {
  const double tau = t - t0;
  for (int a = 0; a < s.rank; ++a) {
    if (s.exact[a].empty()) continue;
    if (tau != s.exactT[a] || s.exactDiag[a][0] == dcomp(0, 0)) {
      s.exactT[a] = tau;
      for (long n = 0; n < s.dims[a]; ++n) s.exactDiag[a][n] = std::exp(s.exact[a][n] * tau);
    }
    int ax[1] = {a};
    forEachSlice(s, ax, 1, [&](long base) {
      for (long n = 0; n < s.dims[a]; ++n) psi[base + n * s.strides[a]] *= s.exactDiag[a][n];
    });
  }
}

void actWithJ(System& s, dcomp* psi, int m) {
  const Term& J = s.jumps[m].J;
  std::vector<dcomp> in(psi, psi + s.D);
  std::fill(psi, psi + s.D, dcomp(0, 0));
  applyTerm(s, J, J.orig, in.data(), psi);
}

double normSq(const dcomp* v, size_t D) {
  double r = 0;
  for (size_t i = 0; i < D; ++i) r += std::norm(v[i]);
  return r;
}

// rates: element closed forms over the normalised state (sum of weights |psi|^2), or
// ||J psi||^2 for special jumps
std::vector<double> rates(System& s, const dcomp* psi) {
  std::vector<double> r(s.jumps.size());
  for (size_t m = 0; m < s.jumps.size(); ++m) {
    const auto& j = s.jumps[m];
    if (!j.weights.empty()) {
      const int a = j.rateAxis;
      double sum = 0;
      for (size_t i = 0; i < s.D; ++i) sum += j.weights[(i / s.strides[a]) % s.dims[a]] * std::norm(psi[i]);
      r[m] = sum;
    } else
      r[m] = -1;
  }
  return r;
}

////////////////////////////////////////////////////////////////////////////////
// Boost.Odeint controlled Cash-Karp 54 and ode_engine::Base
////////////////////////////////////////////////////////////////////////////////

struct CashKarp {
  // published Cash-Karp tableau
  static constexpr double c[6] = {0., 1. / 5, 3. / 10, 3. / 5, 1., 7. / 8};
  double a[5][5];
  double b[6], db[6];
  CashKarp() {
    std::memset(a, 0, sizeof a);
    a[0][0] = 1. / 5;
    a[1][0] = 3. / 40;
    a[1][1] = 9. / 40;
    a[2][0] = 3. / 10;
    a[2][1] = -9. / 10;
    a[2][2] = 6. / 5;
    a[3][0] = -11. / 54;
    a[3][1] = 5. / 2;
    a[3][2] = -70. / 27;
    a[3][3] = 35. / 27;
    a[4][0] = 1631. / 55296;
    a[4][1] = 175. / 512;
    a[4][2] = 575. / 13824;
    a[4][3] = 44275. / 110592;
    a[4][4] = 253. / 4096;
    const double b5[6] = {37. / 378, 0., 250. / 621, 125. / 594, 0., 512. / 1771};
    const double b4[6] = {2825. / 27648, 0., 18575. / 48384, 13525. / 55296, 277. / 14336, 1. / 4};
    for (int i = 0; i < 6; ++i) {
      b[i] = b5[i];
      db[i] = b5[i] - b4[i];
    }
  }
};
const CashKarp CK;

struct OdeEngine {
  double dtDid = 0, dtTry;
  double absSlot, relSlot;  // Boost's (eps_abs, eps_rel) after make_controlled(epsRel, epsAbs)
  size_t nDerivs = 0, nSteps = 0, nFailed = 0;
  size_t maxAttempts = 1000000;
  std::vector<CVec> k;
  CVec xtmp, xout, xerr;

  // try_step(system, x, t, dt): dxdt = f(x,t), then the embedded step.  Returns true on success.
  template <typename Sys>
  bool tryStep(Sys&& sys, CVec& x, double& t, double& dt) {
    const size_t D = x.size();
    k.resize(6, CVec(D));
    xtmp.resize(D);
    xout.resize(D);
    xerr.resize(D);
    sys(x, k[0], t);
    ++nDerivs;
    for (int s = 1; s < 6; ++s) {
      double coef[5];
      for (int i = 0; i < s; ++i) coef[i] = dt * CK.a[s - 1][i];
      for (size_t n = 0; n < D; ++n) {
        dcomp acc = 1.0 * x[n];
        for (int i = 0; i < s; ++i) acc += coef[i] * k[i][n];
        xtmp[n] = acc;
      }
      sys(xtmp, k[s], t + CK.c[s] * dt);
      ++nDerivs;
    }
    double cb[6], ce[6];
    for (int i = 0; i < 6; ++i) {
      cb[i] = dt * CK.b[i];
      ce[i] = dt * CK.db[i];
    }
    for (size_t n = 0; n < D; ++n) {
      dcomp acc = 1.0 * x[n];
      for (int i = 0; i < 6; ++i) acc += cb[i] * k[i][n];
      xout[n] = acc;
      dcomp e = ce[0] * k[0][n];
      for (int i = 1; i < 6; ++i) e += ce[i] * k[i][n];
      xerr[n] = e;
    }
    const double adxdt = std::fabs(dt);
    double err = 0;
    for (size_t n = 0; n < D; ++n)
      err = std::max(err, std::abs(xerr[n]) / (absSlot + relSlot * (std::abs(x[n]) + adxdt * std::abs(k[0][n]))));
    if (err > 1.0) {
      dt *= std::max(0.9 * std::pow(err, -1. / 3.), 0.2);
      return false;
    }
    t += dt;
    if (err < 0.5) {
      err = std::max(std::pow(5.0, -5.), err);
      dt *= 0.9 * std::pow(err, -1. / 5.);
    }
    x.swap(xout);
    return true;
  }

  // ode_engine::Base::step (ODE.h:234-262)
  template <typename Sys>
  void step(double deltaT, Sys&& sys, double& time, CVec& x) {
    const double timeBefore = time;
    const double nextDtTry = std::fabs(deltaT) < std::fabs(dtTry / 10.) ? dtTry : 0.;
    if ((deltaT > 0) != (dtTry > 0)) dtTry = -dtDid;
    if (std::fabs(dtTry) > std::fabs(deltaT)) dtTry = deltaT;
    size_t nf = 0;
    while (!tryStep(sys, x, time, dtTry)) {
      ++nf;
      if (nf > maxAttempts) throw std::runtime_error("ODE attempt limit exceeded");
    }
    dtDid = time - timeBefore;
    if (nextDtTry) dtTry = nextDtTry;
    ++nSteps;
    nFailed += nf;
  }
};

////////////////////////////////////////////////////////////////////////////////
// MCWF_Trajectory
////////////////////////////////////////////////////////////////////////////////

struct Trajectory {
  System* sys;
  CVec psi;
  double t = 0, t0 = 0;
  OdeEngine ode;
  pcg64 re;
  std::uniform_real_distribution<double> distro{};
  double dpLimit, overshootTolerance;
  bool noise;
  // logger
  size_t nSteps = 0, nOvershot = 0, nToleranceOvershot = 0;
  double dpMaxOvershoot = 0, dpToleranceMaxOvershoot = 0, normMaxDeviation = 0;
  std::vector<std::pair<double, int>> jumps;

  Trajectory(System* s, const CVec& psi0, const cqg_mcwf_pars& p, unsigned long stream)
      : sys(s), psi(psi0), re(p.seed, stream), dpLimit(p.dp_limit), overshootTolerance(p.overshoot_tolerance),
        noise(p.noise != 0) {
    ode.dtTry = p.dt_init > 0 ? p.dt_init : 1. / (10. * s->fmax);
    ode.absSlot = p.eps_rel;
    ode.relSlot = p.eps_abs;
    if (p.max_attempts > 0) ode.maxAttempts = size_t(p.max_attempts);
    if (hasLi() && !t) {  // MCWF_Trajectory.h:114-117
      auto r = rates(*sys, psi.data());
      calculateSpecialRates(r);
      manageTimeStep(r, 0, 0, false);
    }
  }

  bool hasLi() const { return noise && sys->hasLi; }

  std::vector<std::pair<int, CVec>> calculateSpecialRates(std::vector<double>& r) {
    std::vector<std::pair<int, CVec>> res;
    for (size_t i = 0; i < r.size(); ++i)
      if (r[i] < 0) {
        CVec tmp(psi);
        actWithJ(*sys, tmp.data(), int(i));
        const double n = std::sqrt(normSq(tmp.data(), tmp.size()));
        for (auto& v : tmp) v /= n;
        r[i] = n * n;
        res.push_back({int(i), tmp});
      }
    return res;
  }

  void coherentTimeDevelopment(double Dt) {
    if (sys->hasH) {
      ode.step(
          Dt,
          [this](const CVec& y, CVec& dydt, double tt) {
            std::fill(dydt.begin(), dydt.end(), dcomp(0, 0));
            addContribution(*sys, tt, y.data(), dydt.data(), t0);
          },
          t, psi);
    } else {
      const double stepToDo = hasLi() ? std::min(ode.dtTry, Dt) : Dt;
      t += stepToDo;
      ode.dtDid = stepToDo;
    }
    if (sys->hasEx) {
      actWithU(*sys, t, psi.data(), t0);
      t0 = t;
    }
    const double n = std::sqrt(normSq(psi.data(), psi.size()));
    for (auto& v : psi) v /= n;  // StateVector::renorm
    normMaxDeviation = std::max(normMaxDeviation, std::fabs(1 - n));
  }

  bool manageTimeStep(const std::vector<double>& r, double tCache, double dtDidCache, bool logControl = true) {
    double totalRate = 0.;
    for (double x : r) totalRate += x;
    const double dtDid = ode.dtDid, dtTry = ode.dtTry;
    const double liouvilleanSuggestedDtTry = dpLimit / totalRate;
    if (totalRate * dtDid > overshootTolerance * dpLimit) {
      t = tCache;
      ode.dtDid = dtDidCache;
      ode.dtTry = liouvilleanSuggestedDtTry;
      ++nToleranceOvershot;
      if (logControl) dpToleranceMaxOvershoot = std::max(dpToleranceMaxOvershoot, totalRate * dtDid);
      return true;
    } else if (totalRate * dtTry > dpLimit) {
      ++nOvershot;
      if (logControl) dpMaxOvershoot = std::max(dpMaxOvershoot, totalRate * dtTry);
    }
    ode.dtTry = sys->hasH ? std::min(ode.dtTry, liouvilleanSuggestedDtTry) : liouvilleanSuggestedDtTry;
    return false;
  }

  void performJump(const std::vector<double>& r, const std::vector<std::pair<int, CVec>>& special) {
    double random = distro(re) / ode.dtDid;
    size_t lindbladNo = 0;
    for (; random > 0 && lindbladNo != r.size(); random -= r[lindbladNo++])
      ;
    if (random < 0) {
      --lindbladNo;
      auto it = std::find_if(special.begin(), special.end(), [&](auto& x) { return x.first == int(lindbladNo); });
      if (it != special.end())
        psi = it->second;
      else {
        actWithJ(*sys, psi.data(), int(lindbladNo));
        const double normFactor = std::sqrt(r[lindbladNo]);
        if (!std::isfinite(normFactor)) throw std::runtime_error("Infinite detected in MCWF_Trajectory::performJump");
        for (auto& v : psi) v /= normFactor;
      }
      jumps.push_back({t, int(lindbladNo)});
    }
  }

  void step(double Dt) {
    const CVec psiCache(psi);
    const double tCache = t, dtDidCache = ode.dtDid;
    coherentTimeDevelopment(Dt);
    if (hasLi()) {
      auto r = rates(*sys, psi.data());
      auto special = calculateSpecialRates(r);
      for (double x : r)
        if (!std::isfinite(x)) throw std::runtime_error("non-finite rate");
      while (manageTimeStep(r, tCache, dtDidCache)) {
        psi = psiCache;
        coherentTimeDevelopment(Dt);
        r = rates(*sys, psi.data());
        special = calculateSpecialRates(r);
      }
      performJump(r, special);
    }
    ++nSteps;
  }

  void advance(double deltaT) {  // cppqedutils::advance (Trajectory.h:44-50)
    const double endTime = t + deltaT;
    while (double dt = endTime - t) step(dt);
  }
};

////////////////////////////////////////////////////////////////////////////////
// Averages
////////////////////////////////////////////////////////////////////////////////

// <psi|O|psi> for a pure state
dcomp expectation(System& s, const Obs& o, const dcomp* psi) {
  CVec opsi(s.D, dcomp(0, 0));
  if (o.dense) {
    const int a = o.denseAxis;
    int ax[1] = {a};
    const long N = s.dims[a];
    forEachSlice(s, ax, 1, [&](long base) {
      for (long i = 0; i < N; ++i) {
        dcomp acc = 0;
        for (long j = 0; j < N; ++j) acc += o.mat[i * N + j] * psi[base + j * s.strides[a]];
        opsi[base + i * s.strides[a]] = acc;
      }
    });
  } else
    applyTerm(s, o.op, o.op.orig, psi, opsi.data());
  dcomp r = 0;
  for (size_t i = 0; i < s.D; ++i) r += std::conj(psi[i]) * opsi[i];
  return r;
}

// Tr(rho O) for a density operator (row-major D x D)
dcomp expectationRho(System& s, const Obs& o, const CVec& rho) {
  // Tr(rho O) = sum_j (O rho^T ...) computed column by column: sum_i (O rho)_{ii}
  dcomp r = 0;
  CVec col(s.D), ocol(s.D);
  for (size_t j = 0; j < s.D; ++j) {
    for (size_t i = 0; i < s.D; ++i) col[i] = rho[i * s.D + j];
    std::fill(ocol.begin(), ocol.end(), dcomp(0, 0));
    if (o.dense) {
      const int a = o.denseAxis;
      int ax[1] = {a};
      const long N = s.dims[a];
      forEachSlice(s, ax, 1, [&](long base) {
        for (long i = 0; i < N; ++i) {
          dcomp acc = 0;
          for (long jj = 0; jj < N; ++jj) acc += o.mat[i * N + jj] * col[base + jj * s.strides[a]];
          ocol[base + i * s.strides[a]] = acc;
        }
      });
    } else
      applyTerm(s, o.op, o.op.orig, col.data(), ocol.data());
    r += ocol[j];
  }
  return r;
}

void averagesPure(System& s, const dcomp* psi, double* out) {
  std::fill(out, out + s.nAvr, 0.);
  for (auto& o : s.obs) {
    const dcomp e = expectation(s, o, psi);
    if (o.colRe >= 0) out[o.colRe] = e.real();
    if (o.colIm >= 0) out[o.colIm] = e.imag();
  }
}

void averagesRho(System& s, const CVec& rho, double* out) {
  std::fill(out, out + s.nAvr, 0.);
  for (auto& o : s.obs) {
    const dcomp e = expectationRho(s, o, rho);
    if (o.colRe >= 0) out[o.colRe] = e.real();
    if (o.colIm >= 0) out[o.colIm] = e.imag();
  }
}

// AverageTrajectories<MCWF_Trajectory> (MCWF_Trajectory.h:406-420)
void ensembleRho(const std::vector<Trajectory>& trajs, size_t D, CVec& rho) {
  rho.assign(D * D, dcomp(0, 0));
  for (auto& tr : trajs)
    for (size_t i = 0; i < D; ++i)
      for (size_t j = 0; j < D; ++j) rho[i * D + j] += tr.psi[i] * std::conj(tr.psi[j]);
  const double n = double(trajs.size());
  for (auto& v : rho) v /= n;
}

////////////////////////////////////////////////////////////////////////////////
// Master equation (Master.h:153-208)
////////////////////////////////////////////////////////////////////////////////

struct Master {
  System* sys;
  CVec rho;  // row-major D x D
  double t = 0, t0 = 0;
  OdeEngine ode;

  Master(System* s, const CVec& psi0, const cqg_mcwf_pars& p) : sys(s) {
    const size_t D = s->D;
    rho.resize(D * D);
    for (size_t i = 0; i < D; ++i)
      for (size_t j = 0; j < D; ++j) rho[i * D + j] = psi0[i] * std::conj(psi0[j]);
    ode.dtTry = p.dt_init > 0 ? p.dt_init : 1. / (10. * s->fmax);
    ode.absSlot = p.eps_rel;
    ode.relSlot = p.eps_abs;
  }

  void derivs(const CVec& r, CVec& dr, double tt) {
    const size_t D = sys->D;
    std::fill(dr.begin(), dr.end(), dcomp(0, 0));
    CVec col(D), dcol(D);
    for (size_t j = 0; j < D; ++j) {  // H/i on every column (fullRange<Left>)
      for (size_t i = 0; i < D; ++i) col[i] = r[i * D + j];
      std::fill(dcol.begin(), dcol.end(), dcomp(0, 0));
      addContribution(*sys, tt, col.data(), dcol.data(), t0);
      for (size_t i = 0; i < D; ++i) dr[i * D + j] = dcol[i];
    }
    // calculateTwoTimesRealPartOfSelf (CMatrix.cc:15-31)
    for (size_t i = 0; i < D; ++i) {
      dr[i * D + i] = 2. * dr[i * D + i].real();
      for (size_t j = i + 1; j < D; ++j) {
        dr[i * D + j] = dr[i * D + j] + std::conj(dr[j * D + i]);
        dr[j * D + i] = std::conj(dr[i * D + j]);
      }
    }
    // sum_m J_m rho J_m^dagger
    for (size_t m = 0; m < sys->jumps.size(); ++m) {
      CVec tmp(D * D, dcomp(0, 0));
      // J on columns
      for (size_t j = 0; j < D; ++j) {
        for (size_t i = 0; i < D; ++i) col[i] = r[i * D + j];
        actWithJ(*sys, col.data(), int(m));
        for (size_t i = 0; i < D; ++i) tmp[i * D + j] = col[i];
      }
      // Hermitian conjugate, then J on columns again
      CVec h(D * D);
      for (size_t i = 0; i < D; ++i)
        for (size_t j = 0; j < D; ++j) h[i * D + j] = std::conj(tmp[j * D + i]);
      for (size_t j = 0; j < D; ++j) {
        for (size_t i = 0; i < D; ++i) col[i] = h[i * D + j];
        actWithJ(*sys, col.data(), int(m));
        for (size_t i = 0; i < D; ++i) dr[i * D + j] += col[i];
      }
    }
  }

  void step(double deltaT) {
    const size_t D = sys->D;
    ode.step(
        deltaT, [this](const CVec& r, CVec& dr, double tt) { derivs(r, dr, tt); }, t, rho);
    if (sys->hasEx) {  // rho -> U rho U^dagger
      CVec col(D);
      for (size_t j = 0; j < D; ++j) {
        for (size_t i = 0; i < D; ++i) col[i] = rho[i * D + j];
        actWithU(*sys, t, col.data(), t0);
        for (size_t i = 0; i < D; ++i) rho[i * D + j] = col[i];
      }
      for (size_t i = 0; i < D; ++i) {
        for (size_t j = 0; j < D; ++j) col[j] = std::conj(rho[i * D + j]);
        actWithU(*sys, t, col.data(), t0);
        for (size_t j = 0; j < D; ++j) rho[i * D + j] = std::conj(col[j]);
      }
    }
    t0 = t;
    for (size_t i = 0; i < D; ++i) {
      rho[i * D + i] = 2. * rho[i * D + i].real();
      for (size_t j = i + 1; j < D; ++j) {
        rho[i * D + j] = rho[i * D + j] + std::conj(rho[j * D + i]);
        rho[j * D + i] = std::conj(rho[i * D + j]);
      }
    }
    dcomp tr = 0;
    for (size_t i = 0; i < D; ++i) tr += rho[i * D + i];
    for (auto& v : rho) v /= tr.real();
  }

  void advance(double deltaT) {
    const double endTime = t + deltaT;
    while (double dt = endTime - t) step(dt);
  }
};

////////////////////////////////////////////////////////////////////////////////
// trajectory::run (Trajectory.h:462-610) — rows of (t, dtDid, linear averages)
////////////////////////////////////////////////////////////////////////////////

struct Rows {
  std::vector<double> data;
  int width;
  void push(double t, double dtDid, const double* avr) {
    data.push_back(t);
    data.push_back(dtDid);
    for (int i = 0; i < width - 2; ++i) data.push_back(avr[i]);
  }
};

template <typename Traj, typename StepF, typename AdvanceF, typename StreamF>
void runLoop(Traj& traj, const cqg_run_pars& rp, bool hasStep, StepF&& stepF, AdvanceF&& advanceF, StreamF&& streamF) {
  auto getTime = [&] { return traj.time(); };
  if (hasStep && rp.dc) {  // dc mode, endTime mode
    const double length = rp.T;
    bool streamed = false;
    for (long count = 0; getTime() < length; ++count) {
      streamed = false;
      if (count) stepF(length - getTime());
      if (!count || !(count % rp.dc)) {
        streamF();
        streamed = true;
      }
    }
    if (!streamed) streamF();
    return;
  }
  if (!rp.Dt) throw std::runtime_error("Nonzero Dt required in trajectory::run");
  bool streamed = false;
  if (rp.NDt) {
    for (long count = 0; count <= rp.NDt; ++count) {
      if (count) advanceF(rp.Dt);
      streamF();
      streamed = true;
    }
  } else {
    const double length = rp.T;
    for (long count = 0; getTime() < length; ++count) {
      streamed = false;
      if (count) advanceF(std::min(rp.Dt, length - getTime()));
      streamF();
      streamed = true;
    }
  }
  if (!streamed) streamF();
}

struct SingleWrap {
  Trajectory* tr;
  double time() const { return tr->t; }
};
struct EnsembleWrap {
  std::vector<Trajectory>* trs;
  double time() const { return trs->front().t; }
};
struct MasterWrap {
  Master* m;
  double time() const { return m->t; }
};

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return oracleError.c_str(); }

// pcg64{seed, stream} followed by std::uniform_real_distribution<double> draws
int oracle_pcg64_uniform(uint64_t seed, uint64_t stream, int64_t n, double* out) {
  pcg64 e(seed, stream);
  std::uniform_real_distribution<double> d{};
  for (int64_t i = 0; i < n; ++i) out[i] = d(e);
  return 0;
}

// The reference's serialised pcg64 state text after seeding ("multiplier increment state").
int oracle_pcg64_state_text(uint64_t seed, uint64_t stream, int64_t n_draws, char* buf, size_t cap) {
  pcg64 e(seed, stream);
  std::uniform_real_distribution<double> d{};
  for (int64_t i = 0; i < n_draws; ++i) d(e);
  std::ostringstream os;
  os << e;
  std::strncpy(buf, os.str().c_str(), cap - 1);
  buf[cap - 1] = 0;
  return 0;
}

// dpsi = (H/i) psi at picture time tau, from freshly propagated coefficients
int oracle_apply_hamiltonian(const cqg_system_desc* d, const cqg_complex* psi, double tau, cqg_complex* dpsi) {
  try {
    System s(*d);
    CVec in(s.D), out(s.D, dcomp(0, 0));
    for (size_t i = 0; i < s.D; ++i) in[i] = C(psi[i]);
    addContribution(s, tau, in.data(), out.data(), 0.);
    for (size_t i = 0; i < s.D; ++i) dpsi[i] = {out[i].real(), out[i].imag()};
    return 0;
  } catch (const std::exception& e) {
    oracleError = e.what();
    return -1;
  }
}

// Runs the reference's run loop for rp->evol; rows are (t, dtDid, n_avr linear averages).
// final_state: D (single) or D*D (ensemble rho / master rho) complex values, may be NULL.
int oracle_run(const cqg_system_desc* d, const cqg_complex* psi0c, const cqg_run_pars* rp, double* rows,
               int64_t max_rows, int64_t* n_rows, cqg_complex* final_state) {
  try {
    System s(*d);
    CVec psi0(s.D);
    for (size_t i = 0; i < s.D; ++i) psi0[i] = C(psi0c[i]);
    Rows R;
    R.width = 2 + s.nAvr;
    std::vector<double> avr(s.nAvr);
    if (rp->evol == CQG_EVOL_SINGLE) {
      Trajectory tr(&s, psi0, rp->mcwf, rp->mcwf.prng_stream);
      SingleWrap w{&tr};
      runLoop(
          w, *rp, true, [&](double dt) { tr.step(dt); }, [&](double dt) { tr.advance(dt); },
          [&] {
            averagesPure(s, tr.psi.data(), avr.data());
            R.push(tr.t, tr.ode.dtDid, avr.data());
          });
      if (final_state)
        for (size_t i = 0; i < s.D; ++i) final_state[i] = {tr.psi[i].real(), tr.psi[i].imag()};
    } else if (rp->evol == CQG_EVOL_ENSEMBLE) {
      std::vector<Trajectory> trs;
      for (int64_t i = 0; i < rp->n_traj; ++i) trs.emplace_back(&s, psi0, rp->mcwf, rp->mcwf.prng_stream + i);
      EnsembleWrap w{&trs};
      CVec rho;
      runLoop(
          w, *rp, false, [&](double) {},
          [&](double dt) {
            for (auto& tr : trs) tr.advance(dt);
          },
          [&] {
            ensembleRho(trs, s.D, rho);
            averagesRho(s, rho, avr.data());
            double dtDid = 0;
            for (auto& tr : trs) dtDid += tr.ode.dtDid;
            R.push(trs.front().t, dtDid / double(trs.size()), avr.data());
          });
      if (final_state)
        for (size_t i = 0; i < s.D * s.D; ++i) final_state[i] = {rho[i].real(), rho[i].imag()};
    } else {
      Master m(&s, psi0, rp->mcwf);
      MasterWrap w{&m};
      runLoop(
          w, *rp, true, [&](double dt) { m.step(dt); }, [&](double dt) { m.advance(dt); },
          [&] {
            averagesRho(s, m.rho, avr.data());
            R.push(m.t, m.ode.dtDid, avr.data());
          });
      if (final_state)
        for (size_t i = 0; i < s.D * s.D; ++i) final_state[i] = {m.rho[i].real(), m.rho[i].imag()};
    }
    const int64_t nr = int64_t(R.data.size() / R.width);
    *n_rows = nr;
    if (nr > max_rows) {
      oracleError = "row buffer too small";
      return -2;
    }
    std::memcpy(rows, R.data.data(), R.data.size() * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    oracleError = e.what();
    return -1;
  }
}

// A single trajectory advanced by n_intervals of Dt (or, with Dt <= 0, n_intervals
// MCWF steps of size T - t): final state, times and logger counters.
// counters: 0 steps, 1 ODE steps, 2 failed ODE steps, 3 RHS calls, 4 overshoots,
// 5 step-backs, 6 jumps.
int oracle_trajectory(const cqg_system_desc* d, const cqg_complex* psi0c, const cqg_mcwf_pars* p, uint64_t stream,
                      double Dt, int64_t n_intervals, double T, cqg_complex* psi_out, double* times3,
                      uint64_t* counters, double* jump_times, int32_t* jump_lindblads, int64_t jump_cap,
                      int64_t* n_jumps) {
  try {
    System s(*d);
    CVec psi0(s.D);
    for (size_t i = 0; i < s.D; ++i) psi0[i] = C(psi0c[i]);
    Trajectory tr(&s, psi0, *p, stream);
    for (int64_t k = 0; k < n_intervals; ++k) {
      if (Dt > 0)
        tr.advance(Dt);
      else {
        if (tr.t >= T) break;
        tr.step(T - tr.t);
      }
    }
    if (psi_out)
      for (size_t i = 0; i < s.D; ++i) psi_out[i] = {tr.psi[i].real(), tr.psi[i].imag()};
    if (times3) {
      times3[0] = tr.t;
      times3[1] = tr.ode.dtDid;
      times3[2] = tr.ode.dtTry;
    }
    if (counters) {
      counters[0] = tr.nSteps;
      counters[1] = tr.ode.nSteps + tr.ode.nFailed;
      counters[2] = tr.ode.nFailed;
      counters[3] = tr.ode.nDerivs;
      counters[4] = tr.nOvershot;
      counters[5] = tr.nToleranceOvershot;
      counters[6] = tr.jumps.size();
    }
    if (n_jumps) *n_jumps = int64_t(tr.jumps.size());
    for (int64_t k = 0; k < jump_cap && k < int64_t(tr.jumps.size()); ++k) {
      if (jump_times) jump_times[k] = tr.jumps[k].first;
      if (jump_lindblads) jump_lindblads[k] = tr.jumps[k].second;
    }
    return 0;
  } catch (const std::exception& e) {
    oracleError = e.what();
    return -1;
  }
}

// Timed CPU ensemble (the reference's serial Ensemble::advance plus the rho average at
// every Dt), run on `threads` host threads over disjoint trajectory subsets, each
// thread with its own system copy (the reference's caches are not thread-safe).
// Returns accepted MCWF steps and wall seconds.
int oracle_ensemble_bench(const cqg_system_desc* d, const cqg_complex* psi0c, const cqg_mcwf_pars* p, int64_t n_traj,
                          double Dt, int64_t warm_intervals, int64_t n_intervals, int32_t threads, int32_t with_rho,
                          uint64_t* steps_out, double* seconds_out, double* avr_sum_out) {
  // The serial Ensemble::advance of the reference (StochasticTrajectory.h:220-245) with the
  // density-operator average at every Dt (MCWF_Trajectory.h:406-420), its trajectories split
  // over `threads` workers: warm_intervals untimed intervals first (the same time window as a
  // device run that starts after its warm-up), then n_intervals timed ones.  Steps and seconds
  // are those of the timed intervals.
  try {
    if (threads < 1) threads = 1;
    if (warm_intervals < 0 || n_intervals < 0) throw std::invalid_argument("negative interval count");
    const System proto(*d);
    CVec psi0(proto.D);
    for (size_t i = 0; i < proto.D; ++i) psi0[i] = C(psi0c[i]);
    std::vector<std::unique_ptr<System>> systems;
    std::vector<std::vector<Trajectory>> trs(threads);
    for (int w = 0; w < threads; ++w) systems.emplace_back(new System(*d));
    std::vector<uint64_t> steps(threads, 0);
    std::vector<std::vector<double>> avrs(threads, std::vector<double>(proto.nAvr * n_intervals, 0.));
    std::vector<std::string> errs(threads);
    auto phase = [&](int64_t first, int64_t count, bool timed) {
      std::vector<std::thread> pool;
      for (int w = 0; w < threads; ++w)
        pool.emplace_back([&, w] {
          try {
            System& s = *systems[w];
            if (trs[w].empty())
              for (int64_t i = w; i < n_traj; i += threads) trs[w].emplace_back(&s, psi0, *p, p->prng_stream + i);
            size_t before = 0;
            for (auto& tr : trs[w]) before += tr.nSteps;
            CVec rho;
            std::vector<double> avr(s.nAvr);
            for (int64_t k = first; k < first + count; ++k) {
              for (auto& tr : trs[w]) tr.advance(Dt);
              if (with_rho && !trs[w].empty()) {
                ensembleRho(trs[w], s.D, rho);
                averagesRho(s, rho, avr.data());
                if (timed)
                  for (int c = 0; c < s.nAvr; ++c) avrs[w][k * s.nAvr + c] = avr[c] * double(trs[w].size());
              }
            }
            size_t after = 0;
            for (auto& tr : trs[w]) after += tr.nSteps;
            if (timed) steps[w] = after - before;
          } catch (const std::exception& e) {
            errs[w] = e.what();
          }
        });
      for (auto& th : pool) th.join();
      for (auto& e : errs)
        if (!e.empty()) throw std::runtime_error(e);
    };
    phase(0, warm_intervals, false);
    auto t0 = std::chrono::steady_clock::now();
    phase(0, n_intervals, true);
    auto t1 = std::chrono::steady_clock::now();
    uint64_t total = 0;
    for (auto s : steps) total += s;
    *steps_out = total;
    *seconds_out = std::chrono::duration<double>(t1 - t0).count();
    if (avr_sum_out) {
      for (int64_t k = 0; k < proto.nAvr * n_intervals; ++k) {
        double acc = 0;
        for (int w = 0; w < threads; ++w) acc += avrs[w][k];
        avr_sum_out[k] = acc;
      }
    }
    return 0;
  } catch (const std::exception& e) {
    oracleError = e.what();
    return -1;
  }
}

}  // extern "C"
