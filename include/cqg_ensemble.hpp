// cqg_ensemble.hpp — C++ host side of the B200 MCWF engine, over the C ABI of cqg.h and
// cqg_model.h.
//
// This is what a C++QED program links instead of its serial ensemble: a trajectory object
// with the interface that cppqedutils::trajectory::run drives (advance, getTime, getDtDid,
// stream, streamKey, streamParameters, logOnEnd, state input/output), and the run loop
// itself with the reference's dc / Dt / NDt cadence and its output format (a '#'-commented
// header with the parameters and the key to the columns, fixed-width rows, the end-of-run
// log).  Header only, C++17; link with libcqg.so.
//
//   EnsembleMCWF   quantumtrajectory::Ensemble of MCWF_Trajectory (StochasticTrajectory.h:
//                  193-256, MCWF_Trajectory.h:213-234, :406-420), every trajectory on the
//                  device; a single trajectory is an ensemble of one (with dc-mode steps)
//   MasterDevice   quantumtrajectory::Master (Master.h:153-208) on the device
//   run            cppqedutils::trajectory::run (Trajectory.h:310-339, :462-610)
//   evolve         evolve(psi, sys, pe) of a workload script (Evolution_.h:174-209)
//
// Errors are thrown as cqg::Error (a std::runtime_error carrying the CQG_E_* code), where
// the reference throws its own exception types.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cqg.h"
#include "cqg_model.h"

namespace cqg {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

inline void check(int rc) {
  if (rc != CQG_OK) throw Error(rc, cqg_last_error());
}

// ---- output formatting (CPPQEDutils/FormDouble.h:78-120, FormDouble.cc:30-40) -----------
namespace format {
constexpr int kDefaultPrecision = 6;
inline int actualPrecision(int precision) { return std::max(kDefaultPrecision, precision); }
// widest positive number: exponent digits + precision + 4 (with the separating space)
inline int widthPositive(int precision) {
  return int(std::log10(-std::log10(std::numeric_limits<double>::min()))) + 1 + precision + 4;
}
inline int widthAny(int precision) { return widthPositive(precision) + 1; }
// one number, left-adjusted in its field
inline std::string field(double v, int precision, int width) {
  std::ostringstream s;
  s.precision(precision);
  s.width(width);
  s.setf(std::ios_base::left, std::ios_base::adjustfield);
  s << v;
  return s.str();
}
// every line of text prefixed with "# " (empty lines stay empty), as CommentingStream
inline std::string commented(const std::string& text) {
  std::string out;
  std::istringstream in(text);
  std::string line;
  while (std::getline(in, line)) out += line.empty() ? "\n" : "# " + line + "\n";
  return out;
}
}  // namespace format

// ---- the model and the device system -----------------------------------------------------
class Model {
 public:
  Model(const std::string& script, const std::vector<std::string>& args) {
    std::vector<const char*> argv;
    for (auto& a : args) argv.push_back(a.c_str());
    check(cqg_model_create(script.c_str(), int32_t(argv.size()), argv.data(), &m_));
  }
  ~Model() { cqg_model_destroy(m_); }
  Model(const Model&) = delete;
  Model& operator=(const Model&) = delete;

  const cqg_system_desc& desc() const {
    const cqg_system_desc* d = nullptr;
    check(cqg_model_desc(m_, &d));
    return *d;
  }
  int64_t dimension() const {
    int64_t d = 0;
    check(cqg_model_dimension(m_, &d));
    return d;
  }
  int nAvr() const {
    int32_t n = 0;
    check(cqg_model_n_avr(m_, &n));
    return n;
  }
  std::vector<cqg_complex> initialState() const {
    std::vector<cqg_complex> psi(static_cast<size_t>(dimension()));
    check(cqg_model_initial_state(m_, psi.data()));
    return psi;
  }
  cqg_run_pars runPars() const {
    cqg_run_pars p{};
    check(cqg_model_run_pars(m_, &p));
    return p;
  }
  void process(std::vector<double>& averages) const { check(cqg_model_process(m_, averages.data())); }
  std::string keyText(int firstColumn) const { return text(&cqg_model_key_text, firstColumn); }
  std::string parametersText() const { return text(&cqg_model_parameters_text); }
  std::string commandLine() const { return text(&cqg_model_command_line); }

 private:
  template <typename F, typename... A>
  std::string text(F f, A... a) const {
    size_t need = 0;
    check(f(m_, a..., nullptr, 0, &need));
    std::string s(need, '\0');
    check(f(m_, a..., &s[0], need, &need));
    s.resize(need ? need - 1 : 0);
    return s;
  }
  cqg_model* m_ = nullptr;
};

class System {
 public:
  explicit System(const Model& m) { check(cqg_system_create(&m.desc(), &s_)); }
  ~System() { cqg_system_destroy(s_); }
  System(const System&) = delete;
  System& operator=(const System&) = delete;
  const cqg_system* get() const { return s_; }

 private:
  cqg_system* s_ = nullptr;
};

// ---- the ensemble logger's histogram (MCWF_TrajectoryLogger.cc:79-121) ---------------------
// Boost.Accumulators' density with the whole sample as its cache: nBins equal bins between
// the smallest and the largest sample, an underflow bin in front and an overflow bin behind;
// per bin its lower edge and the fraction of the samples in it.
inline std::vector<std::pair<double, double>> jumpDensity(const std::vector<double>& samples, size_t nBins) {
  const auto mm = std::minmax_element(samples.begin(), samples.end());
  const double lo = *mm.first, hi = *mm.second, width = (hi - lo) / double(nBins);
  std::vector<double> edges(nBins + 2);
  for (size_t i = 0; i < nBins + 2; ++i) edges[i] = lo + (double(i) - 1.) * width;
  std::vector<double> counts(nBins + 2, 0.);
  for (double x : samples) {
    if (x < edges[1])
      counts[0] += 1;
    else if (x >= edges[nBins + 1])
      counts[nBins + 1] += 1;
    else {
      size_t k = 1;
      while (k < nBins + 1 && x >= edges[k + 1]) ++k;
      counts[k] += 1;
    }
  }
  std::vector<std::pair<double, double>> out;
  for (size_t i = 0; i < nBins + 2; ++i) out.emplace_back(edges[i], counts[i] / double(samples.size()));
  return out;
}

// ---- the ensemble ----------------------------------------------------------------------
class EnsembleMCWF {
 public:
  // nTraj trajectories from the model's initial state, trajectory i on random stream
  // p.prng_stream + i (mcwf::makeEnsemble, MCWF_Trajectory.h:213-234)
  EnsembleMCWF(const Model& model, const System& system, int64_t nTraj, const cqg_mcwf_pars& p, int logLevel = 0)
      : model_(model), nTraj_(nTraj), pars_(p), logLevel_(logLevel) {
    const auto psi0 = model.initialState();
    check(cqg_ensemble_create(system.get(), psi0.data(), nTraj, &p, &e_));
    check(cqg_ensemble_set_jump_capacity(e_, 256));
    int64_t n = 0;
    check(cqg_ensemble_size(e_, &n, &nAvr_));
    sums_.assign(size_t(nAvr_) + 1, 0.);
    drained_.assign(size_t(nTraj), 0);
    jumps_.resize(size_t(nTraj));
    check(cqg_ensemble_steps(e_, 0, 0., sums_.data()));  // averages of the initial states
  }
  ~EnsembleMCWF() { cqg_ensemble_destroy(e_); }
  EnsembleMCWF(const EnsembleMCWF&) = delete;
  EnsembleMCWF& operator=(const EnsembleMCWF&) = delete;

  // Ensemble::advance (StochasticTrajectory.h:220): every trajectory by deltaT
  void advance(double deltaT) {
    check(cqg_ensemble_run(e_, deltaT, 1, sums_.data()));
    time_ = time_ + deltaT;
    drainJumps();
  }
  // n consecutive intervals of Dt in one launch; rows[k] receives the ensemble sums after
  // interval k (the linear averages, then dtDid), the state after the last is kept
  void advanceIntervals(double Dt, int n, std::vector<std::vector<double>>& rows) {
    std::vector<double> all(size_t(n) * (size_t(nAvr_) + 1));
    check(cqg_ensemble_run(e_, Dt, n, all.data()));
    rows.clear();
    for (int k = 0; k < n; ++k) {
      rows.emplace_back(all.begin() + size_t(k) * (nAvr_ + 1), all.begin() + size_t(k + 1) * (nAvr_ + 1));
      time_ = time_ + Dt;
    }
    sums_ = rows.back();
    drainJumps();
  }
  // dc mode of a single trajectory: n MCWF steps of size T - t, stopping at T
  // (MCWF_Trajectory::step, MCWF_Trajectory.h:347-374)
  void steps(int n, double T) {
    check(cqg_ensemble_steps(e_, n, T, sums_.data()));
    std::vector<double> t(static_cast<size_t>(nTraj_));
    check(cqg_ensemble_get_times(e_, t.data(), nullptr, nullptr));
    time_ = t[0];
    drainJumps();
  }

  double getTime() const { return time_; }
  double getDtDid() const { return sums_[size_t(nAvr_)] / double(nTraj_); }
  int64_t size() const { return nTraj_; }

  // processed ensemble averages of the last advance, '\t' first (Ensemble::stream)
  std::vector<double> averages() const {
    std::vector<double> a(sums_.begin(), sums_.begin() + nAvr_);
    for (auto& v : a) v /= double(nTraj_);
    model_.process(a);
    return a;
  }
  std::ostream& stream(std::ostream& os, int precision) const {
    os << '\t';
    const int p = format::actualPrecision(precision);
    for (double v : averages()) os << format::field(v, p, format::widthAny(p));
    return os;
  }
  std::ostream& streamKey(std::ostream& os) const { return os << model_.keyText(3); }
  std::ostream& streamParameters(std::ostream& os) const {
    if (nTraj_ > 1) os << "Ensemble of " << nTraj_ << " trajectories.\n";
    os << "ODE engine: Boost.Odeint controlled stepper RKCK54. Parameters: epsRel=" << pars_.eps_rel
       << ", epsAbs=" << pars_.eps_abs << "\n";
    os << "Random engine: " << (pars_.rng == CQG_RNG_PCG64 ? "PCG64" : "Philox4x32-10")
       << ". Parameters: seed=" << pars_.seed << ", streamOrdo=" << pars_.prng_stream << "\n";
    os << "MCWF Trajectory Parameters: dpLimit=" << pars_.dp_limit
       << " (overshoot tolerance factor)=" << pars_.overshoot_tolerance << "\n\n";
    return os << model_.parametersText();
  }

  // end-of-run log: mcwf::EnsembleLogger::stream for an ensemble, mcwf::Logger::onEnd (at
  // log level > 0) for a single trajectory (MCWF_TrajectoryLogger.cc:19-33, 79-121)
  std::ostream& logOnEnd(std::ostream& os, size_t nBins = 0, size_t nJumpsPerBin = 50) const {
    const size_t n = size_t(nTraj_);
    std::vector<uint64_t> c(8 * n);
    std::vector<double> mo(n), mt(n), mn(n);
    check(cqg_ensemble_get_counters(e_, c.data()));
    check(cqg_ensemble_get_logger_maxima(e_, mo.data(), mt.data(), mn.data()));
    if (nTraj_ == 1) {
      if (logLevel_) {
        os << "\nTotal number of MCWF steps: " << c[0] << "\n\ndpLimit overshot: " << c[4]
           << " times, maximal overshoot: " << mo[0] << "\ndpTolerance overshot: " << c[5]
           << " times, maximal overshoot: " << mt[0] << "\n\nMaximal deviation of norm from 1: " << mn[0]
           << "\n\nMCWF Trajectory:\n";
        for (auto& j : jumps_[0]) os << j.first << "\t" << j.second << "\n";
        os << "\n";
      }
      return os;
    }
    auto avg = [&](int k) {
      double s = 0;
      for (size_t i = 0; i < n; ++i) s += double(c[8 * i + k]);
      return s / double(n);
    };
    os << "\nAverage number of total steps: " << avg(0) << "\n"
       << "\nOn average, dpLimit overshot: " << avg(4) << " times, maximal overshoot: "
       << *std::max_element(mo.begin(), mo.end()) << "\nOn average, dpTolerance overshot: " << avg(5)
       << " times, maximal overshoot: " << *std::max_element(mt.begin(), mt.end()) << "\n"
       << "\nMaximal deviation of norm from 1: " << *std::max_element(mn.begin(), mn.end()) << "\n";
    size_t total = 0;
    for (size_t i = 0; i < n; ++i) total += size_t(c[8 * i + 6]);
    if (!nBins && total < 2 * nJumpsPerBin) {
      os << "\nToo few jumps for a histogram\n";
    } else {
      const size_t bins = nBins ? nBins : total / nJumpsPerBin;
      std::vector<double> times;
      for (auto& tr : jumps_)
        for (auto& j : tr) times.push_back(j.first);
      os << "\nHistogram of jumps. Number of bins=" << bins + 2 << "\n";
      if (!jumpsComplete_) os << "(from the last jumps of each trajectory: earlier records were overwritten)\n";
      for (auto& b : jumpDensity(times, bins)) os << b.first << "\t" << b.second << "\n";
    }
    return os << "\nAverage number of total jumps: " << double(total) / double(n) << "\n";
  }

  // every jump (time, Lindblad ordinal) of trajectory i so far; complete unless some
  // trajectory jumped more often within one advance than its ring holds
  const std::vector<std::pair<double, int>>& jumps(int64_t i) const { return jumps_.at(size_t(i)); }
  bool jumpsComplete() const { return jumpsComplete_; }

  // state input / output (trajectory::writeViaSStream / readViaSStream, Trajectory.h:353-424)
  std::string saveState() const {
    uint64_t size = 0;
    check(cqg_ensemble_save(e_, nullptr, 0, &size));
    std::string buf(size, '\0');
    check(cqg_ensemble_save(e_, &buf[0], size, &size));
    std::ostringstream os;
    os.write(reinterpret_cast<const char*>(&time_), sizeof time_);
    os.write(buf.data(), std::streamsize(buf.size()));
    return os.str();
  }
  void loadState(const std::string& s) {
    if (s.size() < sizeof time_) throw Error(CQG_E_INVALID, "state too short");
    std::memcpy(&time_, s.data(), sizeof time_);
    check(cqg_ensemble_load(e_, s.data() + sizeof time_, s.size() - sizeof time_));
    check(cqg_ensemble_steps(e_, 0, 0., sums_.data()));
    std::vector<uint64_t> counts(static_cast<size_t>(nTraj_));
    check(cqg_ensemble_get_jump_rings(e_, nullptr, counts.data(), nullptr, nullptr));
    for (size_t i = 0; i < counts.size(); ++i) drained_[i] = counts[i];
    for (auto& j : jumps_) j.clear();
    jumpsComplete_ = false;  // the records before the checkpoint are not kept here
  }

  cqg_ensemble* get() const { return e_; }

 private:
  // copies the jump records made since the last call into the host lists, and doubles the
  // ring capacity when an advance came close to filling a ring
  void drainJumps() {
    int32_t cap = 0;
    check(cqg_ensemble_get_jump_rings(e_, &cap, nullptr, nullptr, nullptr));
    std::vector<uint64_t> counts(static_cast<size_t>(nTraj_));
    std::vector<double> t(size_t(nTraj_) * size_t(cap));
    std::vector<int32_t> l(t.size());
    check(cqg_ensemble_get_jump_rings(e_, nullptr, counts.data(), t.data(), l.data()));
    uint64_t most = 0;
    for (size_t i = 0; i < counts.size(); ++i) {
      const uint64_t fresh = counts[i] - drained_[i];
      most = std::max(most, fresh);
      if (fresh > uint64_t(cap)) jumpsComplete_ = false;
      for (uint64_t k = counts[i] - std::min<uint64_t>(fresh, uint64_t(cap)); k < counts[i]; ++k)
        jumps_[i].emplace_back(t[i * size_t(cap) + k % uint64_t(cap)], int(l[i * size_t(cap) + k % uint64_t(cap)]));
      drained_[i] = counts[i];
    }
    if (2 * most > uint64_t(cap) && cap < (1 << 16)) check(cqg_ensemble_set_jump_capacity(e_, 4 * cap));
  }

  const Model& model_;
  cqg_ensemble* e_ = nullptr;
  int64_t nTraj_ = 0;
  int32_t nAvr_ = 0;
  cqg_mcwf_pars pars_{};
  int logLevel_ = 0;
  double time_ = 0.;
  std::vector<double> sums_;
  std::vector<uint64_t> drained_;
  std::vector<std::vector<std::pair<double, int>>> jumps_;
  bool jumpsComplete_ = true;
};

// ---- the master equation on the device ----------------------------------------------------
class MasterDevice {
 public:
  MasterDevice(const Model& model, const System& system, const cqg_mcwf_pars& p) : model_(model), pars_(p) {
    const auto psi0 = model.initialState();
    check(cqg_master_create(system.get(), psi0.data(), &p, &m_));
    nAvr_ = model.nAvr();
    vals_.assign(size_t(nAvr_) + 1, 0.);
    check(cqg_master_averages(m_, vals_.data()));
  }
  ~MasterDevice() { cqg_master_destroy(m_); }
  MasterDevice(const MasterDevice&) = delete;
  MasterDevice& operator=(const MasterDevice&) = delete;

  void advance(double deltaT) {
    check(cqg_master_run(m_, deltaT, 1, vals_.data()));
    readTime();
  }
  void advanceIntervals(double Dt, int n, std::vector<std::vector<double>>& rows) {
    rows.clear();
    for (int k = 0; k < n; ++k) {
      advance(Dt);
      rows.push_back(vals_);
    }
  }
  void steps(int n, double T) {
    check(cqg_master_steps(m_, n, T, vals_.data()));
    readTime();
  }
  double getTime() const { return time_; }
  double getDtDid() const { return vals_[size_t(nAvr_)]; }
  int64_t size() const { return 1; }
  std::vector<double> averages() const {
    std::vector<double> a(vals_.begin(), vals_.begin() + nAvr_);
    model_.process(a);
    return a;
  }
  std::ostream& stream(std::ostream& os, int precision) const {
    os << '\t';
    const int p = format::actualPrecision(precision);
    for (double v : averages()) os << format::field(v, p, format::widthAny(p));
    return os;
  }
  std::ostream& streamKey(std::ostream& os) const { return os << model_.keyText(3); }
  std::ostream& streamParameters(std::ostream& os) const {
    os << "ODE engine: Boost.Odeint controlled stepper RKCK54. Parameters: epsRel=" << pars_.eps_rel
       << ", epsAbs=" << pars_.eps_abs << "\nSolving Master equation.\n\n";
    return os << model_.parametersText();
  }
  std::ostream& logOnEnd(std::ostream& os) const { return os; }

 private:
  void readTime() {
    double t = 0, did = 0, tr = 0;
    check(cqg_master_get_times(m_, &t, &did, &tr));
    time_ = t;
  }
  const Model& model_;
  cqg_master* m_ = nullptr;
  cqg_mcwf_pars pars_{};
  int32_t nAvr_ = 0;
  double time_ = 0.;
  std::vector<double> vals_;
};

// ---- the run loop (Trajectory.h:462-610) ---------------------------------------------------
// Streams the header (unless continuing), a row at t = 0 (unless continuing), then rows in
// dc mode (every dc steps until T, for a trajectory that has steps), NDt mode (NDt intervals
// of Dt) or Dt mode (intervals of Dt until T, the last one shortened), and the end-of-run
// log.  Consecutive full intervals go to the device in one launch; each trajectory advances
// by exactly the same Dt as cppqedutils::advance would make it.
template <typename Traj>
void run(Traj& traj, const Model& model, const cqg_run_pars& p, std::ostream& os, bool continuing = false) {
  using format::actualPrecision;
  using format::field;
  using format::widthPositive;
  const int prec = actualPrecision(format::kDefaultPrecision);
  const bool dcMode = p.dc && traj.size() == 1 && p.evol != CQG_EVOL_ENSEMBLE;
  if (!dcMode && !(p.Dt > 0)) throw Error(CQG_E_INVALID, "Nonzero Dt required in trajectory::run");
  const double timeToReach = p.NDt ? traj.getTime() + double(p.NDt) * p.Dt : p.T;
  if (timeToReach && timeToReach <= traj.getTime()) return;
  os.precision(prec);
  if (!continuing) {
    std::ostringstream h;
    h << model.commandLine() << "\n\n"
      << "B200 MCWF engine (cppqed_b200), C ABI version " << cqg_abi_version() << "\n\n";
    traj.streamParameters(h);
    h << "\nKey to data:\nTrajectory\n 1. time\n 2. dtDid\n";
    traj.streamKey(h);
    h << "\nRun Trajectory up to time " << timeToReach << " -- Stream period: ";
    if (dcMode)
      h << p.dc << " timestep";
    else
      h << p.Dt;
    h << "\n\n";
    os << format::commented(h.str());
  } else {
    os << format::commented("Continuing from time " + field(traj.getTime(), prec, 0) + " up to time " +
                            field(timeToReach, prec, 0) + "\n");
  }
  auto row = [&](double t, double dtDid, const std::vector<double>& processed) {
    os << field(t, prec, widthPositive(prec)) << field(dtDid, prec, widthPositive(prec)) << '\t';
    for (double v : processed) os << field(v, prec, format::widthAny(prec));
    os << std::endl;
  };
  auto streamNow = [&]() {
    os << field(traj.getTime(), prec, widthPositive(prec)) << field(traj.getDtDid(), prec, widthPositive(prec));
    traj.stream(os, prec);
    os << std::endl;
  };
  if (!continuing) streamNow();
  if (dcMode) {
    while (traj.getTime() < p.T) {
      traj.steps(p.dc, p.T);
      streamNow();
    }
  } else if (p.NDt) {
    std::vector<std::vector<double>> rows;
    double t = traj.getTime();
    traj.advanceIntervals(p.Dt, int(p.NDt), rows);
    for (auto& r : rows) {
      t = t + p.Dt;
      std::vector<double> a(r.begin(), r.end() - 1);
      const double n = double(traj.size());
      for (auto& v : a) v /= n;
      model.process(a);
      row(t, r.back() / n, a);
    }
  } else {
    double t = traj.getTime();
    while (t < p.T) {
      int n = 0;
      double tt = t;
      std::vector<double> ts;
      while (tt < p.T && std::min(p.Dt, p.T - tt) == p.Dt) {
        tt = tt + p.Dt;
        ts.push_back(tt);
        ++n;
      }
      if (n) {
        std::vector<std::vector<double>> rows;
        traj.advanceIntervals(p.Dt, n, rows);
        for (int k = 0; k < n; ++k) {
          std::vector<double> a(rows[k].begin(), rows[k].end() - 1);
          const double m = double(traj.size());
          for (auto& v : a) v /= m;
          model.process(a);
          row(ts[size_t(k)], rows[k].back() / m, a);
        }
        t = ts.back();
      } else {
        const double delta = p.T - t;
        traj.advance(delta);
        t = t + delta;
        streamNow();
      }
    }
  }
  std::ostringstream log;
  log.precision(prec);
  traj.logOnEnd(log);
  os << format::commented(log.str());
}

// evolve(psi, sys, pe) of a workload script: --evol single / ensemble / master on the device,
// output in the reference's trajectory file format.
inline void evolve(const std::string& script, const std::vector<std::string>& args, std::ostream& os) {
  Model model(script, args);
  System system(model);
  const cqg_run_pars p = model.runPars();
  if (p.evol == CQG_EVOL_MASTER) {
    MasterDevice m(model, system, p.mcwf);
    run(m, model, p, os);
    return;
  }
  EnsembleMCWF e(model, system, p.evol == CQG_EVOL_SINGLE ? 1 : p.n_traj, p.mcwf, p.log_level);
  run(e, model, p, os);
}

}  // namespace cqg
