#include "model.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <sstream>

namespace cqg {

size_t System::totalDimension() const {
  size_t d = 1;
  for (auto n : dims_) d *= n;
  return d;
}

bool System::isHamiltonian() const {
  for (auto& p : placed_)
    if (p.e->isHamiltonian) return true;
  return false;
}
bool System::isLiouvillean() const {
  for (auto& p : placed_)
    if (p.e->isLiouvillean) return true;
  return false;
}
bool System::isExact() const {
  for (auto& p : placed_)
    if (p.e->isExact()) return true;
  return false;
}

System System::free(const ElementPtr& f) {
  System s;
  s.dims_ = f->dims;
  s.placed_.push_back({f, {0}, 0});
  s.highestFrequency_ = f->highestFrequency;
  s.lower();
  return s;
}

System System::binary(const ElementPtr& ia) {
  if (ia->frees.size() != 2) throw std::invalid_argument("binary::make needs a binary interaction");
  System s;
  s.binary_ = true;
  s.dims_ = {ia->frees[0]->dims.at(0), ia->frees[1]->dims.at(0)};
  s.placed_.push_back({ia->frees[0], {0}, 0});
  s.placed_.push_back({ia->frees[1], {1}, 0});
  s.placed_.push_back({ia, {0, 1}, 0});
  // binary::Base::highestFrequency_v (BinarySystem.cc:47-51)
  s.highestFrequency_ =
      std::max(ia->highestFrequency, std::max(ia->frees[0]->highestFrequency, ia->frees[1]->highestFrequency));
  s.lower();
  return s;
}

System System::composite(const std::vector<ElementPtr>& frees, const std::vector<Act>& acts) {
  System s;
  for (auto& f : frees) s.dims_.push_back(f->dims.at(0));
  for (size_t i = 0; i < frees.size(); ++i) s.placed_.push_back({frees[i], {int(i)}, 0});
  for (auto& a : acts) {
    if (a.axes.size() != a.ia->frees.size()) throw std::invalid_argument("composite act arity mismatch");
    for (size_t k = 0; k < a.axes.size(); ++k) {
      if (a.axes[k] < 0 || size_t(a.axes[k]) >= frees.size() || frees[a.axes[k]] != a.ia->frees[k])
        throw std::invalid_argument("composite act does not match the frees");
    }
    s.placed_.push_back({a.ia, a.axes, 0});
  }
  // composite::Base::highestFrequency_v takes the frees only (Composite.tcc:117-125)
  for (auto& f : frees) s.highestFrequency_ = std::max(s.highestFrequency_, f->highestFrequency);
  s.lower();
  return s;
}

const cqg_complex* System::store(const CVec& v) {
  arrays_.emplace_back(v.size());
  auto& a = arrays_.back();
  for (size_t i = 0; i < v.size(); ++i) a[i] = cqg_complex{v[i].real(), v[i].imag()};
  return a.data();
}

cqg_tridiagonal System::place(const Tridiagonal& t, const std::vector<int>& axes) {
  cqg_tridiagonal d{};
  d.rank = t.rank();
  if (d.rank < 1 || d.rank > CQG_MAX_RANK || size_t(d.rank) != axes.size())
    throw std::invalid_argument("tridiagonal rank does not match its axes");
  for (int a = 0; a < d.rank; ++a) {
    d.axes[a] = axes[a];
    d.differences[a] = int64_t(t.differences()[a]);
    if (t.dims()[a] != dims_[axes[a]]) throw std::invalid_argument("tridiagonal dimension does not match the system");
  }
  ptrArrays_.emplace_back(t.length(), nullptr);
  auto& dp = ptrArrays_.back();
  for (size_t j = 0; j < t.length(); ++j)
    if (!t.diagonals()[j].empty()) {
      if (t.diagonals()[j].size() != t.boxSize(j)) throw std::invalid_argument("diagonal has the wrong size");
      dp[j] = store(t.diagonals()[j]);
    }
  d.diagonals = dp.data();
  if (t.hasFreqs()) {
    ptrArrays_.emplace_back(t.length(), nullptr);
    auto& fp = ptrArrays_.back();
    for (size_t j = 0; j < t.length(); ++j)
      if (!t.freqs()[j].empty() && !t.diagonals()[j].empty()) fp[j] = store(t.freqs()[j]);
    d.freqs = fp.data();
  }
  return d;
}

void System::lower() {
  // column offsets: frees then acts, as binary::average / composite::averageLA
  int col = 0;
  for (auto& p : placed_) {
    p.colOffset = col;
    col += int(p.e->avLabels.size());
    for (auto& l : p.e->avLabels) labels_.push_back(l);
  }
  nAvr_ = col;

  for (auto& p : placed_)
    for (auto& h : p.e->hOverI) ham_.push_back(place(h, p.axes));

  desc_ = cqg_system_desc{};
  desc_.rank = int32_t(dims_.size());
  if (desc_.rank < 1 || desc_.rank > CQG_MAX_RANK) throw std::invalid_argument("system rank out of range");
  for (int a = 0; a < desc_.rank; ++a) desc_.dims[a] = int64_t(dims_[a]);

  for (auto& p : placed_)
    if (p.axes.size() == 1 && !p.e->exact.empty() && !p.e->exact[0].empty())
      desc_.exact[p.axes[0]] = store(p.e->exact[0]);

  for (auto& p : placed_)
    for (auto& j : p.e->jumps) {
      cqg_jump cj{};
      cj.op = place(j.J, p.axes);
      cj.rate_axis = p.axes.at(j.rateAxis);
      if (!j.weights.empty()) {
        weights_.push_back(j.weights);
        cj.rate_weights = weights_.back().data();
      }
      jumps_.push_back(cj);
    }

  for (auto& p : placed_)
    for (auto& o : p.e->obs) {
      cqg_observable co{};
      if (!o.dense.empty()) {
        co.dense = store(o.dense);
        co.dense_axis = p.axes.at(o.denseAxis);
        co.op.rank = 0;
        if (!o.fourierWeights.empty()) {
          weights_.push_back(o.fourierWeights);
          co.fourier = 1;
          co.fourier_weights = weights_.back().data();
        }
      } else {
        co.op = place(o.op, p.axes);
      }
      co.col_re = o.colRe >= 0 ? o.colRe + p.colOffset : -1;
      co.col_im = o.colIm >= 0 ? o.colIm + p.colOffset : -1;
      obs_.push_back(co);
    }

  desc_.n_ham = int32_t(ham_.size());
  desc_.ham = ham_.data();
  desc_.has_hamiltonian = isHamiltonian() ? 1 : 0;
  desc_.n_jumps = int32_t(jumps_.size());
  desc_.jumps = jumps_.data();
  desc_.n_obs = int32_t(obs_.size());
  desc_.obs = obs_.data();
  desc_.n_avr = nAvr_;
  desc_.highest_frequency = highestFrequency_;
}

void System::process(double* averages) const {
  for (auto& p : placed_)
    if (p.e->process) p.e->process(averages + p.colOffset);
}

EvolutionPars::EvolutionPars(ParameterTable& p) {
  const std::string m;
  epsRel = p.add<double>("eps", m, 1e-6);
  epsAbs = p.add<double>("epsAbs", m, 1e-12);
  logLevel = p.add<int>("logLevel", m, 0);
  seed = p.add<unsigned long>("seed", m, 1001ul);
  prngStream = p.add<unsigned long>("prngStream", m, 1ul);
  noise = p.addSwitch("noise", m, true);
  nTraj = p.add<size_t>("nTraj", m, 500);
  dpLimit = p.add<double>("dpLimit", m, 0.01);
  overshootTolerance = p.add<double>("overshootTolerance", m, 10.);
  nBins = p.add<size_t>("nBins", m, 0);
  nJumpsPerBin = p.add<size_t>("nJumpsPerBin", m, 50);
  T = p.add<double>("T", m, 1.);
  dc = p.add<int>("dc", m, 10);
  Dt = p.add<double>("Dt", m, .1);
  NDt = p.add<long>("NDt", m, 0L);
  p.add<std::string>("o", m, "");
  p.add<std::string>("initialFileName", m, "");
  precision = p.add<int>("precision", m, 6);
  p.addSwitch("streamInfo", m, true);
  p.addSwitch("firstStateStream", m, true);
  sdf = p.add<unsigned>("sdf", m, 0u);
  p.add<double>("autoStopEpsilon", m, 1e-6);
  p.add<double>("autoStopEpsilonAbs", m, 1e-12);
  p.add<unsigned>("autoStopRepetition", m, 0u);
  evol = p.add<std::string>("evol", m, "single");
  p.add<int>("ems", m, 0);
  if (evol != "single" && evol != "ensemble" && evol != "master")
    throw std::invalid_argument("Parameter \"evol\" supplied with incorrect syntax");
  picture = parsePicture(p.add<std::string>("picture", m, "IP"));
  if (evol == "master" && picture == Picture::IP) picture = Picture::UIP;  // QM_Picture.cc:41-50
  prec = p.add<std::string>("enginePrecision", m, "fp64");
  rng = p.add<std::string>("rng", m, "pcg64");
}

std::string System::keyText(int firstColumn) const {
  std::ostringstream os;
  if (binary_) os << "Binary system\n";  // binary::streamKey (BinarySystem.cc:120-127)
  int col = firstColumn;
  for (auto& p : placed_) {
    if (p.e->avLabels.empty()) continue;
    os << p.e->keyTitle << "\n";
    for (auto& l : p.e->avLabels) {
      char num[16];
      std::snprintf(num, sizeof num, "%2d. ", col++);
      os << num << l << "\n";
    }
  }
  return os.str();
}

std::string System::parametersText() const {
  std::ostringstream os;
  for (auto& p : placed_) {
    std::string t = p.e->parsStream;
    if (t.empty()) t = p.e->keyTitle + "\n";
    if (t.back() != '\n') t += "\n";
    os << t;
    if (p.axes.size() == 1) os << "Dimension: " << dims_[p.axes[0]] << "\n";
    os << "\n";
  }
  os << "System characteristics: " << (isExact() ? "Interaction picture, " : "")
     << (isHamiltonian() ? "Hamiltonian evolution, " : "") << (isLiouvillean() ? "Liouvillean evolution, " : "")
     << (nAvr_ ? "calculates Averages." : "no Averages.") << "\n";
  os << "Decay channels:\n";
  int ordinal = 0;
  for (auto& p : placed_) {
    if (p.e->jumps.empty()) continue;
    os << p.e->keyTitle << "\n";
    for (auto& j : p.e->jumps) {
      char num[16];
      std::snprintf(num, sizeof num, "%2d. ", ordinal++);
      os << num << (j.label.empty() ? std::string("jump") : j.label) << "\n";
    }
  }
  os << "Alternative Lindblads: none\n";
  return os.str();
}

}  // namespace cqg
