#include "elements.hpp"

#include <cmath>
#include <sstream>

namespace cqg {

namespace {
const dcomp I1(0., 1.);
bool isNonZero(dcomp c) { return c != dcomp(0., 0.); }
}  // namespace

Picture parsePicture(const std::string& s) {
  if (s == "IP") return Picture::IP;
  if (s == "UIP") return Picture::UIP;
  if (s == "Sch") return Picture::Sch;
  throw std::invalid_argument("Parameter \"picture\" supplied with incorrect syntax");
}

double highestFrequencyOf(const std::vector<std::pair<double, double>>& realFreqs,
                          const std::vector<std::pair<dcomp, double>>& complexFreqs) {
  double r = 0, c = 0;
  for (auto& f : realFreqs) r = std::max(r, std::fabs(f.first * f.second));
  for (auto& f : complexFreqs) c = std::max(c, std::abs(f.first * f.second));
  return std::max(r, c);
}

////////////////////////////////////////////////////////////////////////////////
// Mode
////////////////////////////////////////////////////////////////////////////////
namespace mode {

Pars::Pars(ParameterTable& p, const std::string& mod) {
  cutoff = p.add<size_t>("cutoff", mod, 10);
  minitFock = p.add<size_t>("minitFock", mod, 0);
  minit = p.add<dcomp>("minit", mod, 0);
  streamLevel = p.add<size_t>("modeStreamLevel", mod, 0);
  delta = p.add<double>("deltaC", mod, -10.);
  omegaKerr = p.add<double>("omegaKerr", mod, 0.);
  omegaKerrAlter = p.add<double>("omegaKerrAlter", mod, 0.);
  eta = p.add<dcomp>("eta", mod, 0.);
  kappa = p.add<double>("kappa", mod, 10.);  // default -deltaC evaluated at registration (-(-10))
  nTh = p.add<double>("nTh", mod, 0.);
}

CVec mainDiagonal(dcomp z, double omegaKerr, size_t dim) {
  CVec res(dim);
  for (size_t n = 0; n < dim; ++n) {
    dcomp r1 = double(n) * z;
    dcomp r2 = ((double(n) - 1.) * double(n)) * (omegaKerr / I1);
    res[n] = r1 + r2;
  }
  return res;
}

Tridiagonal aop(size_t dim) {
  CVec plus(dim - 1);
  for (size_t n = 0; n + 1 < dim; ++n) plus[n] = std::sqrt(double(n) + 1.);
  return Tridiagonal::unary({}, 1, {}, plus);
}

Tridiagonal aop(const ElementPtr& m) {
  const size_t dim = m->dims.at(0);
  Tridiagonal res(aop(dim));
  if (m->modeExact) res.furnishWithFreqs(mainDiagonal(m->zI, m->omegaKerr, dim));
  return res;
}

Tridiagonal nop(const ElementPtr& m) { return Tridiagonal::unary(mainDiagonal(1., 0., m->dims.at(0))); }

namespace {

Tridiagonal pumping(dcomp eta, size_t dim) { return tridiagMinusHC(eta * aop(dim).dagger()); }

// hOverI (Mode.cc:72-84): returns an empty (rank-0) tridiagonal when neither term exists
Tridiagonal hOverI(dcomp z, dcomp eta, double omegaKerr, size_t dim) {
  const bool isPumped = isNonZero(eta);
  if (isNonZero(z)) {
    Tridiagonal res = Tridiagonal::unary(mainDiagonal(-z, omegaKerr, dim));
    if (isPumped) return res + pumping(eta, dim);
    return res;
  } else if (isPumped)
    return pumping(eta, dim);
  return Tridiagonal();
}

// mode::Hamiltonian<IS_TIME_DEPENDENT> (Mode.cc:89-107): the H/i term list
void fillHamiltonian(Element& e, bool timeDependent, dcomp zSch, dcomp zI, dcomp eta, double omegaKerr,
                     double omegaKerrAlter, size_t dim) {
  e.isHamiltonian = true;
  Tridiagonal h = hOverI(zSch, eta, omegaKerr, dim);
  if (timeDependent && h.rank() == 1) h.furnishWithFreqs(mainDiagonal(zI, omegaKerr, dim));
  if (h.rank() && !h.empty()) e.hOverI.push_back(h);
  if (omegaKerrAlter != 0.) {  // FILLKERR: a separate main-diagonal term
    CVec temp(dim);
    for (size_t n = 0; n < dim; ++n) temp[n] = ((double(n) - 1.) * double(n)) * (omegaKerrAlter / I1);
    e.hOverI.push_back(Tridiagonal::unary(temp));
  }
}

// mode::Exact (Mode.cc:36-45): U(t) = exp(-zI * t * n)
void fillExact(Element& e, dcomp zI, double omegaKerr, size_t dim) {
  e.modeExact = true;
  e.zI = zI;
  e.omegaKerr = omegaKerr;
  CVec lambda(dim);
  for (size_t n = 0; n < dim; ++n) lambda[n] = -zI * double(n);
  e.exact = {lambda};
}

// aJump / aDagJump (Mode.cc:116-135) with their rates (Mode_.h:180-211)
ElementJump aJump(double kappa, size_t dim, const std::string& label) {
  ElementJump j;
  const double fact = std::sqrt(2. * kappa);
  CVec plus(dim - 1);
  for (size_t n = 0; n + 1 < dim; ++n) plus[n] = fact * std::sqrt(double(n) + 1.);
  j.J = Tridiagonal::unary({}, 1, {}, plus);
  j.weights.resize(dim);
  for (size_t n = 0; n < dim; ++n) j.weights[n] = 2. * kappa * double(n);
  j.label = label;
  return j;
}

ElementJump aDagJump(double kappa, size_t dim, const std::string& label) {
  ElementJump j;
  const double fact = std::sqrt(2. * kappa);
  CVec minus(dim - 1);
  for (size_t n = 1; n < dim; ++n) minus[n - 1] = fact * std::sqrt(double(n));
  j.J = Tridiagonal::unary({}, 1, minus, {});
  // rate1 = 2 kappa nTh (<n> + trace)  (kappa here is kappa*nTh)
  j.weights.resize(dim);
  for (size_t n = 0; n < dim; ++n) j.weights[n] = 2. * kappa * (double(n) + 1.);
  j.label = label;
  return j;
}

void fillLiouvillean(Element& e, double kappa, double nTh, size_t dim) {
  e.isLiouvillean = true;
  if (nTh) {
    e.jumps.push_back(aJump(kappa * (nTh + 1), dim, "excitation loss"));
    e.jumps.push_back(aDagJump(kappa * nTh, dim, "excitation absorption"));
  } else
    e.jumps.push_back(aJump(kappa, dim, "excitation loss"));
}

// mode::Averaged (Mode.cc:158-201) and AveragedQuadratures (:203-267)
void fillAveraged(Element& e, size_t dim, Averaging av) {
  if (av == Averaging::None) return;
  e.avLabels = {"<number operator>", "VAR(number operator)", "real(<ladder operator>)", "imag(\")"};
  ElementObservable n, n2, a;
  CVec dn(dim), dn2(dim);
  for (size_t k = 0; k < dim; ++k) {
    dn[k] = double(k);
    dn2[k] = double(k) * double(k);
  }
  n.op = Tridiagonal::unary(dn);
  n.colRe = 0;
  n2.op = Tridiagonal::unary(dn2);
  n2.colRe = 1;
  a.op = aop(dim);
  a.colRe = 2;
  a.colIm = 3;
  e.obs = {n, n2, a};
  if (av == Averaging::Standard) {
    e.process = [](double* avr) { avr[1] -= avr[0] * avr[0]; };
  } else {
    e.avLabels.insert(e.avLabels.end(), {"VAR(X)", "VAR(Y)", "COV(X,Y)"});
    ElementObservable a2;
    CVec plus2(dim >= 2 ? dim - 2 : 0);
    for (size_t m = 0; m + 2 < dim; ++m) plus2[m] = std::sqrt((double(m) + 2.) * (double(m) + 1.));
    a2.op = Tridiagonal::unary({}, 2, {}, plus2);
    a2.colRe = 4;
    a2.colIm = 5;
    e.obs.push_back(a2);
    e.process = [](double* avr) {
      avr[1] -= avr[0] * avr[0];
      const double Re_aSqrExpVal = avr[4], Re_aExpVal = avr[2], Im_aExpVal = avr[3];
      const double a = avr[0] + .5 + Re_aSqrExpVal - 2 * Re_aExpVal * Re_aExpVal;
      const double b = avr[0] + .5 - Re_aSqrExpVal - 2 * Im_aExpVal * Im_aExpVal;
      const double c = avr[5] - 2 * Re_aExpVal * Im_aExpVal;
      avr[4] = a;
      avr[5] = b;
      avr[6] = c;
    };
  }
}

}  // namespace

// mode::make (Mode.tcc:22-55) with the class constructors (Mode.tcc:74-200)
ElementPtr make(const Pars& p, Picture qmp, Averaging av) {
  auto e = std::make_shared<Element>();
  const size_t dim = p.cutoff;
  e->keyTitle = "Mode";
  e->dims = {dim};
  const double nCut = double(dim), sqrtCut = std::sqrt(double(dim));
  std::vector<std::pair<double, double>> rf;
  std::vector<std::pair<dcomp, double>> cf;
  std::ostringstream os;
  os << "Mode\nDimension: " << dim << "\n";

  const bool lossy = p.kappa != 0., pumped = isNonZero(p.eta);
  const double kappaH = p.nTh ? p.kappa * (2. * p.nTh + 1) : p.kappa;  // finiteTemperatureHamiltonianDecay
  const dcomp zDelta(0, -p.delta);

  if (!lossy && !pumped) {
    if (qmp == Picture::Sch) {  // ModeSch
      fillHamiltonian(*e, false, zDelta, 0, 0, p.omegaKerr, p.omegaKerrAlter, dim);
      rf.push_back({-zDelta.imag(), nCut});
      os << "Schroedinger picture.\n";
    } else {  // Mode / ModeUIP
      fillExact(*e, zDelta, p.omegaKerr, dim);
      rf.push_back({-zDelta.imag(), 1.});
    }
  } else if (!lossy) {  // pumped only
    if (qmp == Picture::Sch) {
      fillHamiltonian(*e, false, zDelta, 0, p.eta, p.omegaKerr, p.omegaKerrAlter, dim);
      rf.push_back({-zDelta.imag(), nCut});
      os << "Pumped, Schroedinger picture.\n";
    } else {  // PumpedMode(UIP): Hamiltonian<true>(0, zI, eta)
      fillHamiltonian(*e, true, 0, zDelta, p.eta, p.omegaKerr, p.omegaKerrAlter, dim);
      fillExact(*e, zDelta, p.omegaKerr, dim);
      rf.push_back({-zDelta.imag(), 1.});
      os << "Pumped.\n";
    }
    cf.push_back({p.eta, sqrtCut});
  } else {
    fillLiouvillean(*e, p.kappa, p.nTh, dim);
    const dcomp zFull(kappaH, -p.delta);
    if (!pumped) {
      if (qmp == Picture::IP) {  // LossyMode: Exact only
        fillExact(*e, zFull, p.omegaKerr, dim);
        cf.push_back({std::conj(zFull), 1.});
        os << "Lossy.\n";
      } else if (qmp == Picture::UIP) {  // LossyModeUIP: Hamiltonian<true>((kappa,0),(0,-delta),0)
        fillHamiltonian(*e, true, dcomp(kappaH, 0.), zDelta, 0, p.omegaKerr, p.omegaKerrAlter, dim);
        fillExact(*e, zDelta, p.omegaKerr, dim);
        rf.push_back({kappaH, nCut});
        rf.push_back({-zDelta.imag(), 1.});
        os << "Lossy, Unitary interaction picture.\n";
      } else {  // LossyModeSch
        fillHamiltonian(*e, false, zFull, 0, 0, p.omegaKerr, p.omegaKerrAlter, dim);
        rf.push_back({kappaH, nCut});
        rf.push_back({-zFull.imag(), nCut});
        os << "Lossy, Schroedinger picture.\n";
      }
    } else {
      if (qmp == Picture::IP) {  // PumpedLossyMode: Hamiltonian<true>(0, zI, eta)
        fillHamiltonian(*e, true, 0, zFull, p.eta, p.omegaKerr, p.omegaKerrAlter, dim);
        fillExact(*e, zFull, p.omegaKerr, dim);
        cf.push_back({std::conj(zFull), 1.});
        os << "PumpedLossy.\n";
      } else if (qmp == Picture::UIP) {  // PumpedLossyModeUIP
        fillHamiltonian(*e, true, dcomp(kappaH, 0.), zDelta, p.eta, p.omegaKerr, p.omegaKerrAlter, dim);
        fillExact(*e, zDelta, p.omegaKerr, dim);
        rf.push_back({kappaH, nCut});
        rf.push_back({-zDelta.imag(), 1.});
        os << "PumpedLossy, Unitary interaction picture.\n";
      } else {  // PumpedLossyModeSch
        fillHamiltonian(*e, false, zFull, 0, p.eta, p.omegaKerr, p.omegaKerrAlter, dim);
        cf.push_back({std::conj(zFull), nCut});
        os << "PumpedLossy, Schroedinger picture.\n";
      }
      cf.push_back({p.eta, sqrtCut});
    }
  }
  fillAveraged(*e, dim, av);
  e->highestFrequency = highestFrequencyOf(rf, cf);
  e->parsStream = os.str();
  return e;
}

CVec coherent(dcomp alpha, size_t dim) {
  CVec psi(dim);
  const double norm = std::exp(-std::norm(alpha) / 2.);
  for (size_t n = 0; n < dim; ++n) {
    // mathutils::coherentElement (MathExtensions.cc:35-41) below the factorial overflow limit
    dcomp el(1., 0.);
    if (n) {
      if (n < 170) {
        double fact = 1;
        for (size_t k = 2; k <= n; ++k) fact *= double(k);
        el = std::pow(alpha, double(n)) / std::sqrt(fact);
      } else {
        const double PI = 3.14159265358979323846, EULER = 2.71828182845904523536;
        el = std::pow(2 * double(n) * PI, -.25) * std::pow(alpha / std::sqrt(double(n) / EULER), double(n));
      }
    }
    psi[n] = norm * el;
  }
  return psi;
}

CVec fock(size_t n, size_t dim, double phase) {
  if (n >= dim) throw std::overflow_error("Fock state " + std::to_string(n) + " higher than dim " + std::to_string(dim));
  CVec res(dim);
  res[n] = std::exp(I1 * phase);
  return res;
}

CVec init(const Pars& p) { return p.minitFock ? fock(p.minitFock, p.cutoff) : coherent(p.minit, p.cutoff); }

}  // namespace mode

////////////////////////////////////////////////////////////////////////////////
// Qbit: a two-level ModeBase (Qbit_.h:100-116, Qbit.cc)
////////////////////////////////////////////////////////////////////////////////
namespace qbit {

Pars::Pars(ParameterTable& p, const std::string& mod) {
  qbitInit = p.add<dcomp>("qbitInit", mod, 0.);
  delta = p.add<double>("deltaA", mod, -10.);
  eta = p.add<dcomp>("etat", mod, 0.);
  gamma = p.add<double>("gamma", mod, 10.);  // default fabs(deltaA) evaluated at registration
  gamma_parallel = p.add<double>("gamma_parallel", mod, 0.);
}

void fillQbitAveraged(Element& e);
namespace {

}  // namespace

void fillQbitAveraged(Element& e) {  // Qbit.cc:22-32
  e.avLabels = {"rho00", "rho11", "real(rho10=<sigma>)", "imag(\")"};
  ElementObservable r00, r11, s;
  r00.op = Tridiagonal::unary(CVec{1., 0.});
  r00.colRe = 0;
  r11.op = Tridiagonal::unary(CVec{0., 1.});
  r11.colRe = 1;
  s.op = mode::aop(2);
  s.colRe = 2;
  s.colIm = 3;
  e.obs = {r00, r11, s};
}

namespace {

// qbit::Hamiltonian passes -eta to mode::Hamiltonian (Qbit_.h:100-107)
void fillQbitHamiltonian(Element& e, bool td, dcomp zSch, dcomp zI, dcomp eta) {
  e.isHamiltonian = true;
  Tridiagonal h;
  const bool isPumped = isNonZero(-eta);
  if (isNonZero(zSch)) {
    h = Tridiagonal::unary(mode::mainDiagonal(-zSch, 0., 2));
    if (isPumped) h += tridiagMinusHC((-eta) * mode::aop(2).dagger());
  } else if (isPumped)
    h = tridiagMinusHC((-eta) * mode::aop(2).dagger());
  if (td && h.rank() == 1) h.furnishWithFreqs(mode::mainDiagonal(zI, 0., 2));
  if (h.rank() && !h.empty()) e.hOverI.push_back(h);
}

void fillQbitExact(Element& e, dcomp zI) {
  e.modeExact = true;
  e.zI = zI;
  e.exact = {CVec{0., -zI}};
}

ElementJump sigmaJump(double gamma) {  // Qbit.cc:38-42 and mode::aJump with dim 2
  ElementJump j;
  j.J = Tridiagonal::unary({}, 1, {}, CVec{std::sqrt(2. * gamma) * std::sqrt(1.)});
  j.weights = {0., 2. * gamma * 1.};
  j.label = "excitation loss";
  return j;
}

}  // namespace

ElementPtr make(const Pars& p, Picture qmp) {
  auto e = std::make_shared<Element>();
  e->keyTitle = "Qbit";
  e->dims = {2};
  fillQbitAveraged(*e);
  std::vector<std::pair<double, double>> rf;
  std::vector<std::pair<dcomp, double>> cf;
  const dcomp zDelta(0, -p.delta), zFull(p.gamma, -p.delta);
  const bool lossy = p.gamma != 0, pumped = isNonZero(p.eta);

  if (p.gamma_parallel) {  // LiouvilleanPhaseNoise: both jumps use the special-rate convention
    e->isLiouvillean = true;
    ElementJump s;
    s.J = Tridiagonal::unary({}, 1, {}, CVec{std::sqrt(2. * p.gamma)});
    s.label = "excitation loss";
    ElementJump z;
    const double f = std::sqrt(2. * p.gamma_parallel);
    z.J = Tridiagonal::unary(CVec{f, -f});
    z.label = "phase noise";
    e->jumps = {s, z};
    rf.push_back({p.gamma_parallel, 1.});
    if (qmp == Picture::UIP) {
      fillQbitHamiltonian(*e, true, dcomp(p.gamma, 0), zDelta, p.eta);
      fillQbitExact(*e, zDelta);
      rf.push_back({p.gamma, 1.});
      rf.push_back({-zDelta.imag(), 1.});
    } else {
      if (pumped) fillQbitHamiltonian(*e, true, 0, zFull, p.eta);
      fillQbitExact(*e, zFull);
      cf.push_back({std::conj(zFull), 1.});
    }
    if (pumped) cf.push_back({-p.eta, 1.});
    e->highestFrequency = highestFrequencyOf(rf, cf);
    return e;
  }

  if (lossy) {
    e->isLiouvillean = true;
    e->jumps.push_back(sigmaJump(p.gamma));
  }
  if (!lossy && !pumped) {
    if (qmp == Picture::Sch) {
      fillQbitHamiltonian(*e, false, zDelta, 0, 0);
      rf.push_back({-zDelta.imag(), 1.});
    } else {
      fillQbitExact(*e, zDelta);
      rf.push_back({-zDelta.imag(), 1.});
    }
  } else if (!lossy) {
    if (qmp == Picture::Sch) {
      fillQbitHamiltonian(*e, false, zDelta, 0, p.eta);
    } else {
      fillQbitHamiltonian(*e, true, 0, zDelta, p.eta);
      fillQbitExact(*e, zDelta);
    }
    rf.push_back({-zDelta.imag(), 1.});
    cf.push_back({-p.eta, 1.});
  } else if (!pumped) {
    if (qmp == Picture::IP) {
      fillQbitExact(*e, zFull);
      cf.push_back({std::conj(zFull), 1.});
    } else if (qmp == Picture::UIP) {
      fillQbitHamiltonian(*e, true, dcomp(p.gamma, 0), zDelta, 0);
      fillQbitExact(*e, zDelta);
      rf.push_back({p.gamma, 1.});
      rf.push_back({-zDelta.imag(), 1.});
    } else {
      fillQbitHamiltonian(*e, false, zFull, 0, 0);
      rf.push_back({p.gamma, 1.});
      rf.push_back({-zFull.imag(), 1.});
    }
  } else {
    if (qmp == Picture::IP) {
      fillQbitHamiltonian(*e, true, 0, zFull, p.eta);
      fillQbitExact(*e, zFull);
      cf.push_back({std::conj(zFull), 1.});
    } else if (qmp == Picture::UIP) {
      fillQbitHamiltonian(*e, true, dcomp(p.gamma, 0), zDelta, p.eta);
      fillQbitExact(*e, zDelta);
      rf.push_back({p.gamma, 1.});
      rf.push_back({-zDelta.imag(), 1.});
    } else {
      fillQbitHamiltonian(*e, false, zFull, 0, p.eta);
      cf.push_back({std::conj(zFull), 1.});
    }
    cf.push_back({-p.eta, 1.});
  }
  e->highestFrequency = highestFrequencyOf(rf, cf);
  return e;
}

Tridiagonal sigmaop(const ElementPtr& q) { return mode::aop(q); }

CVec init(dcomp psi1) { return CVec{std::sqrt(1 - std::norm(psi1)), psi1}; }

}  // namespace qbit

////////////////////////////////////////////////////////////////////////////////
// PumpedTwoLevelAtomSch (PumpedTwoLevelAtom.cc): H/i = [[0, conj(eta)], [-eta, za]]
////////////////////////////////////////////////////////////////////////////////
namespace ptla {

ElementPtr makeSch(const qbit::Pars& p) {
  auto e = std::make_shared<Element>();
  e->keyTitle = "Qbit";
  e->dims = {2};
  const dcomp za(-p.gamma, p.delta), eta = p.eta;
  e->isHamiltonian = true;
  e->hOverI.push_back(Tridiagonal::unary(CVec{0., za}, 1, CVec{-eta}, CVec{std::conj(eta)}));
  e->isLiouvillean = true;
  ElementJump j;
  j.J = Tridiagonal::unary({}, 1, {}, CVec{std::sqrt(-2. * za.real())});
  j.weights = {0., -2. * za.real()};
  j.label = "atomic decay";
  e->jumps.push_back(j);
  qbit::fillQbitAveraged(*e);
  e->highestFrequency = highestFrequencyOf({}, {{dcomp(p.gamma, p.delta), 1.}, {p.eta, 1.}});
  std::ostringstream os;
  os << "Pumped Two-Level Atom\nSchroedinger picture.\n";
  e->parsStream = os.str();
  return e;
}

}  // namespace ptla

////////////////////////////////////////////////////////////////////////////////
// JaynesCummings: H/i = tridiagMinusHC(conj(g) sigma (x) a^dagger)
////////////////////////////////////////////////////////////////////////////////
namespace jaynescummings {

ElementPtr make(const ElementPtr& q, const ElementPtr& m, dcomp g) {
  auto e = std::make_shared<Element>();
  e->keyTitle = "JaynesCummings";
  e->dims = {q->dims.at(0), m->dims.at(0)};
  e->frees = {q, m};
  if (isNonZero(g)) {
    e->isHamiltonian = true;
    e->hOverI.push_back(tridiagMinusHC((std::conj(g) * qbit::sigmaop(q)) * mode::aop(m).dagger()));
  }
  e->highestFrequency = highestFrequencyOf({}, {{g, std::sqrt(double(q->dims[0] * m->dims[0]))}});
  return e;
}

}  // namespace jaynescummings

////////////////////////////////////////////////////////////////////////////////
// CoupledModes (CoupledModes.cc:9-41)
////////////////////////////////////////////////////////////////////////////////
namespace coupledmodes {

ElementPtr make(const ElementPtr& m0, const ElementPtr& m1, Kind kind, dcomp u) {
  auto e = std::make_shared<Element>();
  e->keyTitle = "CoupledModes";
  e->dims = {m0->dims.at(0), m1->dims.at(0)};
  e->frees = {m0, m1};
  if (std::abs(u)) {
    e->isHamiltonian = true;
    auto xop = [](const ElementPtr& m) { return tridiagPlusHC(mode::aop(m)) / std::sqrt(2.); };
    switch (kind) {
      case Kind::NX:
        e->hOverI.push_back(u.real() * mode::nop(m0) * xop(m1) / I1);
        break;
      case Kind::XX:
        e->hOverI.push_back(u.real() * xop(m0) * xop(m1) / I1);
        break;
      case Kind::XX_RWA:
        e->hOverI.push_back(tridiagMinusHC((std::conj(u) * mode::aop(m0)) * mode::aop(m1).dagger()));
        break;
    }
  }
  e->highestFrequency = highestFrequencyOf({}, {{u, double(m0->dims[0]) * std::sqrt(double(m1->dims[0]))}});
  return e;
}

}  // namespace coupledmodes

////////////////////////////////////////////////////////////////////////////////
// Mode functions (ModeFunction.cc), Particle (Particle.cc), ParticleCavity
// (ParticleCavity.cc), ParticleTwoModes (ParticleTwoModes.cc)
////////////////////////////////////////////////////////////////////////////////

std::istream& operator>>(std::istream& is, ModeFunctionType& mf) {
  std::string s;
  is >> s;
  if (s == "Sin")
    mf = ModeFunctionType::Sin;
  else if (s == "Cos")
    mf = ModeFunctionType::Cos;
  else if (s == "Plus")
    mf = ModeFunctionType::Plus;
  else if (s == "Minus")
    mf = ModeFunctionType::Minus;
  else
    is.setstate(std::ios_base::failbit);
  return is;
}

namespace {
const double kPi = 3.14159265358979323846;
int gslSign(double x) { return x >= 0. ? 1 : -1; }  // GSL_SIGN, used by cppqedutils::sign
}  // namespace

namespace particle {

std::istream& operator>>(std::istream& is, InitialCondition& ic) {
  std::string s;
  is >> s;
  if (s.size() < 2 || s.front() != '(' || s.back() != ')') {
    is.setstate(std::ios_base::failbit);
    return is;
  }
  std::string body = s.substr(1, s.size() - 2);
  for (char& c : body)
    if (c == ',') c = ' ';
  std::istringstream in(body);
  InitialCondition r;
  std::string flag;
  in >> r.x0 >> r.k0 >> r.sig >> flag;
  if (in.fail()) {
    is.setstate(std::ios_base::failbit);
    return is;
  }
  r.inK = flag == "1" || flag == "true";
  ic = r;
  return is;
}

Pars::Pars(ParameterTable& p, const std::string& mod) {
  omrec = p.add<double>("omrec", mod, 1.);
  fin = p.add<size_t>("fin", mod, 6);
  init = p.add<InitialCondition>("pinit", mod, InitialCondition{});
  hoInitn = p.add<int>("HOinitn", mod, -1);
}

ParsPumped::ParsPumped(ParameterTable& p, const std::string& mod) : Pars(p, mod) {
  vClass = p.add<double>("vClass", mod, -10.);
  kPart = p.add<size_t>("kPart", mod, 1);
  modePart = p.add<ModeFunctionType>("modePart", mod, ModeFunctionType::Sin);
}

Spatial::Spatial(size_t f, double dk) : fin(f), deltaK(dk) {
  xMax = kPi / deltaK;
  deltaX = 2 * xMax / double(size_t(1) << fin);
  kMax = kPi / deltaX;
}

void ffTransform(CVec& psi, Direction dir) {
  const size_t N = psi.size();
  if (N < 2) return;
  const double sgn = dir == Direction::XK ? -1. : 1.;
  CVec y(N);
  for (size_t k = 0; k < N; ++k) {
    dcomp acc = 0;
    for (size_t j = 0; j < N; ++j) {
      const double ang = sgn * 2. * kPi * double((j * k) % N) / double(N);
      acc += psi[j] * dcomp(std::cos(ang), std::sin(ang));
    }
    y[k] = acc;
  }
  const double norm = 1. / std::sqrt(double(N));
  const size_t half = N >> 1;
  for (size_t m = 0; m < N; ++m) psi[m] = norm * y[(m + half) % N] * ((m & 1) ? -1. : 1.);
}

namespace {

CVec kSquared(const Spatial& space, dcomp factor) {  // mainDiagonal(space, omrec) (Particle.cc:92-95)
  CVec d(space.dim());
  for (size_t i = 0; i < d.size(); ++i) d[i] = factor * space.k(i) * space.k(i);
  return d;
}

Tridiagonal expINKXdim(size_t dim, long nK) {  // Particle.cc:60-73
  const long D = long(dim) - (nK > 0 ? nK : -nK);
  if (D < 0) return Tridiagonal();
  CVec ones(size_t(D), dcomp(1., 0.));
  if (nK > 0) return Tridiagonal::unary({}, size_t(nK), ones, {});
  if (nK == 0) return Tridiagonal::unary(ones);
  return Tridiagonal::unary({}, size_t(-nK), {}, ones);
}

Tridiagonal cosNKXdim(size_t dim, long nK) { return (expINKXdim(dim, nK) + expINKXdim(dim, -nK)) / 2.; }

// the particle's own pump term, H/i (Particle.cc:83-87)
Tridiagonal pumpHOverI(size_t dim, double vClass, const ModeFunction& mf) {
  if (vClass && !isComplex(mf.type))
    return vClass * (mf.type == ModeFunctionType::Sin ? -1. : 1.) * cosNKXdim(dim, mf.k << 1) / (2. * I1);
  return Tridiagonal();
}

// particle::Averaged (Particle.cc:128-163): <P>, VAR(P), <X>, DEV(X); <X> and <X^2> are the
// position-space moments of the k-space state, i.e. of M rho M^+ with M the k -> x transform
void fillParticleAveraged(Element& e, const Spatial& space) {
  const size_t N = space.dim();
  e.avLabels = {"<P>", "VAR(P)", "<X>", "DEV(X)"};
  CVec dk(N), dk2(N);
  for (size_t i = 0; i < N; ++i) {
    dk[i] = space.k(i);
    dk2[i] = space.k(i) * space.k(i);
  }
  std::vector<CVec> M(N, CVec(N));  // M[m][j]: column j = transform of the unit vector e_j
  for (size_t j = 0; j < N; ++j) {
    CVec v(N, 0.);
    v[j] = 1.;
    ffTransform(v, Direction::KX);
    for (size_t m = 0; m < N; ++m) M[m][j] = v[m];
  }
  auto dense = [&](int power) {
    CVec O(N * N, 0.);
    for (size_t i = 0; i < N; ++i)
      for (size_t j = 0; j < N; ++j) {
        dcomp acc = 0;
        for (size_t m = 0; m < N; ++m) acc += std::conj(M[m][i]) * std::pow(space.x(m), power) * M[m][j];
        O[i * N + j] = acc;
      }
    return O;
  };
  ElementObservable p, p2, x, x2;
  p.op = Tridiagonal::unary(dk);
  p.colRe = 0;
  p2.op = Tridiagonal::unary(dk2);
  p2.colRe = 1;
  x.dense = dense(1);
  x.colRe = 2;
  x2.dense = dense(2);
  x2.colRe = 3;
  x.fourierWeights.resize(N);
  x2.fourierWeights.resize(N);
  for (size_t m = 0; m < N; ++m) {
    x.fourierWeights[m] = space.x(m);
    x2.fourierWeights[m] = space.x(m) * space.x(m);
  }
  e.obs = {p, p2, x, x2};
  e.process = [](double* avr) {
    avr[1] -= avr[0] * avr[0];
    avr[3] = std::sqrt(avr[3] - avr[2] * avr[2]);
  };
}

std::shared_ptr<Element> particleBase(size_t fin) {
  auto e = std::make_shared<Element>();
  e->keyTitle = "Particle";
  e->dims = {size_t(1) << fin};
  e->fin = fin;
  fillParticleAveraged(*e, Spatial(fin));
  return e;
}

void particleExact(Element& e, const Spatial& space, double omrec) {  // particle::Exact (Particle.cc:33-46)
  e.particleExact = true;
  e.omrec = omrec;
  e.exact = {kSquared(space, dcomp(0., -omrec))};  // U = exp(-i omrec k^2 t)
}

}  // namespace

// particle::make (Particle.cc:452-456): ParticleSch in the Schroedinger picture, else the
// free Particle with its Exact part only
ElementPtr make(const Pars& p, Picture qmp) {
  const Spatial space(p.fin);
  auto e = particleBase(p.fin);
  e->omrec = p.omrec;
  const double dim = double(space.dim());
  if (qmp == Picture::Sch) {
    e->isHamiltonian = true;
    e->hOverI.push_back(Tridiagonal::unary(kSquared(space, dcomp(0., -p.omrec))));
    e->highestFrequency = highestFrequencyOf({{p.omrec, dim * dim}}, {});
  } else {
    particleExact(*e, space, p.omrec);
    e->highestFrequency = highestFrequencyOf({{p.omrec, dim}}, {});
  }
  return e;
}

// particle::makePumped (Particle.cc:459-462): PumpedParticleSch / PumpedParticle
ElementPtr makePumped(const ParsPumped& p, Picture qmp) {
  const Spatial space(p.fin);
  auto e = particleBase(p.fin);
  e->omrec = p.omrec;
  e->pumpedParticle = true;
  e->vClass = p.vClass;
  e->pumpMF = ModeFunction{p.modePart, long(p.kPart)};
  const double dim = double(space.dim());
  e->isHamiltonian = true;
  Tridiagonal pump = pumpHOverI(space.dim(), p.vClass, e->pumpMF);
  if (qmp == Picture::Sch) {  // Hamiltonian<false>: -i omrec k^2 + pump
    e->hOverI.push_back(Tridiagonal::unary(kSquared(space, dcomp(0., -p.omrec))) + pump);
    e->highestFrequency = highestFrequencyOf({{p.omrec, dim * dim}, {p.vClass, 1.}}, {});
  } else {  // Hamiltonian<true>: the pump term furnished with i omrec k^2, and Exact
    if (!pump.empty()) e->hOverI.push_back(pump.furnishWithFreqs(kSquared(space, dcomp(0., p.omrec))));
    particleExact(*e, space, p.omrec);
    e->highestFrequency = highestFrequencyOf({{p.omrec, dim}, {p.vClass, 1.}}, {});
  }
  return e;
}

CVec wavePacket(const InitialCondition& init, const Spatial& space, bool kFlag) {  // Particle.cc:351-371
  double offset1 = kPi * init.x0, offset2 = init.k0;
  if (init.inK) {
    std::swap(offset1, offset2);
    offset2 = -offset2;
  }
  const size_t N = space.dim();
  CVec psi(N);
  for (size_t i = 0; i < N; ++i) {
    const double a = init.inK ? space.k(i) : space.x(i);
    psi[i] = std::exp(dcomp(-(a - offset1) * (a - offset1) / (4 * init.sig * init.sig), a * offset2));
  }
  if (kFlag && !init.inK)
    ffTransform(psi, Direction::XK);
  else if (!kFlag && init.inK)
    ffTransform(psi, Direction::KX);
  double n2 = 0;
  for (auto& c : psi) n2 += std::norm(c);
  for (auto& c : psi) c /= std::sqrt(n2);
  return psi;
}

CVec hoState(int n, const InitialCondition& init, const Spatial& space, bool kFlag) {  // Particle.cc:398-418
  if (n < 0) n = 0;
  const double kx0 = kPi * init.x0;
  const size_t N = space.dim();
  CVec psi(N);
  for (size_t j = 0; j < N; ++j) {
    const double t = (space.x(j) - kx0) / init.sig;
    double h0 = 1., h1 = 2. * t, h = n == 0 ? h0 : h1;  // physicists' Hermite polynomial H_n(t)
    for (int m = 1; m < n; ++m) {
      h = 2. * t * h1 - 2. * double(m) * h0;
      h0 = h1;
      h1 = h;
    }
    psi[j] = std::exp(-t * t / 2.) * h;
  }
  if (kFlag) ffTransform(psi, Direction::XK);
  double n2 = 0;
  for (auto& c : psi) n2 += std::norm(c);
  for (auto& c : psi) c /= std::sqrt(n2);
  return psi;
}

CVec init(const Pars& p) {  // Particle.cc:434-441
  const Spatial space(p.fin);
  return p.hoInitn < 0 ? wavePacket(p.init, space) : hoState(p.hoInitn, p.init, space);
}

CVec init(const ParsPumped& p) {
  // without an initial spread, the ground state of the pump's harmonic approximation
  // (coherent(ParsPumped), Particle.cc:377-380)
  const Spatial space(p.fin);
  InitialCondition ic = p.init;
  if (!p.init.sig) ic = InitialCondition{p.init.x0, p.init.k0, std::pow(p.omrec / std::fabs(p.vClass), .25) / std::sqrt(2.), false};
  return p.hoInitn < 0 ? wavePacket(ic, space) : hoState(p.hoInitn, ic, space);
}

Tridiagonal expINKX(const ElementPtr& particle, long nK) {  // Particle.cc:206-213
  Tridiagonal res = expINKXdim(particle->dims.at(0), nK);
  if (particle->particleExact && !res.empty())
    res.furnishWithFreqs(kSquared(Spatial(particle->fin), dcomp(0., particle->omrec)));
  return res;
}

Tridiagonal cosNKX(const ElementPtr& particle, long nK) { return (expINKX(particle, nK) + expINKX(particle, -nK)) / 2.; }
Tridiagonal sinNKX(const ElementPtr& particle, long nK) {
  return (expINKX(particle, nK) - expINKX(particle, -nK)) / (2. * I1);
}

Tridiagonal mfNKX(const ElementPtr& particle, const ModeFunction& mf) {  // Particle.cc:216-227
  switch (mf.type) {
    case ModeFunctionType::Sin:
      return sinNKX(particle, mf.k);
    case ModeFunctionType::Cos:
      return cosNKX(particle, mf.k);
    case ModeFunctionType::Plus:
      return expINKX(particle, mf.k);
    case ModeFunctionType::Minus:
      break;
  }
  return expINKX(particle, -mf.k);
}

Tridiagonal mfComposition(const ElementPtr& particle, const ModeFunction& f1, const ModeFunction& f2) {
  // Particle.cc:229-336: f1^*(k1 x) f2(k2 x) for |k1| == |k2|
  using MF = ModeFunctionType;
  MF mf1 = f1.type, mf2 = f2.type;
  long nK1 = f1.k, nK2 = f2.k;
  const long nK = std::labs(nK1);
  const double sign1 = mf1 == MF::Sin && nK1 < 0 ? -1 : 1;
  const double sign2 = mf2 == MF::Sin && nK2 < 0 ? -1 : 1;
  const double sign = sign1 * sign2;
  if (std::labs(nK1) != std::labs(nK2)) throw std::runtime_error("Not a Tridiagonal");
  if (mf1 == MF::Plus && nK1 < 0) { mf1 = MF::Minus; nK1 *= -1; }
  if (mf1 == MF::Minus && nK1 < 0) { mf1 = MF::Plus; nK1 *= -1; }
  if (mf2 == MF::Plus && nK2 < 0) { mf2 = MF::Minus; nK2 *= -1; }
  if (mf2 == MF::Minus && nK2 < 0) { mf2 = MF::Plus; nK2 *= -1; }
  const Tridiagonal id = Tridiagonal::identity(particle->dims.at(0));
  auto is = [&](MF a, MF b) { return mf1 == a && mf2 == b; };
  if (is(MF::Sin, MF::Sin)) return sign * (id - cosNKX(particle, 2 * nK)) / 2.;
  if (is(MF::Cos, MF::Cos)) return (id + cosNKX(particle, 2 * nK)) / 2.;
  if (is(MF::Sin, MF::Cos) || is(MF::Cos, MF::Sin)) return sign * sinNKX(particle, 2 * nK) / 2.;
  if (is(MF::Plus, MF::Plus) || is(MF::Minus, MF::Minus)) return id;
  if (is(MF::Plus, MF::Minus)) return expINKX(particle, -2 * nK);
  if (is(MF::Minus, MF::Plus)) return expINKX(particle, 2 * nK);
  if (is(MF::Plus, MF::Sin) || is(MF::Sin, MF::Minus)) return sign * (expINKX(particle, -2 * nK) - id) * I1 / 2.;
  if (is(MF::Plus, MF::Cos) || is(MF::Cos, MF::Minus)) return (id + expINKX(particle, -2 * nK)) / 2.;
  if (is(MF::Minus, MF::Cos) || is(MF::Cos, MF::Plus)) return (id + expINKX(particle, 2 * nK)) / 2.;
  if (!(is(MF::Minus, MF::Sin) || is(MF::Sin, MF::Plus))) throw std::logic_error("In mfComposition");
  return -sign * (expINKX(particle, 2 * nK) - id) * I1 / 2.;
}

}  // namespace particle

namespace particlecavity {

namespace {

double etaEff(double uNot, double vClass) {  // ParticleCavity.cc:16-20
  if (uNot * vClass >= 0) return gslSign(uNot) * std::sqrt(uNot * vClass);
  throw std::domain_error("Unot VClass sign discrepancy");
}

Tridiagonal plusHCOverI(const Tridiagonal& t) { return tridiagPlusHC(t) / I1; }  // Tridiagonal.h:347

void dispersive(std::vector<Tridiagonal>& res, const ElementPtr& mode, const ElementPtr& part, double uNot,
                const ModeFunction& mf) {  // ParticleCavity.cc:23-30
  if (uNot && !isComplex(mf.type))
    res.push_back(uNot * mode::nop(mode) * (mf.type == ModeFunctionType::Sin ? -1. : 1.) *
                  particle::cosNKX(part, mf.k << 1) / (2. * I1));
}

Tridiagonal interfericOneModeFN(const ElementPtr& mode, const ElementPtr& part, double etaeff, const ModeFunction& mf) {
  return etaeff * plusHCOverI(mode::aop(mode) * particle::mfNKX(part, mf));
}

Tridiagonal interfericTwoModeFN(const ElementPtr& mode, const ElementPtr& part, double etaeff, const ModeFunction& mfCav,
                                const ModeFunction& mfPart) {
  return etaeff * plusHCOverI(mode::aop(mode).dagger() * particle::mfComposition(part, mfCav, mfPart));
}

std::shared_ptr<Element> base(const ElementPtr& mode, const ElementPtr& part, double uNot, double etaeff) {
  auto e = std::make_shared<Element>();  // particlecavity::Base (ParticleCavity.cc:61-66)
  e->keyTitle = "ParticleCavity";
  e->dims = {mode->dims.at(0), part->dims.at(0)};
  e->frees = {mode, part};
  e->isHamiltonian = true;
  const double md = double(mode->dims[0]);
  e->highestFrequency = highestFrequencyOf({{uNot, md}, {etaeff, std::sqrt(md)}}, {});
  return e;
}

}  // namespace

ElementPtr orthogonal(const ElementPtr& mode, const ElementPtr& part, double uNot) {  // ParticleCavity.cc:69-80
  if (!part->pumpedParticle) throw std::invalid_argument("ParticleOrthogonalToCavity needs a pumped particle");
  const double etaeff = etaEff(uNot, part->vClass);
  auto e = base(mode, part, uNot, etaeff);
  e->hOverI.push_back(interfericOneModeFN(mode, part, etaeff, part->pumpMF));
  return e;
}

ElementPtr along(const ElementPtr& mode, const ElementPtr& part, double uNot, size_t kCav, ModeFunctionType modeCav,
                 double vClass) {  // ParticleCavity.cc:83-96 (fillT, :40-45)
  const double etaeff = etaEff(uNot, vClass);
  auto e = base(mode, part, uNot, etaeff);
  const ModeFunction mf{modeCav, long(kCav)};
  dispersive(e->hOverI, mode, part, uNot, mf);
  if (etaeff) e->hOverI.push_back(interfericOneModeFN(mode, part, etaeff, mf));
  return e;
}

ElementPtr alongPumped(const ElementPtr& mode, const ElementPtr& part, double uNot, size_t kCav,
                       ModeFunctionType modeCav) {  // ParticleCavity.cc:99-109 (fillTTwoModeFN, :48-55)
  if (!part->pumpedParticle) throw std::invalid_argument("ParticleAlongCavity: pumped particle expected");
  const double etaeff = etaEff(uNot, part->vClass);
  if (long(kCav) != std::labs(part->pumpMF.k))
    throw std::invalid_argument("ParticleAlongCavity with kCav != |kPart| is not a single Tridiagonal: not supported");
  auto e = base(mode, part, uNot, etaeff);
  const ModeFunction mf{modeCav, long(kCav)};
  dispersive(e->hOverI, mode, part, uNot, mf);
  if (etaeff) e->hOverI.push_back(interfericTwoModeFN(mode, part, etaeff, mf, part->pumpMF));
  return e;
}

}  // namespace particlecavity

namespace particletwomodes {

ElementPtr make(const ElementPtr& m0, const ElementPtr& m1, const ElementPtr& part, double uNot0, double uNot1,
                const ModeFunction& mf0, const ModeFunction& mf1, double phi) {
  if (uNot0 * uNot1 < 0) throw std::domain_error("Unots sign discrepancy");
  if (std::labs(mf0.k) != std::labs(mf1.k))
    throw std::invalid_argument("ParticleTwoModes with |k0| != |k1| is not a single Tridiagonal: not supported");
  const dcomp factor = double(gslSign(uNot0)) * std::sqrt(uNot0 * uNot1) * std::exp(I1 * phi);
  auto e = std::make_shared<Element>();
  e->keyTitle = "ParticleTwoModes";
  e->dims = {m0->dims.at(0), m1->dims.at(0), part->dims.at(0)};
  e->frees = {m0, m1, part};
  e->isHamiltonian = true;
  e->hOverI.push_back(tridiagPlusHC((factor * mode::aop(m0).dagger()) * mode::aop(m1) *
                                    particle::mfComposition(part, mf0, mf1)) /
                      I1);
  e->highestFrequency =
      highestFrequencyOf({{uNot0, std::sqrt(double(m0->dims[0]))}, {uNot1, std::sqrt(double(m1->dims[0]))}}, {});
  return e;
}

}  // namespace particletwomodes

}  // namespace cqg
