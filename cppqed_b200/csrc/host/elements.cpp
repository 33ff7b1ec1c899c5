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

}  // namespace cqg
