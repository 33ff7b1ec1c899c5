// Workload definitions with the command-line interface of the reference's scripts
// (CPPQEDscripts/*.cc): the same parameter names, defaults and element choices.
#include <cmath>

#include "model.hpp"

namespace cqg {

namespace {

CVec directProduct(const CVec& a, const CVec& b) {
  CVec r(a.size() * b.size());
  for (size_t i = 0; i < a.size(); ++i)
    for (size_t j = 0; j < b.size(); ++j) r[i * b.size() + j] = a[i] * b[j];
  return r;
}

void renorm(CVec& v) {
  double s = 0;
  for (auto& x : v) s += std::norm(x);
  const double n = std::sqrt(s);
  for (auto& x : v) x /= n;
}

std::string joinCommandLine(const std::string& script, const std::vector<std::string>& args) {
  std::string s = script;
  for (auto& a : args) s += " " + a;
  return s;
}

}  // namespace

std::unique_ptr<Model> makeModel(const std::string& script, const std::vector<std::string>& args) {
  ParameterTable p;
  p.parse(args);
  auto m = std::make_unique<Model>();
  m->script = script;
  m->commandLine = joinCommandLine(script, args);
  m->pe = EvolutionPars(p);
  const Picture qmp = m->pe.picture;

  if (script == "PTLA_C++QED") {  // CPPQEDscripts/PTLA_C++QED.cc
    qbit::Pars pp2la(p);
    const bool fullImpl = p.addSwitch("fullImpl", "", false);
    ElementPtr e = fullImpl ? qbit::make(pp2la, qmp) : ptla::makeSch(pp2la);
    m->sys = std::make_unique<System>(System::free(e));
    m->psi0 = qbit::init(pp2la.qbitInit);
  } else if (script == "PumpedLossyMode_C++QED") {  // PumpedLossyMode_C++QED.cc (quadrature averages)
    mode::Pars pplm(p);
    const bool quadratures = p.addSwitch("quadratures", "", true);
    ElementPtr e = mode::make(pplm, qmp, quadratures ? mode::Averaging::Quadratures : mode::Averaging::Standard);
    m->sys = std::make_unique<System>(System::free(e));
    m->psi0 = mode::init(pplm);
  } else if (script == "QbitMode_C++QED") {  // QbitMode_C++QED.cc
    qbit::Pars pplqb(p);
    mode::Pars pplm(p);
    const dcomp g = p.add<dcomp>("g", "", 1.);  // jaynescummings::Pars (JaynesCummings.cc:10-12)
    ElementPtr q = qbit::make(pplqb, qmp), md = mode::make(pplm, qmp);
    m->sys = std::make_unique<System>(System::binary(jaynescummings::make(q, md, g)));
    m->psi0 = directProduct(qbit::init(pplqb.qbitInit), mode::init(pplm));
  } else if (script == "Optomechanics") {  // Optomechanics.cc: CM_NX coupling, u -> -sqrt(2) u
    mode::Pars pA(p, "Opt"), pB(p, "Mech");
    pB.eta = 0;
    const double u = p.add<double>("u", "", 1.);
    ElementPtr a = mode::make(pA, qmp, mode::Averaging::Standard), b = mode::make(pB, qmp, mode::Averaging::Standard);
    m->sys = std::make_unique<System>(
        System::binary(coupledmodes::make(a, b, coupledmodes::Kind::NX, dcomp(-std::sqrt(2.) * u, 0.))));
    m->psi0 = directProduct(mode::init(pA), mode::init(pB));
    renorm(m->psi0);
  } else if (script == "1particle1mode") {  // CPPQEDscripts/1particle1mode.cc
    const int conf = p.add<int>("1p1mconf", "", 1);
    mode::Pars pplm(p);
    particle::ParsPumped ppp(p);
    // particlecavity::ParsAlong (ParsParticleCavity.cc:9-15)
    const double uNot = p.add<double>("Unot", "", -1.);
    const size_t kCav = p.add<size_t>("kCav", "", 1);
    const ModeFunctionType modeCav = p.add<ModeFunctionType>("modeCav", "", ModeFunctionType::Sin);
    const dcomp superposition = p.add<dcomp>("superposition", "", 0.);
    if (conf != 1) pplm.delta -= uNot / (isComplex(modeCav) ? 1. : 2.);
    ElementPtr md = mode::make(pplm, qmp);
    ElementPtr part = particle::make(ppp, qmp), pumped = particle::makePumped(ppp, qmp);
    ElementPtr ia;
    switch (conf) {
      case 1:  // pumped particle moving orthogonal to the (pumped) cavity
        ia = particlecavity::orthogonal(md, pumped, uNot);
        break;
      case 2:  // particle along the cavity, scattering from the transverse pump
        if (!std::abs(pplm.eta) && !ppp.vClass) throw std::invalid_argument("No driving in the system!");
        if (!ppp.init.sig) throw std::invalid_argument("No initial spread specified!");
        ia = particlecavity::along(md, part, uNot, kCav, modeCav, ppp.vClass);
        break;
      case 3:  // pumped particle along the cavity, pump along the cavity
        ia = particlecavity::alongPumped(md, pumped, uNot, kCav, modeCav);
        break;
      case 4:  // as 3, without scattering from the pump into the cavity
        ia = particlecavity::along(md, pumped, uNot, kCav, modeCav, 0.);
        break;
      default:
        throw std::invalid_argument("Configuration not recognized!");
    }
    const particle::Spatial space(ppp.fin);
    CVec psiPart;
    if (std::abs(superposition) > 0) {
      const CVec h0 = particle::hoState(0, ppp.init, space), h2 = particle::hoState(2, ppp.init, space);
      psiPart.resize(h0.size());
      for (size_t i = 0; i < h0.size(); ++i)
        psiPart[i] = std::sqrt(1 - std::norm(superposition)) * h0[i] + superposition * h2[i];
    } else {
      psiPart = particle::init(ppp);
    }
    m->sys = std::make_unique<System>(System::binary(ia));
    m->psi0 = directProduct(mode::init(pplm), psiPart);
    renorm(m->psi0);
  } else if (script == "Ring") {  // CPPQEDscripts/Ring.cc
    particle::Pars pp(p);
    mode::Pars pmP(p, "P"), pmM(p, "M");
    const double uNotP = p.add<double>("Unot", "P", -1.), uNotM = p.add<double>("Unot", "M", -1.);
    const size_t kCavP = p.add<size_t>("kCav", "P", 1), kCavM = p.add<size_t>("kCav", "M", 1);
    p.add<ModeFunctionType>("modeCav", "P", ModeFunctionType::Sin);  // overridden by the script
    p.add<ModeFunctionType>("modeCav", "M", ModeFunctionType::Sin);
    const ModeFunctionType mfP = ModeFunctionType::Plus, mfM = ModeFunctionType::Minus;
    pmP.delta -= uNotP / (isComplex(mfP) ? 1. : 2.);
    pmM.delta -= uNotM / (isComplex(mfM) ? 1. : 2.);
    ElementPtr part = particle::make(pp, qmp), plus = mode::make(pmP, qmp), minus = mode::make(pmM, qmp);
    std::vector<Act> acts = {
        {{1, 0}, particlecavity::along(plus, part, uNotP, kCavP, mfP, 0.)},
        {{2, 0}, particlecavity::along(minus, part, uNotM, kCavM, mfM, 0.)},
        {{1, 2, 0},
         particletwomodes::make(plus, minus, part, uNotP, uNotM, ModeFunction{mfP, long(kCavP)},
                                ModeFunction{mfM, long(kCavM)})}};
    m->sys = std::make_unique<System>(System::composite({part, plus, minus}, acts));
    m->psi0 = directProduct(directProduct(particle::init(pp), mode::init(pmP)), mode::init(pmM));
  } else if (script == "QbitChain") {
    // Synthetic spin chain: nQbit lossy Qbits with nearest-neighbour CM_XX_RWA couplings
    // (composite of ModeBase qubits, the coupling of CoupledModes.cc:33-38); the first
    // qubit is driven.  No reference script exists for it.
    const int nQbit = p.add<int>("nQbit", "", 6);
    qbit::Pars base(p);
    const dcomp u = p.add<dcomp>("u", "", 1.);
    if (nQbit < 2 || nQbit > CQG_MAX_RANK) throw std::invalid_argument("nQbit out of range");
    std::vector<ElementPtr> frees;
    for (int i = 0; i < nQbit; ++i) {
      qbit::Pars qi = base;
      if (i) qi.eta = 0;
      frees.push_back(qbit::make(qi, qmp));
    }
    std::vector<Act> acts;
    for (int i = 0; i + 1 < nQbit; ++i)
      acts.push_back({{i, i + 1}, coupledmodes::make(frees[i], frees[i + 1], coupledmodes::Kind::XX_RWA, u)});
    m->sys = std::make_unique<System>(System::composite(frees, acts));
    CVec psi = qbit::init(base.qbitInit);
    for (int i = 1; i < nQbit; ++i) psi = directProduct(psi, qbit::init(0.));
    m->psi0 = psi;
  } else {
    throw std::invalid_argument("unknown script \"" + script + "\"");
  }
  p.checkAllKnown();
  if (m->psi0.size() != m->sys->totalDimension()) throw std::invalid_argument("initial state dimension mismatch");
  return m;
}

}  // namespace cqg
