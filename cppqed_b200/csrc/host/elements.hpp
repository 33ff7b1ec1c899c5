// Host-side element library: free systems and interactions described the way the
// reference's CPPQEDelements build them (Mode, Qbit, PumpedTwoLevelAtom, Particle,
// JaynesCummings, ParticleCavity, CoupledModes), but producing plain data — banded
// H/i terms, interaction-picture exponents, jump operators with closed-form rate
// weights, and linear observables — instead of virtual callbacks.  The data is
// lowered to the device by cqg_system_create and read by the CPU oracle.
#pragma once

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "pars.hpp"
#include "tridiagonal.hpp"

namespace cqg {

enum class Picture { IP, UIP, Sch };  // QM_Picture (high/QM_Picture.h), default IP
Picture parsePicture(const std::string& s);

enum class ModeFunctionType { Sin, Cos, Plus, Minus };  // ModeFunction.h
std::istream& operator>>(std::istream& is, ModeFunctionType& mf);
inline bool isComplex(ModeFunctionType mf) { return mf == ModeFunctionType::Plus || mf == ModeFunctionType::Minus; }
struct ModeFunction {
  ModeFunctionType type = ModeFunctionType::Sin;
  long k = 1;
};

struct ElementJump {
  Tridiagonal J;     // on the element's local axes
  int rateAxis = 0;  // local axis of the closed-form weights
  DVec weights;      // empty: rate = ||J psi||^2 (special jump)
  std::string label;
};

struct ElementObservable {
  Tridiagonal op;  // banded (unused when dense is non-empty)
  CVec dense;      // dense N x N on `denseAxis`
  int denseAxis = 0;
  int colRe = -1, colIm = -1;  // local average columns
  DVec fourierWeights;  // non-empty: dense = F^+ diag(w) F with F the k -> x transform
};

struct Element;
using ElementPtr = std::shared_ptr<const Element>;

struct Element {
  std::string keyTitle;
  std::vector<size_t> dims;        // one entry for a free, one per coupled free for an interaction
  std::vector<ElementPtr> frees;   // interactions only

  bool isHamiltonian = false;      // the class derives from structure::Hamiltonian
  std::vector<Tridiagonal> hOverI;
  std::vector<CVec> exact;         // per local axis lambda[n] (U = exp(lambda tau)), empty = none
  bool isExact() const {
    for (auto& e : exact)
      if (!e.empty()) return true;
    return false;
  }

  bool isLiouvillean = false;
  std::vector<ElementJump> jumps;

  std::vector<std::string> avLabels;
  std::vector<ElementObservable> obs;
  std::function<void(double*)> process;  // Averaged::process_v on the element's columns

  double highestFrequency = 0;  // DynamicsBase::highestFrequency (DynamicsBase.cc:49-66)
  std::string parsStream;

  // mode::Exact information, needed when other elements build ladder operators
  // furnished with frequencies (mode::aop(Ptr), Mode.cc:285-292)
  bool modeExact = false;
  dcomp zI = 0;
  double omegaKerr = 0;
  // particle::Exact information (particle::expINKX(Ptr), Particle.cc:206-213)
  bool particleExact = false;
  double omrec = 0;
  size_t fin = 0;
  // PumpedParticleBase (Particle_.h:199-214): pump strength and mode function
  bool pumpedParticle = false;
  double vClass = 0;
  ModeFunction pumpMF;
};

// ---- helpers shared by elements ------------------------------------------
double highestFrequencyOf(const std::vector<std::pair<double, double>>& realFreqs,
                          const std::vector<std::pair<dcomp, double>>& complexFreqs);

// ---- Mode ------------------------------------------------------------------
namespace mode {
struct Pars {  // ParsMode.cc:9-37 (mode::ParsPumpedLossy)
  size_t cutoff = 10, minitFock = 0, streamLevel = 0;
  dcomp minit = 0, eta = 0;
  double delta = -10, omegaKerr = 0, omegaKerrAlter = 0, kappa = 10, nTh = 0;
  Pars() = default;
  Pars(ParameterTable& p, const std::string& mod = "");
};
enum class Averaging { Standard, Quadratures, None };
ElementPtr make(const Pars& p, Picture qmp, Averaging av = Averaging::Standard);
CVec mainDiagonal(dcomp z, double omegaKerr, size_t dim);  // Mode.cc:53-61
Tridiagonal aop(size_t dim);                                 // Mode.cc:270-276
Tridiagonal aop(const ElementPtr& mode);                     // furnished if mode::Exact
Tridiagonal nop(const ElementPtr& mode);
CVec coherent(dcomp alpha, size_t dim);  // Mode.cc:321-324
CVec fock(size_t n, size_t dim, double phase = 0);
CVec init(const Pars& p);
}  // namespace mode

// ---- Qbit ------------------------------------------------------------------
namespace qbit {
struct Pars {  // ParsQbit.h (ParsPumpedLossyPhaseNoise)
  dcomp qbitInit = 0, eta = 0;
  double delta = -10, gamma = 10, gamma_parallel = 0;
  Pars() = default;
  Pars(ParameterTable& p, const std::string& mod = "");
};
ElementPtr make(const Pars& p, Picture qmp);  // Qbit.cc:217-266
Tridiagonal sigmaop(const ElementPtr& qbit);  // = mode::aop(qbit)
CVec init(dcomp psi1);                        // Qbit.cc:275-280
}  // namespace qbit

// ---- PumpedTwoLevelAtomSch (PumpedTwoLevelAtom.{h,cc}) --------------------------
namespace ptla {
ElementPtr makeSch(const qbit::Pars& p);
}

// ---- JaynesCummings (JaynesCummings_.h:54-97) ------------------------------------
namespace jaynescummings {
ElementPtr make(const ElementPtr& qbit, const ElementPtr& mode, dcomp g);
}

// ---- CoupledModes (CoupledModes.{h,cc}) ------------------------------------------
namespace coupledmodes {
enum class Kind { NX, XX, XX_RWA };  // coupledmodes::Coupling (CoupledModes.h)
ElementPtr make(const ElementPtr& m0, const ElementPtr& m1, Kind kind, dcomp u);
}

// ---- Particle (Particle.{h,cc}, Particle_.h, ParsParticle.cc) ---------------------

namespace particle {
struct InitialCondition {  // ParticleInitialCondition.h: (x0, k0, sig, isInK)
  double x0 = -.5, k0 = 0, sig = .1;
  bool inK = false;
};
std::istream& operator>>(std::istream& is, InitialCondition& ic);  // "(x0,k0,sig,isInK)"

struct Pars {  // ParsParticle.cc:8-14
  double omrec = 1;
  size_t fin = 6;
  InitialCondition init;
  int hoInitn = -1;
  Pars() = default;
  Pars(ParameterTable& p, const std::string& mod = "");
};
struct ParsPumped : Pars {  // ParsParticle.cc:17-23
  double vClass = -10;
  size_t kPart = 1;
  ModeFunctionType modePart = ModeFunctionType::Sin;
  ParsPumped() = default;
  ParsPumped(ParameterTable& p, const std::string& mod = "");
};

// Spatial (Particle.cc:257-272): x_i = deltaX i - xMax, k_i = deltaK i - kMax
struct Spatial {
  size_t fin;
  double xMax, deltaX, kMax, deltaK;
  explicit Spatial(size_t fin, double deltaK = 1);
  size_t dim() const { return size_t(1) << fin; }
  double x(size_t i) const { return deltaX * double(i) - xMax; }
  double k(size_t i) const { return deltaK * double(i) - kMax; }
};

enum class Direction { XK, KX };  // fft::Direction: forward (x -> k), backward
// quantumdata::ffTransform of a vector (LazyDensityOperatorFFT.cc:12-31): radix-2 DFT
// (sign -1 for XK, +1 for KX, unnormalised), halves swapped with factor N^-1/2, odd
// entries negated.
void ffTransform(CVec& psi, Direction dir);

ElementPtr make(const Pars& p, Picture qmp);              // Particle / ParticleSch
ElementPtr makePumped(const ParsPumped& p, Picture qmp);  // PumpedParticle / PumpedParticleSch
CVec wavePacket(const InitialCondition& init, const Spatial& space, bool kFlag = true);
CVec hoState(int n, const InitialCondition& init, const Spatial& space, bool kFlag = true);
CVec init(const Pars& p);
CVec init(const ParsPumped& p);

// operators on a particle element, furnished with frequencies in the interaction picture
Tridiagonal expINKX(const ElementPtr& particle, long nK);
Tridiagonal cosNKX(const ElementPtr& particle, long nK);
Tridiagonal sinNKX(const ElementPtr& particle, long nK);
Tridiagonal mfNKX(const ElementPtr& particle, const ModeFunction& mf);
Tridiagonal mfComposition(const ElementPtr& particle, const ModeFunction& mf1, const ModeFunction& mf2);
}  // namespace particle

// ---- ParticleCavity (ParticleCavity.cc), ParticleTwoModes (ParticleTwoModes.cc) ----------
namespace particlecavity {
// ParticleOrthogonalToCavity(mode, pumpedParticle, Unot)
ElementPtr orthogonal(const ElementPtr& mode, const ElementPtr& pumpedParticle, double uNot);
// ParticleAlongCavity with a particle that is not pumped along the cavity (etaeff from
// Unot and vClass, 0 for none)
ElementPtr along(const ElementPtr& mode, const ElementPtr& particle, double uNot, size_t kCav, ModeFunctionType modeCav,
                 double vClass);
// ParticleAlongCavity with a pumped particle (the two-mode-function Hamiltonian; only the
// case kCav == |kPart|, a single Tridiagonal, is supported)
ElementPtr alongPumped(const ElementPtr& mode, const ElementPtr& pumpedParticle, double uNot, size_t kCav,
                       ModeFunctionType modeCav);
}  // namespace particlecavity
namespace particletwomodes {
// ParticleTwoModes (ParticleTwoModes.cc:17-33); only |k0| == |k1| (a single Tridiagonal)
ElementPtr make(const ElementPtr& mode0, const ElementPtr& mode1, const ElementPtr& particle, double uNot0,
                double uNot1, const ModeFunction& mf0, const ModeFunction& mf1, double phi = 0);
}

}  // namespace cqg
