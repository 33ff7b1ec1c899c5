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


}  // namespace cqg
