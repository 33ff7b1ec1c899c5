// Composite quantum systems and their lowering to the plain cqg_system_desc.
//
// System::free / binary / composite mirror structure::Free, binary::make
// (BinarySystem.cc:323-333) and composite::make (Composite.h:363-364): they fix the
// order in which Hamiltonian terms are applied (frees in axis order, then
// interactions), the ordinal order of jumps, and the concatenation order of
// averages — all of which the device kernels and the CPU oracle reproduce.
#pragma once

#include <deque>
#include <memory>
#include <string>
#include <vector>

#include "cqg.h"
#include "elements.hpp"

namespace cqg {

struct Act {  // composite::_<i,j,...>(interaction) (Act.h:27-47)
  std::vector<int> axes;
  ElementPtr ia;
};

class System {
 public:
  static System free(const ElementPtr& f);
  static System binary(const ElementPtr& ia);
  static System composite(const std::vector<ElementPtr>& frees, const std::vector<Act>& acts);

  const std::vector<size_t>& dims() const { return dims_; }
  size_t totalDimension() const;
  int nAvr() const { return nAvr_; }
  bool isHamiltonian() const;
  bool isLiouvillean() const;
  bool isExact() const;
  double highestFrequency() const { return highestFrequency_; }
  const std::vector<std::string>& avLabels() const { return labels_; }

  // Applies every element's process_v on its own column range (BinarySystem.cc:73-98).
  void process(double* averages) const;

  // The system's part of the "Key to data" block (LiouvilleanAveragedCommon.h:82-93,
  // KeyPrinter): per averaging element its title, then its columns numbered from
  // firstColumn (" 3. rho00"), one line each.
  std::string keyText(int firstColumn) const;
  // The system's parameter block of a trajectory file's header (Structure.h:178-186,
  // streamParameters): every element's description, the dimension, the system's
  // characteristics and the decay channels in ordinal order, one line each.
  std::string parametersText() const;

  // The descriptor view; pointers stay valid for the lifetime of this object.
  const cqg_system_desc& desc() const { return desc_; }

  System(const System&) = delete;
  System& operator=(const System&) = delete;
  System(System&&) = default;
  System& operator=(System&&) = default;

 private:
  System() = default;
  void lower();
  struct Placed {
    ElementPtr e;
    std::vector<int> axes;
    int colOffset;
  };
  std::vector<Placed> placed_;  // frees (one per axis) then acts
  bool binary_ = false;         // binary::make: its key opens with "Binary system"
  std::vector<size_t> dims_;
  int nAvr_ = 0;
  double highestFrequency_ = 0;
  std::vector<std::string> labels_;

  // storage behind desc_
  std::deque<std::vector<cqg_complex>> arrays_;
  std::deque<std::vector<const cqg_complex*>> ptrArrays_;
  std::deque<DVec> weights_;
  std::vector<cqg_tridiagonal> ham_;
  std::vector<cqg_jump> jumps_;
  std::vector<cqg_observable> obs_;
  cqg_system_desc desc_{};

  cqg_tridiagonal place(const Tridiagonal& t, const std::vector<int>& axes);
  const cqg_complex* store(const CVec& v);
};

// evolution::Pars (Evolution_.h:34-46) + trajectory::Pars (Trajectory.h:77-114) +
// ode_engine::Pars (ODE.h:41-63) + randomutils::Pars<pcg64> (Random.h:137-147) +
// ParsStochastic (StochasticTrajectory.h:21-39) + mcwf::Pars (MCWF_Trajectory.h:28-47)
struct EvolutionPars {
  double T = 1., Dt = .1;
  int dc = 10;
  long NDt = 0;
  unsigned sdf = 0;
  int precision = 6;
  double epsRel = 1e-6, epsAbs = 1e-12;
  int logLevel = 0;
  unsigned long seed = 1001, prngStream = 1;
  bool noise = true;
  size_t nTraj = 500;
  double dpLimit = .01, overshootTolerance = 10.;
  size_t nBins = 0, nJumpsPerBin = 50;
  std::string evol = "single";
  Picture picture = Picture::IP;
  // engine-only extensions (no reference counterpart)
  std::string prec = "fp64";
  std::string rng = "pcg64";
  EvolutionPars() = default;
  EvolutionPars(ParameterTable& p);
};

// A script: the system, its initial state and the run parameters, built from a
// reference-style command line (CPPQEDscripts/*.cc).
struct Model {
  std::string script;
  std::unique_ptr<System> sys;
  CVec psi0;
  EvolutionPars pe;
  std::string commandLine;
};

// Known scripts: "PTLA_C++QED", "PumpedLossyMode_C++QED", "QbitMode_C++QED",
// "JaynesCummingsChain" (synthetic), "Optomechanics", "1particle1mode", "Ring".
std::unique_ptr<Model> makeModel(const std::string& script, const std::vector<std::string>& args);

}  // namespace cqg
