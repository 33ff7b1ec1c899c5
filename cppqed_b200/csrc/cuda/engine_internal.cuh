// Host-side pieces shared by the ensemble entry points (api.cu) and the request server
// (server.cu): the device-resident system, kernel groups and their launches, the
// initial-step rule of the MCWF_Trajectory constructor, CUDA error plumbing.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../host/errors.hpp"
#include "../host/lowering.hpp"
#include "cqg.h"
#include "mcwf_block.cuh"
#include "mcwf_kernel.cuh"

struct cqg_system {
  cqg::LoweredSystem L;
  int device = 0;
  void* dmem = nullptr;
  cqg::dev::SysDev sd{};
  ~cqg_system() {
    if (dmem) cudaFree(dmem);
  }
};

namespace cqg {
namespace engine {

using dcomp = std::complex<double>;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Recycled device blocks (api.cu): ensemble buffers come from and go back to a per-device
// cache instead of cudaMalloc / cudaFree.  deviceAlloc allocates on the current device;
// deviceRelease takes the device the block lives on and the size it was requested with.
void* deviceAlloc(size_t bytes, const char* what);
void deviceRelease(int device, void* p, size_t bytes);

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename F>
int guardedCuda(F&& f) {
  return cqg::guarded([&]() -> int {
    try {
      return f();
    } catch (const CudaError& e) {
      return cqg::fail(CQG_E_CUDA, e.what());
    }
  });
}

// the warp kernel holds up to 4 rows per lane
constexpr int kWarpKernelMaxD = 128;
// kernel groups: warp kernel with E = 1..4 rows per lane, and the block kernel
constexpr int kMaxGroups = 5;

// the warp kernel keeps up to 8 off-diagonal slots per row in registers; the CTA kernel
// walks any number up to kMaxSlots
constexpr int kWarpKernelMaxS = 8;
constexpr int kMaxSlots = 64;

// Group key of a trajectory of dimension D with S off-diagonal slots per row: rows per lane
// 1..4 (warp kernel), or kMaxGroups for the CTA-per-trajectory kernel.
inline int groupKey(int64_t D, int S) {
  return D <= kWarpKernelMaxD && S <= kWarpKernelMaxS ? int((D + 31) / 32) : kMaxGroups;
}

// One persistent launch per run call: the trajectories of one kernel shape, a segment of
// an order array, on their own stream.
struct KernelGroup {
  int kind = 0;     // 0: warp per trajectory, 1: CTA per trajectory
  int E = 0;        // warp kind: rows per lane
  int smax = 0;     // off-diagonal slots per row (max over the group's systems)
  int Dmax = 0;
  bool anyFreq = false;  // some system of the group has interaction-picture frequencies
  bool smemVectors = false;  // CTA kind: stage derivatives in shared memory instead of scratch
  bool highOccupancy = false;  // warp kind: the instance compiled for more resident CTAs
  bool phaseTable = true;    // interaction picture: phases from the systems' tables of
                             // distinct frequencies where they have one
  int phaseElems = 0;        // CTA kind: shared-memory phase table capacity (max over systems)
  int threads = 0;  // CTA size
  int64_t first = 0, count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  void* scratch = nullptr;  // block kind: per-CTA stage vectors
  size_t scratchBytes = 0;
};

inline int defaultThreads(const KernelGroup& g) { return g.kind ? 256 : 128; }

// Dynamic shared memory of the CTA kernel: two stage vectors of Dmax elements, the reduction
// scratch and broadcast words, the interaction-picture phase table of phaseElems double2,
// and with shared-memory vectors the kBlockVectors stage derivatives and second state buffer
// of ceil32(Dmax) elements each.
inline size_t blockSmemBytes(int Dmax, size_t elemBytes, bool vectors, int phaseElems) {
  const size_t base = 2 * size_t(Dmax) * elemBytes + 32 * (dev::MAX_JUMPS + 1) * sizeof(double) + 64 +
                      size_t(phaseElems) * sizeof(double2);
  return base + (vectors ? size_t(dev::kBlockVectors) * size_t((Dmax + 31) / 32 * 32) * elemBytes : 0);
}
// Phase-table capacity a CTA-kernel group needs for one of its systems
inline int blockPhaseElems(const dev::SysDev& sd) { return sd.hasFreq && sd.fIdx ? sd.nFD : 0; }

// One persistent launch of group g over td on stream st (ra.order / nTasks / queue set by
// the caller); allocates or grows the group's block-kernel scratch.
void launchGroup(bool fp64, size_t elemBytes, const dev::TrajDev& td, KernelGroup& g, dev::RunArgs ra, int nSM,
                 cudaStream_t st);

// rates of a state on the host (the MCWF_Trajectory constructor, MCWF_Trajectory.h:114-117)
std::vector<double> hostRates(const LoweredSystem& L, const std::vector<dcomp>& psi);

// Initial dtTry of a trajectory: dt_init or 1/(10 highestFrequency) (Trajectory.h:126),
// then the constructor's manageTimeStep (MCWF_Trajectory.h:114-117).  *overshot is set
// when the initial step overshoots dpLimit (the logger's overshoot counter).
double initialDtTry(const cqg_system& s, const std::vector<dcomp>& psi, const cqg_mcwf_pars& p, bool* overshot);

// dpsi_i += (H/i)(tau) psi_i for nStates contiguous states of sd.D elements (16-byte
// aligned), queued on st: the batched Hamiltonian::addContribution of apply.cu
cudaError_t applyHamiltonian(const dev::SysDev& sd, const double2* psi, double2* dpsi, long long nStates, double tau,
                             cudaStream_t st, int nSM);

}  // namespace engine
}  // namespace cqg
