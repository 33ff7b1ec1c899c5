// Batched H/i application: the drop-in for structure::Hamiltonian::addContribution
// (Hamiltonian.h:38-43), i.e. for the reference's slice-wise Tridiagonal::apply
// (Tridiagonal.tcc:220-263) over a composite system, on many states at once:
//   dpsi_i += (H/i)(tau) psi_i      for every state i,  tau = t - t0.
// The operator is the system's row-gather table (fused diagonal + S off-diagonal
// slots per row, see lowering.hpp).  The kernel streams the states element by element,
// so psi and dpsi are read and written with coalesced 16-byte accesses; the banded
// gathers hit lines the same warp has just brought in, and the tables (a few KB) stay
// in L1.  It is bound by HBM
// bandwidth: 48 bytes per element (read psi, read and write dpsi).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../host/errors.hpp"
#include "cqg.h"
#include "mcwf_kernel.cuh"

namespace cqg {
namespace dev {
const SysDev* systemDescriptor(const cqg_system* sys);
int systemDevice(const cqg_system* sys);
}  // namespace dev
}  // namespace cqg

namespace {

using cqg::fail;
using cqg::dev::SysDev;

// Element-parallel: the flattened [n_states][D] arrays are walked with a grid stride,
// four independent elements per thread in flight (32-bit indices; the entry point
// checks n_states * D < 2^31), so psi and dpsi move with coalesced 16-byte accesses.
template <int S>
__device__ __forceinline__ double2 applyRow(const SysDev& sys, const double2* __restrict__ x, int r, double2 acc,
                                            double tau) {
  const int D = sys.D;
  acc = cqg::dev::cfma(__ldg(&sys.diagD[r]), __ldg(&x[r]), acc);
  const int nS = S >= 0 ? S : sys.S;
#pragma unroll
  for (int s = 0; s < (S >= 0 ? S : 8); ++s) {
    if (S < 0 && s >= nS) break;
    double2 c = __ldg(&sys.valD[s * D + r]);
    if (sys.freq) {
      const double2 f = __ldg(&sys.freq[s * D + r]);
      if (f.x != 0. || f.y != 0.) {
        const double2 ph = cqg::dev::cexpScaled(tau, f);
        c = make_double2(c.x * ph.x - c.y * ph.y, c.x * ph.y + c.y * ph.x);
      }
    }
    acc = cqg::dev::cfma(c, __ldg(&x[__ldg(&sys.col[s * D + r])]), acc);
  }
  return acc;
}

template <int S>
__global__ void __launch_bounds__(256) applyKernel(SysDev sys, const double2* __restrict__ psi,
                                                   double2* __restrict__ dpsi, unsigned total, double tau) {
  const unsigned D = unsigned(sys.D);
  const unsigned stride = gridDim.x * blockDim.x;
  unsigned g = blockIdx.x * blockDim.x + threadIdx.x;
  for (; g + 3 * stride < total; g += 4 * stride) {
    double2 acc[4];
    unsigned gg[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      gg[u] = g + u * stride;
      acc[u] = dpsi[gg[u]];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const unsigned i = gg[u] / D, r = gg[u] - i * D;
      acc[u] = applyRow<S>(sys, psi + size_t(i) * D, int(r), acc[u], tau);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) dpsi[gg[u]] = acc[u];
  }
  for (; g < total; g += stride) {
    const unsigned i = g / D, r = g - i * D;
    dpsi[g] = applyRow<S>(sys, psi + size_t(i) * D, int(r), dpsi[g], tau);
  }
}

template <int S>
cudaError_t launch(const SysDev& sd, const double2* psi, double2* dpsi, long long nStates, double tau,
                   cudaStream_t st, int nSM) {
  const long long total = nStates * sd.D;
  const long long blocksWanted = (total + 1023) / 1024;
  const int blocks = int(std::max<long long>(1, std::min<long long>(blocksWanted, (long long)nSM * 8)));
  applyKernel<S><<<blocks, 256, 0, st>>>(sd, psi, dpsi, unsigned(total), tau);
  return cudaGetLastError();
}

}  // namespace

extern "C" int cqg_system_apply_hamiltonian(const cqg_system* sys, const cqg_complex* psi, cqg_complex* dpsi,
                                            int64_t n_states, double tau, void* stream) {
  if (!sys || !psi || !dpsi || n_states < 1)
    return fail(CQG_E_INVALID, "cqg_system_apply_hamiltonian: null pointer or no states");
  const SysDev* sd = cqg::dev::systemDescriptor(sys);
  if (sd->S > 8) return fail(CQG_E_UNSUPPORTED, "cqg_system_apply_hamiltonian: more than 8 off-diagonal slots per row");
  if (n_states > ((1ll << 31) - 1) / sd->D)
    return fail(CQG_E_INVALID, "cqg_system_apply_hamiltonian: n_states * D must stay below 2^31 per call");
  int device = 0, nSM = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, device);
  if (err != cudaSuccess) return fail(CQG_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
  if (device != cqg::dev::systemDevice(sys))
    return fail(CQG_E_INVALID, "cqg_system_apply_hamiltonian: the current device is not the system's device");
  const double2* p = reinterpret_cast<const double2*>(psi);
  double2* q = reinterpret_cast<double2*>(dpsi);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (sd->S) {
    case 0: err = launch<0>(*sd, p, q, n_states, tau, st, nSM); break;
    case 1: err = launch<1>(*sd, p, q, n_states, tau, st, nSM); break;
    case 2: err = launch<2>(*sd, p, q, n_states, tau, st, nSM); break;
    case 3: err = launch<3>(*sd, p, q, n_states, tau, st, nSM); break;
    case 4: err = launch<4>(*sd, p, q, n_states, tau, st, nSM); break;
    default: err = launch<-1>(*sd, p, q, n_states, tau, st, nSM); break;
  }
  if (err != cudaSuccess) return fail(CQG_E_CUDA, std::string("apply launch: ") + cudaGetErrorString(err));
  return CQG_OK;
}
