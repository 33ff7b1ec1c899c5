// Ensemble sums of the linear averages of caller-owned device states, without any
// device allocation.
//
// The ensemble path keeps one slot of averages per trajectory in memory the library
// allocates, then reduces the slots in a fixed order.  Some callers cannot allocate:
// their device memory belongs to another allocator (a framework's caching pool, or a
// serving runtime that reserved the GPU's memory up front), or they run where
// cudaMalloc is not allowed or would synchronise the device.  For them this file keeps
// the per-state slots in a fixed, file-scope device array instead.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>

#include "../host/errors.hpp"
#include "cqg.h"
#include "mcwf_kernel.cuh"

// cqg_system's layout lives in api.cu; only the device descriptor is needed here.
namespace cqg {
namespace dev {
const SysDev* systemDescriptor(const cqg_system* sys);
int systemDevice(const cqg_system* sys);
}  // namespace dev
}  // namespace cqg

namespace {

using cqg::fail;
using cqg::dev::SysDev;

// Per-state slots: states x averages must fit (2 MiB of doubles).  Every GPU that loads
// the library holds this array until the process exits.
constexpr long long kScratchDoubles = 1ll << 18;
static __device__ __align__(256) double gNoallocScratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex gSetupMutex;
// Per device: the array's device address and the SM count, resolved at the first call on the
// device with that device current.  A cudaDeviceReset would reload the module and move the
// array, so the library must not be used across a device reset.
struct DeviceSetup {
  double* scratch = nullptr;
  int sms = 0;
};
DeviceSetup gSetup[kMaxDevices];

int setupFor(int device, DeviceSetup* out) {
  if (device < 0 || device >= kMaxDevices) return fail(CQG_E_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(gSetupMutex);
  DeviceSetup& d = gSetup[device];
  if (!d.scratch) {
    void* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, gNoallocScratch);
    if (err != cudaSuccess)
      return fail(CQG_E_CUDA, std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(err));
    int sms = 0;
    err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err != cudaSuccess || sms < 1)
      return fail(CQG_E_CUDA, std::string("cudaDeviceGetAttribute(SM count): ") + cudaGetErrorString(err));
    d.sms = sms;
    d.scratch = static_cast<double*>(p);
  }
  *out = d;
  return CQG_OK;
}

// One warp per state: every column of the state's slot is written (zero where no
// observable contributes), so no slot keeps a value from an earlier call.
__global__ void __launch_bounds__(128) stateAveragesKernel(SysDev sys, const double2* __restrict__ psi,
                                                           long long nStates, int nAvr, double* __restrict__ slots) {
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nWarps = (gridDim.x * (long long)blockDim.x) >> 5;
  const int D = sys.D;
  for (long long i = warp; i < nStates; i += nWarps) {
    const double2* x = psi + i * D;
    double* slot = slots + i * nAvr;
    for (int c = lane; c < nAvr; c += 32) slot[c] = 0.;
    __syncwarp();
    for (int k = 0; k < sys.nObs; ++k) {
      const double2* ov = sys.oval + size_t(k) * sys.SO * D;
      const int* oc = sys.ocol + size_t(k) * sys.SO * D;
      const int nSk = sys.oS[k];  // this observable's slots; the rest of SO is zero padding
      double re = 0., im = 0.;
      for (int r = lane; r < D; r += 32) {
        double2 acc = make_double2(0., 0.);
        for (int s = 0; s < nSk; ++s) acc = cqg::dev::cfma(ov[s * D + r], x[oc[s * D + r]], acc);
        const double2 xr = x[r];
        re += xr.x * acc.x + xr.y * acc.y;  // conj(psi_r) (O psi)_r
        im += xr.x * acc.y - xr.y * acc.x;
      }
      re = cqg::dev::warpSum(re);
      im = cqg::dev::warpSum(im);
      if (lane == 0) {
        const int cr = sys.oRe[k], ci = sys.oIm[k];
        if (cr >= 0) slot[cr] = re;
        if (ci >= 0) slot[ci] = im;
      }
    }
  }
}

// One block per column: fixed-order strided partial sums, then a fixed tree.
__global__ void sumSlotsKernel(const double* __restrict__ slots, long long nStates, int nAvr,
                               double* __restrict__ sums) {
  const int c = blockIdx.x;
  __shared__ double part[256];
  double acc = 0.;
  for (long long i = threadIdx.x; i < nStates; i += blockDim.x) acc += slots[i * nAvr + c];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[c] = part[0];
}

}  // namespace

extern "C" int cqg_system_averages_noalloc(const cqg_system* sys, const cqg_complex* psi, int64_t n_states,
                                           double* sums, void* stream) {
  if (!sys || !psi || !sums || n_states < 1)
    return fail(CQG_E_INVALID, "cqg_system_averages_noalloc: null pointer or no states");
  // the kernel reads states as 16-byte complex vectors and writes doubles
  if (reinterpret_cast<uintptr_t>(psi) % 16 != 0)
    return fail(CQG_E_INVALID, "cqg_system_averages_noalloc: psi must be 16-byte aligned");
  if (reinterpret_cast<uintptr_t>(sums) % 8 != 0)
    return fail(CQG_E_INVALID, "cqg_system_averages_noalloc: sums must be 8-byte aligned");
  const SysDev* sd = cqg::dev::systemDescriptor(sys);
  const int nAvr = sd->nAvr;
  if (nAvr < 1) return fail(CQG_E_INVALID, "cqg_system_averages_noalloc: the system has no averages");
  if (n_states > kScratchDoubles / nAvr)
    return fail(CQG_E_INVALID, "cqg_system_averages_noalloc: n_states * n_avr = " + std::to_string(n_states * nAvr) +
                                   " exceeds the fixed scratch of " + std::to_string(kScratchDoubles) + " doubles");
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) return fail(CQG_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
  if (device != cqg::dev::systemDevice(sys))
    return fail(CQG_E_INVALID, "cqg_system_averages_noalloc: the current device is not the system's device");
  DeviceSetup setup;
  if (int rc = setupFor(device, &setup)) return rc;
  double* slots = setup.scratch;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // one warp per state, four per CTA, at most 16 CTAs per SM (grid-stride beyond that)
  const int blocks = int(std::min<long long>((n_states + 3) / 4, 16ll * setup.sms));
  stateAveragesKernel<<<blocks, 128, 0, s>>>(*sd, reinterpret_cast<const double2*>(psi), n_states, nAvr, slots);
  err = cudaGetLastError();
  if (err != cudaSuccess) return fail(CQG_E_CUDA, std::string("state averages launch: ") + cudaGetErrorString(err));
  sumSlotsKernel<<<nAvr, 256, 0, s>>>(slots, n_states, nAvr, sums);
  err = cudaGetLastError();
  if (err != cudaSuccess) return fail(CQG_E_CUDA, std::string("sum launch: ") + cudaGetErrorString(err));
  return CQG_OK;
}
