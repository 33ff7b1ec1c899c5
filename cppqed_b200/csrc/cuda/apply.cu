// Batched H/i application: the drop-in for structure::Hamiltonian::addContribution
// (Hamiltonian.h:38-43), i.e. for the reference's slice-wise Tridiagonal::apply
// (Tridiagonal.tcc:220-263) over a composite system, on many states at once:
//   dpsi_i += (H/i)(tau) psi_i      for every state i,  tau = t - t0.
// The operator is the system's row-gather table (fused diagonal + S off-diagonal
// slots per row, see lowering.hpp).  The work is bound by HBM bandwidth: 48 bytes per
// element (read psi, read and write dpsi); the tables are a few KB.
//
// Main kernel (stagedApplyKernel): persistent CTAs walk chunks of whole states.  One
// thread issues bulk asynchronous copies (cp.async.bulk, completion on an mbarrier) of a
// chunk of psi and the matching chunk of dpsi into shared memory, NST chunks ahead; the
// CTA adds H/i psi into the dpsi chunk in place, gathering the banded neighbours from
// shared memory, and the same thread writes the chunk back with a bulk store.  Each
// thread owns fixed rows, so its coefficients (with the interaction-picture phase
// exp(tau * freq) already applied) sit in registers for the whole launch.
// Fallback (elementApplyKernel): a grid-stride walk over elements with the gathers from
// global memory, for more than 4 off-diagonal slots (any number) or states too large for the
// shared-memory stages.  Both kernels move complex numbers as 16-byte vectors, so the entry
// point refuses psi / dpsi pointers that are not 16-byte aligned.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../host/errors.hpp"
#include "cqg.h"
#include "engine_internal.cuh"
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

// ---- fallback: element-parallel grid-stride walk ------------------------------------

template <int S>
__device__ __forceinline__ double2 applyRow(const SysDev& sys, const double2* __restrict__ x, int r, double2 acc,
                                            double tau) {
  const int D = sys.D;
  acc = cqg::dev::cfma(__ldg(&sys.diagD[r]), __ldg(&x[r]), acc);
  const int nS = S >= 0 ? S : sys.S;
#pragma unroll
  for (int s = 0; s < (S >= 0 ? S : nS); ++s) {
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
__global__ void __launch_bounds__(256) elementApplyKernel(SysDev sys, const double2* __restrict__ psi,
                                                          double2* __restrict__ dpsi, long long total, double tau) {
  const long long D = sys.D;
  for (long long g = blockIdx.x * 256ll + threadIdx.x; g < total; g += gridDim.x * 256ll) {
    const long long i = g / D;
    dpsi[g] = applyRow<S>(sys, psi + i * D, int(g - i * D), dpsi[g], tau);
  }
}

// ---- staged kernel: bulk copies through shared memory --------------------------------

constexpr int kStageTargetBytes = 16384;  // one psi (or dpsi) buffer of a stage
constexpr int kMaxConsumers = 992;         // consumer threads per CTA (+ one producer warp)
constexpr unsigned long long kWaitLimitNs = 1000000000ull;

// Waits that gave up after kWaitLimitNs (a bulk copy that never completed); the CTA then
// stops instead of spinning.  Zero in every healthy run.
__device__ unsigned gApplyWaitTimeouts;

struct StagedGeom {
  int D;
  int m;          // states processed side by side (consumer thread = state lane * D + row)
  int cs;         // states per chunk
  int nst;        // pipeline stages
  int consumers;  // m * D, consumer threads
  long long nStates, nChunks;
};

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbarInit(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarExpectTx(uint32_t bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbarArrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint32_t bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait on one phase of an mbarrier (wall clock, kWaitLimitNs).
__device__ __forceinline__ bool mbarWait(uint32_t bar, unsigned parity) {
  if (mbarTryWait(bar, parity)) return true;
  const unsigned long long t0 = cqg::dev::globalTimerNs();
  while (!mbarTryWait(bar, parity))
    if (cqg::dev::globalTimerNs() - t0 > kWaitLimitNs) {
      atomicAdd(&gApplyWaitTimeouts, 1u);
      return false;
    }
  return true;
}
__device__ __forceinline__ void bulkLoad(uint32_t dst, const void* src, unsigned bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void bulkStore(void* dst, uint32_t src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulkWaitRead() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulkWaitAll() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Shared memory: full[nst] and done[nst] mbarriers (128 bytes), then per stage the psi and
// the dpsi buffer of one chunk.  Warp 0 is the producer (lane 0 issues every bulk copy);
// warps 1.. are consumers, thread c = lane-of-state * D + row owning row c % D of the
// states c / D, c / D + m, ... of each chunk.
//   full[s]  completes when both loads of the stage's chunk have landed (expect_tx);
//   done[s]  completes when every consumer warp has finished the stage's chunk.
// The producer stores a finished chunk, then refills the stage NST chunks ahead, so
// NST - 1 chunks are in flight while the consumers work on one.
template <int S>
__global__ void __launch_bounds__(1024) stagedApplyKernel(SysDev sys, const double2* __restrict__ psi,
                                                          double2* __restrict__ dpsi, StagedGeom g, double tau) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int D = g.D, nst = g.nst;
  const long long stride = gridDim.x;
  const uint32_t bar0 = smemAddr(smem);
  auto fullBar = [&](int s) { return bar0 + 8u * s; };
  auto doneBar = [&](int s) { return bar0 + 8u * (nst + s); };
  double2* stage0 = reinterpret_cast<double2*>(smem + 128);
  auto psiBuf = [&](int s) { return stage0 + size_t(2 * s) * g.cs * D; };
  auto dpsiBuf = [&](int s) { return stage0 + size_t(2 * s + 1) * g.cs * D; };
  const int consumerWarps = (g.consumers + 31) / 32;

  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mbarInit(fullBar(s), 1);
      mbarInit(doneBar(s), consumerWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  auto chunkStates = [&](long long chunk) {
    const long long left = g.nStates - chunk * g.cs;
    return left < g.cs ? int(left) : g.cs;
  };

  if (threadIdx.x < 32) {  // producer warp
    if (threadIdx.x != 0) return;
    for (int s = 0; s < nst; ++s) {
      const long long chunk = blockIdx.x + s * stride;
      if (chunk >= g.nChunks) break;
      const unsigned bytes = unsigned(chunkStates(chunk)) * unsigned(D) * 16u;
      mbarExpectTx(fullBar(s), 2u * bytes);
      bulkLoad(smemAddr(psiBuf(s)), psi + chunk * g.cs * D, bytes, fullBar(s));
      bulkLoad(smemAddr(dpsiBuf(s)), dpsi + chunk * g.cs * D, bytes, fullBar(s));
    }
    int it = 0;
    for (long long chunk = blockIdx.x; chunk < g.nChunks; chunk += stride, ++it) {
      const int s = it % nst;
      if (!mbarWait(doneBar(s), unsigned(it / nst) & 1u)) break;
      bulkStore(dpsi + chunk * g.cs * D, smemAddr(dpsiBuf(s)), unsigned(chunkStates(chunk)) * unsigned(D) * 16u);
      const long long next = chunk + nst * stride;
      if (next < g.nChunks) {
        const unsigned bytes = unsigned(chunkStates(next)) * unsigned(D) * 16u;
        mbarExpectTx(fullBar(s), 2u * bytes);
        bulkLoad(smemAddr(psiBuf(s)), psi + next * g.cs * D, bytes, fullBar(s));
        bulkWaitRead();  // the store has read the dpsi buffer
        bulkLoad(smemAddr(dpsiBuf(s)), dpsi + next * g.cs * D, bytes, fullBar(s));
      }
    }
    bulkWaitAll();
    return;
  }

  // consumers: fixed row, coefficients (interaction-picture phase applied) in registers
  const int c = threadIdx.x - 32;
  const bool active = c < g.consumers;
  const int r = active ? c % D : 0;
  const int lane0 = active ? c / D : 0;
  double2 dg = make_double2(0., 0.);
  double2 cf[S > 0 ? S : 1];
  int cl[S > 0 ? S : 1];
  if (active) {
    dg = __ldg(&sys.diagD[r]);
#pragma unroll
    for (int s = 0; s < S; ++s) {
      double2 v = __ldg(&sys.valD[s * D + r]);
      if (sys.freq) {
        const double2 f = __ldg(&sys.freq[s * D + r]);
        if (f.x != 0. || f.y != 0.) {
          const double2 ph = cqg::dev::cexpScaled(tau, f);
          v = make_double2(v.x * ph.x - v.y * ph.y, v.x * ph.y + v.y * ph.x);
        }
      }
      cf[s] = v;
      cl[s] = __ldg(&sys.col[s * D + r]);
    }
  }
  int it = 0;
  for (long long chunk = blockIdx.x; chunk < g.nChunks; chunk += stride, ++it) {
    const int s = it % nst;
    const bool landed = mbarWait(fullBar(s), unsigned(it / nst) & 1u);
    if (!__all_sync(0xffffffffu, landed)) return;  // the whole warp leaves together
    if (active) {
      const double2* x = psiBuf(s);
      double2* y = dpsiBuf(s);
      const int n = chunkStates(chunk);
      for (int i = lane0; i < n; i += g.m) {
        const double2* xi = x + i * D;
        double2 acc = y[i * D + r];
        acc = cqg::dev::cfma(dg, xi[r], acc);
#pragma unroll
        for (int k = 0; k < S; ++k) acc = cqg::dev::cfma(cf[k], xi[cl[k]], acc);
        y[i * D + r] = acc;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> bulk store
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbarArrive(doneBar(s));
  }
}

// Geometry of the staged kernel for D rows, or false when it does not apply.
bool stagedGeometry(int D, long long nStates, StagedGeom& g, size_t& smemBytes) {
  if (D > kMaxConsumers) return false;
  g.D = D;
  g.m = std::max(1, 256 / D);
  g.consumers = g.m * D;
  const int perLane = std::max(1, kStageTargetBytes / (g.consumers * 16));
  g.cs = g.m * perLane;
  g.nStates = nStates;
  g.nChunks = (nStates + g.cs - 1) / g.cs;
  const size_t stageBytes = 2ull * g.cs * D * 16;
  for (g.nst = 3; g.nst >= 2; --g.nst) {
    smemBytes = 128 + g.nst * stageBytes;
    if (smemBytes <= 227 * 1024) return true;
  }
  return false;
}

template <int S>
cudaError_t launchStaged(const SysDev& sd, const double2* psi, double2* dpsi, const StagedGeom& g, size_t smemBytes,
                         double tau, cudaStream_t st, int nSM) {
  const int threads = 32 + (g.consumers + 31) / 32 * 32;
  cudaError_t err = cudaFuncSetAttribute(stagedApplyKernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smemBytes));
  int perSM = 0;
  if (err == cudaSuccess)
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, stagedApplyKernel<S>, threads, smemBytes);
  if (err != cudaSuccess) return err;
  const long long blocks = std::min<long long>(g.nChunks, (long long)nSM * std::max(1, perSM));
  stagedApplyKernel<S><<<unsigned(blocks), threads, smemBytes, st>>>(sd, psi, dpsi, g, tau);
  return cudaGetLastError();
}

template <int S>
cudaError_t launchElement(const SysDev& sd, const double2* psi, double2* dpsi, long long nStates, double tau,
                          cudaStream_t st, int nSM) {
  int perSM = 0;
  cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, elementApplyKernel<S>, 256, 0);
  if (err != cudaSuccess) return err;
  const long long total = nStates * sd.D;
  const long long blocks = std::min<long long>((total + 255) / 256, (long long)nSM * std::max(1, perSM));
  elementApplyKernel<S><<<unsigned(blocks), 256, 0, st>>>(sd, psi, dpsi, total, tau);
  return cudaGetLastError();
}

}  // namespace

namespace cqg {
namespace engine {

cudaError_t applyHamiltonian(const SysDev& sd, const double2* p, double2* q, long long nStates, double tau,
                             cudaStream_t st, int nSM) {
  StagedGeom g{};
  size_t smemBytes = 0;
  if (sd.S <= 4 && stagedGeometry(sd.D, nStates, g, smemBytes)) {
    switch (sd.S) {
      case 0: return launchStaged<0>(sd, p, q, g, smemBytes, tau, st, nSM);
      case 1: return launchStaged<1>(sd, p, q, g, smemBytes, tau, st, nSM);
      case 2: return launchStaged<2>(sd, p, q, g, smemBytes, tau, st, nSM);
      case 3: return launchStaged<3>(sd, p, q, g, smemBytes, tau, st, nSM);
      default: return launchStaged<4>(sd, p, q, g, smemBytes, tau, st, nSM);
    }
  }
  switch (sd.S) {
    case 0: return launchElement<0>(sd, p, q, nStates, tau, st, nSM);
    case 1: return launchElement<1>(sd, p, q, nStates, tau, st, nSM);
    case 2: return launchElement<2>(sd, p, q, nStates, tau, st, nSM);
    case 3: return launchElement<3>(sd, p, q, nStates, tau, st, nSM);
    case 4: return launchElement<4>(sd, p, q, nStates, tau, st, nSM);
    default: return launchElement<-1>(sd, p, q, nStates, tau, st, nSM);
  }
}

}  // namespace engine
}  // namespace cqg

extern "C" int cqg_system_apply_hamiltonian(const cqg_system* sys, const cqg_complex* psi, cqg_complex* dpsi,
                                            int64_t n_states, double tau, void* stream) {
  if (!sys || !psi || !dpsi || n_states < 1)
    return fail(CQG_E_INVALID, "cqg_system_apply_hamiltonian: null pointer or no states");
  const SysDev* sd = cqg::dev::systemDescriptor(sys);
  int device = 0, nSM = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, device);
  if (err != cudaSuccess) return fail(CQG_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
  if (device != cqg::dev::systemDevice(sys))
    return fail(CQG_E_INVALID, "cqg_system_apply_hamiltonian: the current device is not the system's device");
  if ((reinterpret_cast<uintptr_t>(psi) | reinterpret_cast<uintptr_t>(dpsi)) % 16 != 0)
    return fail(CQG_E_INVALID, "cqg_system_apply_hamiltonian: psi and dpsi must be 16-byte aligned");
  err = cqg::engine::applyHamiltonian(*sd, reinterpret_cast<const double2*>(psi), reinterpret_cast<double2*>(dpsi),
                                      n_states, tau, static_cast<cudaStream_t>(stream), nSM);
  if (err != cudaSuccess) return fail(CQG_E_CUDA, std::string("apply launch: ") + cudaGetErrorString(err));
  return CQG_OK;
}
