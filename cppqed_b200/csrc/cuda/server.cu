// Continuous-batching request server for MCWF ensembles (cqg_server_*, include/cqg.h).
//
// The reference evolves one ensemble at a time (Ensemble::advance,
// StochasticTrajectory.h:220-245, driven by trajectory::run, Trajectory.h:310-339); it has no
// serving mode.  Here requests (a system, an initial state, a number of trajectories, an
// end time T and an output interval Dt) arrive while others run.  A round:
//   1. admits waiting requests, in arrival order, whose trajectories fit the free slots and
//      whose states fit the free part of the state heap (the HBM budget);
//   2. advances every admitted trajectory to its request's next output time, all requests
//      in the same launches (one persistent launch per kernel group, the groups on
//      concurrent streams; each trajectory carries its own end time);
//   3. reduces each request's averages over its own trajectories in a fixed order (the same
//      order as an ensemble of that request alone) and appends one output row;
//   4. releases the slots and heap of requests that reached T.
// States, times and random streams stay on the device between rounds.  Trajectory i of a
// request with stream s draws from pcg64{seed, s + i}, exactly as trajectory i of an
// ensemble with prng_stream s, so a request's result does not depend on what else runs.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <numeric>

#include "engine_internal.cuh"

using cqg::fail;
using namespace cqg::engine;
namespace dev = cqg::dev;

namespace {

constexpr int kJumpCap = 64;
constexpr int kReduceThreads = 256;

// first-fit allocator of index ranges in [0, cap)
class RangeAlloc {
 public:
  explicit RangeAlloc(int64_t cap = 0) {
    if (cap > 0) free_[0] = cap;
  }
  int64_t alloc(int64_t n) {
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= n) {
        const int64_t s = it->first, len = it->second;
        free_.erase(it);
        if (len > n) free_[s + n] = len - n;
        return s;
      }
    return -1;
  }
  void release(int64_t s, int64_t n) {
    auto next = free_.lower_bound(s);
    if (next != free_.end() && next->first == s + n) {
      n += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == s) {
        prev->second += n;
        return;
      }
    }
    free_[s] = n;
  }

 private:
  std::map<int64_t, int64_t> free_;  // start -> length
};

// Fixed-order sums of the averages of each request's trajectories: block (r, c) sums column
// c (the last, c = nCols - 1, is the dtDid slot at stride - 1) over slots
// [first[r], first[r] + count[r]) exactly as the ensemble reduction does.
__global__ void segmentSumsKernel(const double* __restrict__ avr, int stride, const int* __restrict__ first,
                                  const int* __restrict__ count, int nCols, double* __restrict__ sums) {
  const int r = blockIdx.x / nCols, c = blockIdx.x % nCols;
  const int src = c == nCols - 1 ? stride - 1 : c;
  __shared__ double part[kReduceThreads];
  const int f = first[r], n = count[r];
  double acc = 0.;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += avr[size_t(f + i) * stride + src];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[size_t(r) * stride + c] = part[0];
}

// OR of the status words of each request's trajectories
__global__ void segmentStatusKernel(const unsigned* __restrict__ st, const int* __restrict__ first,
                                    const int* __restrict__ count, unsigned* __restrict__ out) {
  const int r = blockIdx.x;
  unsigned v = 0;
  for (int i = threadIdx.x; i < count[r]; i += blockDim.x) v |= st[first[r] + i];
  v = __reduce_or_sync(0xffffffffu, v);
  __shared__ unsigned w[kReduceThreads / 32];
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned a = 0;
    for (int k = 0; k < int(blockDim.x >> 5); ++k) a |= w[k];
    out[r] = a;
  }
}

double secondsSince(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct cqg_server {
  struct Request {
    int64_t id = 0;
    const cqg_system* sys = nullptr;
    int sysSlot = -1;
    std::vector<cqg_complex> psi0;
    int64_t nTraj = 0;
    double T = 0, Dt = 0;
    uint64_t stream = 0;
    int64_t slot0 = -1, elem0 = -1;
    double target = 0;  // end time of the interval in flight
    std::vector<double> out;
    int nRows = 0;
    int nCols = 0;  // averages + dtDid
    unsigned status = 0;
    uint64_t steps = 0;
    double tSubmit = 0, tAdmit = 0, tDone = 0;
  };

  int device = 0;
  cqg_server_pars pars{};
  size_t elemBytes = 16;
  int64_t maxTraj = 0, maxElems = 0;
  int stride = 0;  // averages slot per trajectory (max_averages + 1)
  RangeAlloc slots, heap;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  int64_t nextId = 1;
  std::deque<std::unique_ptr<Request>> waiting;
  std::vector<std::unique_ptr<Request>> active;
  std::map<int64_t, std::unique_ptr<Request>> finished;
  std::vector<const cqg_system*> sysTable;
  // device
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evFork = nullptr;
  void* dmem = nullptr;
  dev::TrajDev td{};
  dev::SysDev* dSystems = nullptr;
  double* dTEnd = nullptr;
  double* dAvr = nullptr;
  int* dOrder = nullptr;
  int* dQueue = nullptr;
  int* dSegFirst = nullptr;
  int* dSegCount = nullptr;
  double* dSums = nullptr;
  unsigned* dSegStatus = nullptr;
  std::vector<KernelGroup> groups;  // one per group key, reused every round
  // statistics
  uint64_t roundSteps = 0;
  double kernelMs = 0;
  int64_t rounds = 0;

  ~cqg_server() {
    for (auto& g : groups) {
      if (g.scratch) cudaFree(g.scratch);
      if (g.done) cudaEventDestroy(g.done);
      if (g.stream) cudaStreamDestroy(g.stream);
    }
    if (dmem) cudaFree(dmem);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (evFork) cudaEventDestroy(evFork);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

using Request = cqg_server::Request;

template <typename T>
void putAsync(void* dst, const std::vector<T>& v, cudaStream_t st) {
  if (!v.empty()) ck(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
}

int systemSlot(cqg_server& s, const cqg_system* sys) {
  for (size_t k = 0; k < s.sysTable.size(); ++k)
    if (s.sysTable[k] == sys) return int(k);
  if (int(s.sysTable.size()) >= s.pars.max_systems) return -1;
  s.sysTable.push_back(sys);
  const int k = int(s.sysTable.size()) - 1;
  ck(cudaMemcpy(s.dSystems + k, &sys->sd, sizeof(dev::SysDev), cudaMemcpyHostToDevice), "cudaMemcpy(system)");
  return k;
}

// Writes the initial trajectory data of an admitted request into its slots.
void initialiseSlots(cqg_server& s, Request& r) {
  const int64_t n = r.nTraj, D = r.sys->L.D, s0 = r.slot0;
  std::vector<dcomp> psi(D);
  for (int64_t k = 0; k < D; ++k) psi[k] = dcomp(r.psi0[k].re, r.psi0[k].im);
  bool overshot = false;
  const double dt0 = initialDtTry(*r.sys, psi, s.pars.mcwf, &overshot);
  std::vector<unsigned char> one(size_t(D) * s.elemBytes);
  for (int64_t k = 0; k < D; ++k) {
    if (s.elemBytes == 16) {
      const double2 v = make_double2(psi[k].real(), psi[k].imag());
      std::memcpy(&one[k * 16], &v, 16);
    } else {
      const float2 v = make_float2(float(psi[k].real()), float(psi[k].imag()));
      std::memcpy(&one[k * 8], &v, 8);
    }
  }
  std::vector<unsigned char> states(size_t(n) * one.size());
  for (int64_t i = 0; i < n; ++i) std::memcpy(&states[size_t(i) * one.size()], one.data(), one.size());
  std::vector<long long> off(n);
  std::vector<int> idx(n, r.sysSlot);
  std::vector<double> zeros(n, 0.), dtTry(n, dt0);
  std::vector<unsigned long long> rng(4 * n, 0), cnt(8 * n, 0);
  for (int64_t i = 0; i < n; ++i) {
    off[i] = r.elem0 + i * D;
    if (s.pars.mcwf.rng == CQG_RNG_PCG64) {
      const auto g = dev::Pcg64::seeded(s.pars.mcwf.seed, r.stream + uint64_t(i));
      rng[4 * i + 0] = g.state.hi;
      rng[4 * i + 1] = g.state.lo;
      rng[4 * i + 2] = g.inc.hi;
      rng[4 * i + 3] = g.inc.lo;
    }
    if (overshot) cnt[8 * i + 4] = 1;
  }
  cudaStream_t st = s.stream;
  char* heap = static_cast<char*>(s.td.psi) + size_t(r.elem0) * s.elemBytes;
  ck(cudaMemcpyAsync(heap, states.data(), states.size(), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(states)");
  putAsync(const_cast<long long*>(s.td.psiOff) + s0, off, st);
  putAsync(const_cast<int*>(s.td.sysIdx) + s0, idx, st);
  putAsync(s.td.t + s0, zeros, st);
  putAsync(s.td.t0 + s0, zeros, st);
  putAsync(s.td.dtTry + s0, dtTry, st);
  putAsync(s.td.dtDid + s0, zeros, st);
  putAsync(s.td.rng + 4 * s0, rng, st);
  putAsync(s.td.cnt + 8 * s0, cnt, st);
  ck(cudaMemsetAsync(s.td.maxima + 3 * s0, 0, size_t(n) * 3 * sizeof(double), st), "cudaMemsetAsync");
  ck(cudaMemsetAsync(s.td.status + s0, 0, size_t(n) * sizeof(unsigned), st), "cudaMemsetAsync");
  ck(cudaMemsetAsync(s.td.jumpN + s0, 0, size_t(n) * sizeof(unsigned long long), st), "cudaMemsetAsync");
  // host buffers above are pageable: the copies have completed when cudaMemcpyAsync returns
  // for them only in the synchronous sense, so wait before they go out of scope
  ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

void admit(cqg_server& s) {
  for (auto it = s.waiting.begin(); it != s.waiting.end();) {
    Request& r = **it;
    const int64_t elems = r.nTraj * r.sys->L.D;
    const int64_t s0 = s.slots.alloc(r.nTraj);
    if (s0 < 0) {
      ++it;
      continue;
    }
    const int64_t e0 = s.heap.alloc(elems);
    if (e0 < 0) {
      s.slots.release(s0, r.nTraj);
      ++it;
      continue;
    }
    r.slot0 = s0;
    r.elem0 = e0;
    r.tAdmit = secondsSince(s.t0);
    initialiseSlots(s, r);
    s.active.push_back(std::move(*it));
    it = s.waiting.erase(it);
  }
}

// One round over the active requests: every trajectory to its request's next output time.
void advance(cqg_server& s) {
  const size_t nReq = s.active.size();
  if (!nReq) return;
  cudaStream_t st = s.stream;
  // per-trajectory end times and the order array, group by group
  std::vector<double> tEnd;
  std::vector<int> segFirst(nReq), segCount(nReq);
  std::vector<std::vector<std::pair<int64_t, int>>> byGroup(kMaxGroups + 1);  // (D, slot)
  for (size_t q = 0; q < nReq; ++q) {
    Request& r = *s.active[q];
    r.target = std::min(r.T, r.target + r.Dt);
    tEnd.assign(r.nTraj, r.target);
    putAsync(s.dTEnd + r.slot0, tEnd, st);
    segFirst[q] = int(r.slot0);
    segCount[q] = int(r.nTraj);
    const int key = groupKey(r.sys->L.D, r.sys->sd.S);
    for (int64_t i = 0; i < r.nTraj; ++i) byGroup[key].push_back({r.sys->L.D, int(r.slot0 + i)});
  }
  std::vector<int> order;
  order.reserve(s.maxTraj);
  std::vector<KernelGroup*> launch;
  for (int key = kMaxGroups; key >= 1; --key) {
    auto& v = byGroup[key];
    if (v.empty()) continue;
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    KernelGroup& g = s.groups[key];
    g.first = int64_t(order.size());
    g.count = int64_t(v.size());
    g.Dmax = 0;
    g.smax = 0;
    g.anyFreq = false;
    g.phaseElems = 0;
    g.phaseTable = s.pars.mcwf.ip_phase_table >= 0;
    for (auto& p : v) {
      order.push_back(p.second);
      g.Dmax = std::max<int>(g.Dmax, int(p.first));
    }
    for (auto& req : s.active)
      if (groupKey(req->sys->L.D, req->sys->sd.S) == key) {
        g.smax = std::max(g.smax, req->sys->sd.S);
        g.anyFreq |= req->sys->sd.hasFreq != 0;
        if (g.kind == 1 && g.phaseTable) g.phaseElems = std::max(g.phaseElems, blockPhaseElems(req->sys->sd));
      }
    launch.push_back(&g);
  }
  putAsync(s.dOrder, order, st);
  putAsync(s.dSegFirst, segFirst, st);
  putAsync(s.dSegCount, segCount, st);
  ck(cudaMemsetAsync(s.dQueue, 0, (kMaxGroups + 1) * sizeof(int), st), "cudaMemsetAsync");

  dev::RunArgs ra{};
  ra.mode = dev::RUN_TO;
  ra.nIntervals = 1;
  ra.tEndPer = s.dTEnd;
  ra.absSlot = s.pars.mcwf.eps_rel;  // make_controlled(epsRel, epsAbs, ...) (ODE.h:205)
  ra.relSlot = s.pars.mcwf.eps_abs;
  ra.dpLimit = s.pars.mcwf.dp_limit;
  ra.overTol = s.pars.mcwf.overshoot_tolerance;
  ra.maxAttempts = s.pars.mcwf.max_attempts;
  ra.noise = s.pars.mcwf.noise;
  ra.rng = s.pars.mcwf.rng;
  ra.seed = s.pars.mcwf.seed;
  ra.maxStepsPerInterval = 2000000000LL;
  ra.timeLimitNs = 120ull * 1000000000ull;
  ra.avrOut = s.dAvr;
  ra.nAvrStride = s.stride;
  int nSM = 0;
  ck(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, s.device), "attribute");
  ck(cudaEventRecord(s.ev0, st), "cudaEventRecord");
  ck(cudaEventRecord(s.evFork, st), "cudaEventRecord");
  for (KernelGroup* g : launch) {
    const int gi = int(g - s.groups.data());
    ck(cudaStreamWaitEvent(g->stream, s.evFork, 0), "cudaStreamWaitEvent");
    ra.order = s.dOrder + g->first;
    ra.nTasks = int(g->count);
    ra.queue = s.dQueue + gi;
    launchGroup(s.pars.mcwf.precision == CQG_FP64, s.elemBytes, s.td, *g, ra, nSM, g->stream);
    ck(cudaEventRecord(g->done, g->stream), "cudaEventRecord");
    ck(cudaStreamWaitEvent(st, g->done, 0), "cudaStreamWaitEvent");
  }
  ck(cudaEventRecord(s.ev1, st), "cudaEventRecord");
  int nCols = 0;
  for (auto& r : s.active) nCols = std::max(nCols, r->nCols);
  segmentSumsKernel<<<unsigned(nReq * nCols), kReduceThreads, 0, st>>>(s.dAvr, s.stride, s.dSegFirst, s.dSegCount,
                                                                       nCols, s.dSums);
  ck(cudaGetLastError(), "segment sums launch");
  segmentStatusKernel<<<unsigned(nReq), kReduceThreads, 0, st>>>(s.td.status, s.dSegFirst, s.dSegCount,
                                                                 s.dSegStatus);
  ck(cudaGetLastError(), "segment status launch");
  std::vector<double> sums(nReq * s.stride);
  std::vector<unsigned> status(nReq);
  ck(cudaMemcpyAsync(sums.data(), s.dSums, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  ck(cudaMemcpyAsync(status.data(), s.dSegStatus, nReq * sizeof(unsigned), cudaMemcpyDeviceToHost, st),
     "cudaMemcpyAsync");
  ck(cudaStreamSynchronize(st), "round");
  float ms = 0;
  ck(cudaEventElapsedTime(&ms, s.ev0, s.ev1), "cudaEventElapsedTime");
  s.kernelMs += ms;
  ++s.rounds;

  // output rows, completions
  for (size_t q = 0; q < nReq; ++q) {
    Request& r = *s.active[q];
    // the request's averages, then the dtDid column (summed into column nCols - 1)
    r.out.insert(r.out.end(), sums.begin() + q * s.stride, sums.begin() + q * s.stride + (r.nCols - 1));
    r.out.push_back(sums[q * s.stride + nCols - 1]);
    ++r.nRows;
    r.status |= status[q];
  }
  for (auto it = s.active.begin(); it != s.active.end();) {
    Request& r = **it;
    if (r.target >= r.T || r.status) {
      std::vector<unsigned long long> cnt(8 * r.nTraj);
      ck(cudaMemcpy(cnt.data(), s.td.cnt + 8 * r.slot0, cnt.size() * sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost),
         "cudaMemcpy(counters)");
      for (int64_t i = 0; i < r.nTraj; ++i) r.steps += cnt[8 * i];
      s.roundSteps += r.steps;
      s.slots.release(r.slot0, r.nTraj);
      s.heap.release(r.elem0, r.nTraj * r.sys->L.D);
      r.tDone = secondsSince(s.t0);
      const int64_t id = r.id;
      s.finished[id] = std::move(*it);
      it = s.active.erase(it);
    } else {
      ++it;
    }
  }
}

}  // namespace

extern "C" {

void cqg_server_pars_default(cqg_server_pars* p) {
  if (!p) return;
  *p = cqg_server_pars{};
  p->hbm_budget_bytes = uint64_t(8) << 30;
  p->max_trajectories = 1 << 16;
  p->max_systems = 1024;
  p->max_averages = 32;
  cqg_mcwf_pars_default(&p->mcwf);
}

int cqg_server_create(const cqg_server_pars* p, cqg_server** out) {
  return guardedCuda([&] {
    if (!p || !out) return fail(CQG_E_INVALID, "cqg_server_create: null argument");
    if (p->max_trajectories < 1 || p->max_systems < 1 || p->max_averages < 1 || p->max_averages > 255)
      return fail(CQG_E_INVALID, "cqg_server_create: bad capacities");
    const auto& m = p->mcwf;
    if (m.precision != CQG_FP64 && m.precision != CQG_FP32) return fail(CQG_E_INVALID, "cqg_server_create: precision");
    if (m.rng != CQG_RNG_PCG64 && m.rng != CQG_RNG_PHILOX) return fail(CQG_E_INVALID, "cqg_server_create: rng");
    if (!(m.eps_rel > 0) || !(m.eps_abs >= 0) || !(m.dp_limit > 0) || !(m.overshoot_tolerance >= 1))
      return fail(CQG_E_INVALID, "cqg_server_create: eps_rel > 0, eps_abs >= 0, dp_limit > 0, overshoot_tolerance >= 1");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
      cudaGetLastError();
      return fail(CQG_E_NODEVICE, "cqg_server_create: no CUDA device");
    }
    auto s = std::make_unique<cqg_server>();
    s->pars = *p;
    if (s->pars.mcwf.max_attempts <= 0) s->pars.mcwf.max_attempts = 100000;
    ck(cudaGetDevice(&s->device), "cudaGetDevice");
    s->elemBytes = m.precision == CQG_FP64 ? 16 : 8;
    s->maxTraj = p->max_trajectories;
    s->stride = p->max_averages + 1;
    // per-slot bytes: offsets, index, 5 times, rng, counters, maxima, status, jump ring,
    // averages slot; the state heap takes the rest of the budget
    const size_t perSlot = 8 + 4 + 5 * 8 + 32 + 64 + 24 + 4 + kJumpCap * 12 + 8 + 4 + size_t(s->stride) * 8 + 8 + 8;
    const size_t fixed = size_t(p->max_systems) * sizeof(dev::SysDev) + size_t(s->maxTraj) * perSlot + (64 << 10);
    if (p->hbm_budget_bytes <= fixed + (1 << 20))
      return fail(CQG_E_INVALID, "cqg_server_create: hbm_budget_bytes below the slot tables");
    s->maxElems = int64_t((p->hbm_budget_bytes - fixed) / s->elemBytes);
    s->slots = RangeAlloc(s->maxTraj);
    s->heap = RangeAlloc(s->maxElems);

    size_t total = 0;
    auto add = [&](size_t bytes) {
      const size_t off = (total + 255) & ~size_t(255);
      total = off + bytes;
      return off;
    };
    const int64_t N = s->maxTraj;
    const size_t oPsi = add(size_t(s->maxElems) * s->elemBytes), oOff = add(N * 8), oIdx = add(N * 4),
                 oT = add(N * 8), oT0 = add(N * 8), oTry = add(N * 8), oDid = add(N * 8), oEnd = add(N * 8),
                 oRng = add(N * 32), oCnt = add(N * 64), oMax = add(N * 24), oSt = add(N * 4),
                 oJT = add(N * kJumpCap * 8), oJL = add(N * kJumpCap * 4), oJN = add(N * 8),
                 oAvr = add(size_t(N) * s->stride * 8), oOrd = add(N * 4), oSegF = add(N * 4), oSegC = add(N * 4),
                 oSums = add(size_t(N) * s->stride * 8), oSegS = add(N * 4), oQ = add((kMaxGroups + 1) * 4),
                 oSys = add(size_t(p->max_systems) * sizeof(dev::SysDev));
    ck(cudaMalloc(&s->dmem, total), "cudaMalloc(server arena)");
    ck(cudaMemset(s->dmem, 0, total), "cudaMemset");
    char* b = static_cast<char*>(s->dmem);
    auto& td = s->td;
    td.nTraj = int(N);
    td.psi = b + oPsi;
    td.psiOff = reinterpret_cast<const long long*>(b + oOff);
    td.sysIdx = reinterpret_cast<const int*>(b + oIdx);
    td.systems = reinterpret_cast<const dev::SysDev*>(b + oSys);
    td.t = reinterpret_cast<double*>(b + oT);
    td.t0 = reinterpret_cast<double*>(b + oT0);
    td.dtTry = reinterpret_cast<double*>(b + oTry);
    td.dtDid = reinterpret_cast<double*>(b + oDid);
    td.rng = reinterpret_cast<unsigned long long*>(b + oRng);
    td.cnt = reinterpret_cast<unsigned long long*>(b + oCnt);
    td.maxima = reinterpret_cast<double*>(b + oMax);
    td.status = reinterpret_cast<unsigned*>(b + oSt);
    td.jumpT = reinterpret_cast<double*>(b + oJT);
    td.jumpL = reinterpret_cast<int*>(b + oJL);
    td.jumpN = reinterpret_cast<unsigned long long*>(b + oJN);
    td.jumpCap = kJumpCap;
    s->dSystems = reinterpret_cast<dev::SysDev*>(b + oSys);
    s->dTEnd = reinterpret_cast<double*>(b + oEnd);
    s->dAvr = reinterpret_cast<double*>(b + oAvr);
    s->dOrder = reinterpret_cast<int*>(b + oOrd);
    s->dSegFirst = reinterpret_cast<int*>(b + oSegF);
    s->dSegCount = reinterpret_cast<int*>(b + oSegC);
    s->dSums = reinterpret_cast<double*>(b + oSums);
    s->dSegStatus = reinterpret_cast<unsigned*>(b + oSegS);
    s->dQueue = reinterpret_cast<int*>(b + oQ);
    ck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreate(&s->ev0), "cudaEventCreate");
    ck(cudaEventCreate(&s->ev1), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&s->evFork, cudaEventDisableTiming), "cudaEventCreate");
    s->groups.resize(kMaxGroups + 1);
    for (int key = 1; key <= kMaxGroups; ++key) {
      KernelGroup& g = s->groups[key];
      g.kind = key == kMaxGroups ? 1 : 0;
      g.E = g.kind ? 0 : key;
      g.threads = m.cta_threads > 0 ? m.cta_threads : defaultThreads(g);
      if (g.threads % 32 || g.threads > (g.kind ? 512 : 128))
        return fail(CQG_E_INVALID, "cqg_server_create: cta_threads must be a multiple of 32, at most 128");
      ck(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking), "cudaStreamCreate");
      ck(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming), "cudaEventCreate");
    }
    *out = s.release();
    return CQG_OK;
  });
}

int cqg_server_submit(cqg_server* s, const cqg_system* sys, const cqg_complex* psi0, int64_t n_traj, double T,
                      double Dt, uint64_t prng_stream, int64_t* request_id) {
  return guardedCuda([&] {
    if (!s || !sys || !psi0 || !request_id) return fail(CQG_E_INVALID, "cqg_server_submit: null argument");
    if (n_traj < 1 || !(T > 0) || !(Dt > 0)) return fail(CQG_E_INVALID, "cqg_server_submit: n_traj >= 1, T > 0, Dt > 0");
    if (sys->device != s->device) return fail(CQG_E_INVALID, "cqg_server_submit: system on another device");
    if (sys->L.nAvr + 1 > s->stride) return fail(CQG_E_UNSUPPORTED, "cqg_server_submit: more averages than max_averages");
    if (int(sys->L.jumps.size()) > dev::MAX_JUMPS)
      return fail(CQG_E_UNSUPPORTED, "cqg_server_submit: more than 8 jump operators");
    if (sys->sd.S > kMaxSlots)
      return fail(CQG_E_UNSUPPORTED, "cqg_server_submit: more than 64 off-diagonal entries per row");
    if (int64_t(sys->L.D) * 2 * int64_t(s->elemBytes) > 200 * 1024)
      return fail(CQG_E_UNSUPPORTED, "cqg_server_submit: the stage vectors of a trajectory exceed shared memory");
    if (n_traj > s->maxTraj || n_traj * sys->L.D > s->maxElems)
      return fail(CQG_E_INVALID, "cqg_server_submit: the request alone exceeds the server's capacity");
    auto r = std::make_unique<Request>();
    r->sysSlot = systemSlot(*s, sys);
    if (r->sysSlot < 0) return fail(CQG_E_INVALID, "cqg_server_submit: more distinct systems than max_systems");
    r->id = s->nextId++;
    r->sys = sys;
    r->psi0.assign(psi0, psi0 + sys->L.D);
    r->nTraj = n_traj;
    r->T = T;
    r->Dt = Dt;
    r->stream = prng_stream;
    r->nCols = sys->L.nAvr + 1;
    r->tSubmit = secondsSince(s->t0);
    *request_id = r->id;
    s->waiting.push_back(std::move(r));
    return CQG_OK;
  });
}

int cqg_server_round(cqg_server* s, int32_t* n_active, int32_t* n_waiting) {
  return guardedCuda([&] {
    if (!s) return fail(CQG_E_INVALID, "cqg_server_round: null server");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    admit(*s);
    advance(*s);
    if (n_active) *n_active = int32_t(s->active.size());
    if (n_waiting) *n_waiting = int32_t(s->waiting.size());
    return CQG_OK;
  });
}

int cqg_server_completed(cqg_server* s, int64_t* ids, int32_t cap, int32_t* n) {
  if (!s || !n || (cap > 0 && !ids)) return fail(CQG_E_INVALID, "cqg_server_completed: null argument");
  int32_t k = 0;
  for (auto& kv : s->finished) {
    if (k < cap) ids[k] = kv.first;
    ++k;
  }
  *n = k;
  return CQG_OK;
}

int cqg_server_result(cqg_server* s, int64_t id, double* rows, int32_t cap_rows, int32_t* n_rows, int32_t* n_cols,
                      uint64_t* steps, double* times, uint32_t* status) {
  if (!s || !n_rows || !n_cols) return fail(CQG_E_INVALID, "cqg_server_result: null argument");
  auto it = s->finished.find(id);
  if (it == s->finished.end()) return fail(CQG_E_INVALID, "cqg_server_result: no finished request with this id");
  const Request& r = *it->second;
  *n_rows = r.nRows;
  *n_cols = r.nCols;
  if (rows && cap_rows > 0)
    std::copy(r.out.begin(), r.out.begin() + size_t(std::min(cap_rows, r.nRows)) * r.nCols, rows);
  if (steps) *steps = r.steps;
  if (times) {
    times[0] = r.tSubmit;
    times[1] = r.tAdmit;
    times[2] = r.tDone;
  }
  if (status) *status = r.status;
  if (rows && cap_rows >= r.nRows) s->finished.erase(it);  // delivered: forget it
  return CQG_OK;
}

int cqg_server_stats(const cqg_server* s, uint64_t* steps, double* kernel_ms, int64_t* rounds) {
  if (!s) return fail(CQG_E_INVALID, "cqg_server_stats: null server");
  if (steps) *steps = s->roundSteps;
  if (kernel_ms) *kernel_ms = s->kernelMs;
  if (rounds) *rounds = s->rounds;
  return CQG_OK;
}

int cqg_server_destroy(cqg_server* s) {
  delete s;
  return CQG_OK;
}

}  // extern "C"
