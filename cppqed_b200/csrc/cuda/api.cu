// extern "C" engine entry points (include/cqg.h): device-resident systems, ensembles
// and the launches of the fused MCWF kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "engine_internal.cuh"

using cqg::fail;
using cqg::guarded;
namespace dev = cqg::dev;
using namespace cqg::engine;

namespace {

// A process-wide pinned host buffer for staging uploads (grown on demand, kept until exit,
// one user at a time).
class HostStaging {
 public:
  explicit HostStaging(size_t bytes) : lock_(mutex()) {
    Buf& b = buf();
    if (b.size < bytes) {
      if (b.ptr) cudaFreeHost(b.ptr);
      b.ptr = nullptr;
      b.size = 0;
      ck(cudaHostAlloc(&b.ptr, bytes, cudaHostAllocPortable), "cudaHostAlloc(staging)");
      b.size = bytes;
    }
  }
  char* data() { return static_cast<char*>(buf().ptr); }

 private:
  struct Buf {
    void* ptr = nullptr;
    size_t size = 0;
  };
  static std::mutex& mutex() {
    static std::mutex m;
    return m;
  }
  static Buf& buf() {
    static Buf b;
    return b;
  }
  std::lock_guard<std::mutex> lock_;
};

// single device allocation carved into aligned sub-buffers
// autotuner shape bit: the warp kernel's instance compiled for more resident CTAs
constexpr int kHighOccupancyFlag = 1 << 17;
// MCWF steps after which a warp hands its trajectory back to the work queue (cqg_mcwf_pars::
// yield_steps = 0), and push slots per trajectory and launch
constexpr int kDefaultYieldSteps = 64;
constexpr int64_t kYieldSlotsPerTrajectory = 64;

struct Arena {
  std::vector<std::pair<size_t, size_t>> parts;  // offset, size
  size_t total = 0;
  size_t add(size_t bytes) {
    const size_t off = (total + 255) & ~size_t(255);
    total = off + bytes;
    return off;
  }
};

}  // namespace

struct cqg_ensemble {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evRun0 = nullptr, evRun1 = nullptr, evFork = nullptr;
  float lastMs = 0, lastRunMs = 0;
  int64_t nTraj = 0;
  int nAvrMax = 0, Dmax = 0, Smax = 0;
  cqg_mcwf_pars pars{};
  std::vector<const cqg_system*> systems;
  std::vector<int> sysIdx;
  std::vector<long long> psiOff;
  std::vector<KernelGroup> groups;
  size_t elemBytes = 16;
  // device buffers (recycled blocks: deviceAlloc / deviceRelease)
  void* dmem = nullptr;
  size_t dmemBytes = 0;
  dev::TrajDev td{};
  dev::SysDev* dSystems = nullptr;
  int* dQueue = nullptr;  // one work-queue counter per group
  int* dOrder = nullptr;
  unsigned* dStatusOr = nullptr;
  double* dAvr = nullptr;
  size_t avrCap = 0;
  double* dSums = nullptr;
  size_t sumsCap = 0;
  int jumpCap = 64;
  void* dJumpRing = nullptr;  // jump rings of a grown capacity (cqg_ensemble_set_jump_capacity)
  size_t jumpRingBytes = 0;
  // warp-kernel yielding (RunArgs::yieldSteps): per group 4 header ints (push tail, finished
  // trajectories, error, pad) and the push marks, then every trajectory's ResumeInfo (these
  // zeroed before each launch), then per group the pushed trajectory indices
  void* dYield = nullptr;
  size_t yieldBytes = 0, yieldZeroBytes = 0;
  std::vector<size_t> yieldHead, yieldSeq, yieldEntry;  // byte offsets per group
  std::vector<int> yieldCap;
  size_t yieldResume = 0;
  ~cqg_ensemble() {
    // nothing of this ensemble may still run on the blocks that go back to the cache
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    for (auto& g : groups)
      if (g.stream) cudaStreamSynchronize(g.stream);
    if (stream) cudaStreamSynchronize(stream);
    for (auto& g : groups) {
      cqg::engine::deviceRelease(device, g.scratch, g.scratchBytes);
      if (g.done) cudaEventDestroy(g.done);
      if (g.stream) cudaStreamDestroy(g.stream);
    }
    cqg::engine::deviceRelease(device, dAvr, avrCap * sizeof(double));
    cqg::engine::deviceRelease(device, dSums, sumsCap * sizeof(double));
    cqg::engine::deviceRelease(device, dmem, dmemBytes);
    cqg::engine::deviceRelease(device, dJumpRing, jumpRingBytes);
    cqg::engine::deviceRelease(device, dYield, yieldBytes);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (evRun0) cudaEventDestroy(evRun0);
    if (evRun1) cudaEventDestroy(evRun1);
    if (evFork) cudaEventDestroy(evFork);
    if (stream) cudaStreamDestroy(stream);
    cudaSetDevice(cur);
  }
};

namespace cqg {
namespace engine {

// ---- recycled device blocks -----------------------------------------------------------
// Ensembles are created and destroyed at a high rate by services, parameter sweeps and
// benchmarks, and cudaMalloc / cudaFree cost driver work (cudaFree also synchronises the
// device).  Freed ensemble buffers are kept per (device, size class) and handed to the
// next request of that class: sizes round up to a power of two from 4 KiB to 2 MiB and to a
// multiple of 2 MiB above.  At most kCacheCap bytes stay cached per device; a cudaMalloc
// that fails returns the device's cached blocks to the driver and is retried once.
namespace blockcache {
constexpr size_t kCacheCap = size_t(8) << 30;
struct BlockCache {
  std::mutex mu;
  std::map<std::pair<int, size_t>, std::vector<void*>> blocks;
  std::map<int, size_t> cached;
};
BlockCache& blockCache() {
  static BlockCache* c = new BlockCache;  // never destroyed: blocks outlive static teardown
  return *c;
}
size_t sizeClass(size_t b) {
  const size_t grain = size_t(2) << 20;
  if (b >= grain) return (b + grain - 1) / grain * grain;
  size_t c = 4096;
  while (c < b) c <<= 1;
  return c;
}
void trimDevice(BlockCache& c, int device) {  // caller holds c.mu and has device current
  for (auto it = c.blocks.begin(); it != c.blocks.end();) {
    if (it->first.first == device) {
      for (void* p : it->second) cudaFree(p);
      it = c.blocks.erase(it);
    } else {
      ++it;
    }
  }
  c.cached[device] = 0;
}
}  // namespace blockcache

void* deviceAlloc(size_t bytes, const char* what) {
  using namespace blockcache;
  int device = 0;
  ck(cudaGetDevice(&device), "cudaGetDevice");
  const size_t sz = sizeClass(bytes);
  BlockCache& c = blockCache();
  std::lock_guard<std::mutex> lock(c.mu);
  auto it = c.blocks.find({device, sz});
  if (it != c.blocks.end() && !it->second.empty()) {
    void* p = it->second.back();
    it->second.pop_back();
    c.cached[device] -= sz;
    return p;
  }
  void* p = nullptr;
  if (cudaMalloc(&p, sz) != cudaSuccess) {
    cudaGetLastError();  // clear the allocation error before retrying
    trimDevice(c, device);
    ck(cudaMalloc(&p, sz), what);
  }
  return p;
}

void deviceRelease(int device, void* p, size_t bytes) {
  using namespace blockcache;
  if (!p) return;
  const size_t sz = sizeClass(bytes);
  BlockCache& c = blockCache();
  std::lock_guard<std::mutex> lock(c.mu);
  if (c.cached[device] + sz > kCacheCap) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    cudaFree(p);
    cudaSetDevice(cur);
    return;
  }
  c.blocks[{device, sz}].push_back(p);
  c.cached[device] += sz;
}

std::vector<double> hostRates(const LoweredSystem& L, const std::vector<dcomp>& psi) {
  std::vector<double> r(L.jumps.size());
  for (size_t m = 0; m < L.jumps.size(); ++m) {
    if (!L.weights[m].empty()) {
      double s = 0;
      for (int64_t i = 0; i < L.D; ++i) s += L.weights[m][i] * std::norm(psi[i]);
      r[m] = s;
    } else {
      const auto& J = L.jumps[m];
      double s = 0;
      for (int64_t i = 0; i < L.D; ++i) {
        dcomp acc = 0;
        for (int k = 0; k < J.S; ++k) acc += J.val[k * L.D + i] * psi[J.col[k * L.D + i]];
        s += std::norm(acc);
      }
      r[m] = s;
    }
  }
  return r;
}

double initialDtTry(const cqg_system& s, const std::vector<dcomp>& psi, const cqg_mcwf_pars& p, bool* overshot) {
  double dt0 = p.dt_init > 0 ? p.dt_init : 1. / (10. * s.L.highestFrequency);
  *overshot = false;
  // MCWF_Trajectory constructor: dpLimit should not be overshot at startup either
  if (p.noise && !s.L.jumps.empty()) {
    double totalRate = 0.;
    for (double r : hostRates(s.L, psi)) totalRate += r;
    const double suggested = p.dp_limit / totalRate;
    *overshot = totalRate * dt0 > p.dp_limit;
    dt0 = s.L.hasH ? std::min(dt0, suggested) : suggested;
  }
  return dt0;
}

}  // namespace engine
}  // namespace cqg

namespace {

template <typename T>
void upload(void* base, size_t off, const std::vector<T>& v) {
  if (!v.empty()) ck(cudaMemcpy(static_cast<char*>(base) + off, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
}

std::vector<double2> toD2(const std::vector<dcomp>& v) {
  std::vector<double2> r(v.size());
  for (size_t i = 0; i < v.size(); ++i) r[i] = make_double2(v[i].real(), v[i].imag());
  return r;
}
std::vector<float2> toF2(const std::vector<dcomp>& v) {
  std::vector<float2> r(v.size());
  for (size_t i = 0; i < v.size(); ++i) r[i] = make_float2(float(v[i].real()), float(v[i].imag()));
  return r;
}

// Twiddle factors of the position averages' radix-2 transform: tw[k] = exp(2 pi i k / N),
// k < N / 2, with the same sincospi the transform's butterflies would call (the butterfly of
// span len at position pos reads tw[pos N / len]: the argument 2 pos / len = 2 k / N exactly).
__global__ void twiddleKernel(double2* tw, int N) {
  for (int k = threadIdx.x; k < N / 2; k += blockDim.x) {
    double s, c;
    sincospi(double(2 * k) / double(N), &s, &c);
    tw[k] = make_double2(c, s);
  }
}

void buildSystemDevice(cqg_system& s) {
  const auto& L = s.L;
  const int64_t D = L.D;
  Arena A;
  const int nJ = int(L.jumps.size()), nObs = int(L.obs.size());
  int SJ = 0, SO = 0;
  for (auto& j : L.jumps) SJ = std::max(SJ, j.S);
  for (auto& o : L.obs) SO = std::max(SO, o.S);
  // pack jump and observable tables to common slot counts
  std::vector<int> jcol(size_t(nJ) * SJ * D), ocol(size_t(nObs) * SO * D);
  std::vector<dcomp> jval(size_t(nJ) * SJ * D), oval(size_t(nObs) * SO * D);
  std::vector<double> jw(size_t(nJ) * D, 0.);
  std::vector<int> jHasW(nJ), oRe(nObs), oIm(nObs), oS(nObs), oF(nObs, 0);
  for (int k : L.fourierObs) oF[k] = 1;
  for (int m = 0; m < nJ; ++m) {
    const auto& J = L.jumps[m];
    for (int k = 0; k < SJ; ++k)
      for (int64_t r = 0; r < D; ++r) {
        const size_t o = (size_t(m) * SJ + k) * D + r;
        jcol[o] = k < J.S ? J.col[k * D + r] : int(r);
        jval[o] = k < J.S ? J.val[k * D + r] : dcomp(0, 0);
      }
    jHasW[m] = L.weights[m].empty() ? 0 : 1;
    if (jHasW[m]) std::copy(L.weights[m].begin(), L.weights[m].end(), jw.begin() + size_t(m) * D);
  }
  for (int q = 0; q < nObs; ++q) {
    const auto& O = L.obs[q];
    for (int k = 0; k < SO; ++k)
      for (int64_t r = 0; r < D; ++r) {
        const size_t o = (size_t(q) * SO + k) * D + r;
        ocol[o] = k < O.S ? O.col[k * D + r] : int(r);
        oval[o] = k < O.S ? O.val[k * D + r] : dcomp(0, 0);
      }
    oRe[q] = L.obsColRe[q];
    oIm[q] = L.obsColIm[q];
    oS[q] = O.S;
  }
  const auto& H = L.ham;
  const int S = H.S;
  // Interaction-picture frequencies as a table of their distinct nonzero values (compared
  // bit for bit) and an index per slot and row (kNoPhase for a zero frequency), when there
  // are at most kPhaseTableMax distinct values: the kernels then form one exponential per
  // value instead of one per row and slot.
  std::vector<dcomp> fDist;
  std::vector<unsigned short> fIdx;
  if (!H.freq.empty()) {
    std::map<std::pair<uint64_t, uint64_t>, int> seen;
    fIdx.resize(H.freq.size());
    for (size_t i = 0; i < H.freq.size(); ++i) {
      const double re = H.freq[i].real(), im = H.freq[i].imag();
      if (re == 0. && im == 0.) {
        fIdx[i] = dev::kNoPhase;
        continue;
      }
      std::pair<uint64_t, uint64_t> key;
      std::memcpy(&key.first, &re, 8);
      std::memcpy(&key.second, &im, 8);
      auto it = seen.find(key);
      if (it == seen.end()) {
        if (fDist.size() == size_t(dev::kPhaseTableMax)) {
          fDist.clear();
          fIdx.clear();
          break;
        }
        it = seen.emplace(key, int(fDist.size())).first;
        fDist.push_back(H.freq[i]);
      }
      fIdx[i] = static_cast<unsigned short>(it->second);
    }
  }
  // The CTA kernel's packed slot records (see SysDev::ctaWord)
  const bool ctaRecords = D < 32768;
  std::vector<int> ctaWord;
  std::vector<int4> ctaRecF;
  if (ctaRecords && S > 0) {
    ctaWord.resize(size_t(S) * D);
    ctaRecF.resize(size_t(S) * D);
    for (int k = 0; k < S; ++k)
      for (int64_t r = 0; r < D; ++r) {
        const size_t o = size_t(k) * D + r;
        const int off = H.col[o] - int(r);
        const unsigned fi = fIdx.empty() ? unsigned(dev::kNoPhase) : unsigned(fIdx[o]);
        const unsigned word = (fi << 16) | (unsigned(off) & 0xffffu);
        ctaWord[o] = int(word);
        const float vx = float(H.val[o].real()), vy = float(H.val[o].imag());
        int4 rec;
        std::memcpy(&rec.x, &vx, 4);
        std::memcpy(&rec.y, &vy, 4);
        rec.z = int(word);
        rec.w = 0;
        ctaRecF[o] = rec;
      }
  }
  const size_t oCtaWord = A.add(ctaWord.size() * 4 + 16), oCtaRecF = A.add(ctaRecF.size() * 16 + 16);
  const int nTw = L.fourierObs.empty() ? 0 : int(L.fourierN / 2);
  const size_t oFTw = A.add(size_t(nTw) * 16 + 16);
  // The warp kernel's padded copies of the hot tables (see SysDev::wcol): rows to
  // Dp = 32 ceil(D / 32), slots to kWarpSlots, zero coefficients on the row itself.
  const bool warpTables = D <= kWarpKernelMaxD && S <= dev::kWarpSlots;
  const int64_t Dp = (D + 31) / 32 * 32, WS = dev::kWarpSlots;
  std::vector<int> wcol;
  std::vector<dcomp> wdiag, wval, wlambda, wfreq;
  std::vector<double> wjw;
  std::vector<unsigned short> wfIdx;
  if (warpTables) {
    wcol.resize(size_t(WS * Dp));
    wval.assign(size_t(WS * Dp), dcomp(0, 0));
    wdiag.assign(size_t(Dp), dcomp(0, 0));
    wjw.assign(size_t(nJ) * size_t(Dp), 0.);
    for (int64_t r = 0; r < Dp; ++r) {
      if (r < D) wdiag[r] = H.diag[r];
      for (int64_t k = 0; k < WS; ++k) {
        const bool real = r < D && k < S;
        wcol[k * Dp + r] = real ? H.col[k * D + r] : int(r);
        if (real) wval[k * Dp + r] = H.val[k * D + r];
      }
    }
    for (int m = 0; m < nJ; ++m)
      for (int64_t r = 0; r < D; ++r) wjw[size_t(m) * Dp + r] = jw[size_t(m) * D + r];
    if (!L.lambda.empty()) {
      wlambda.assign(size_t(Dp), dcomp(0, 0));
      for (int64_t r = 0; r < D; ++r) wlambda[r] = L.lambda[r];
    }
    if (!H.freq.empty()) {
      wfreq.assign(size_t(WS * Dp), dcomp(0, 0));
      for (int64_t k = 0; k < S; ++k)
        for (int64_t r = 0; r < D; ++r) wfreq[k * Dp + r] = H.freq[k * D + r];
    }
    if (!fIdx.empty()) {
      wfIdx.assign(size_t(WS * Dp), dev::kNoPhase);
      for (int64_t k = 0; k < S; ++k)
        for (int64_t r = 0; r < D; ++r) wfIdx[k * Dp + r] = fIdx[k * D + r];
    }
  }
  const size_t oWcol = A.add(wcol.size() * 4 + 4), oWdiagD = A.add(wdiag.size() * 16 + 16),
               oWvalD = A.add(wval.size() * 16 + 16), oWdiagF = A.add(wdiag.size() * 8 + 8),
               oWvalF = A.add(wval.size() * 8 + 8), oWjw = A.add(wjw.size() * 8 + 8),
               oWlambda = A.add(wlambda.size() * 16 + 16), oWfIdx = A.add(wfIdx.size() * 2 + 16),
               oWfreq = A.add(wfreq.size() * 16 + 16);
  const size_t oCol = A.add(H.col.size() * 4 + 4), oJcol = A.add(jcol.size() * 4 + 4), oJw = A.add(jw.size() * 8 + 8),
               oJHasW = A.add(jHasW.size() * 4 + 4), oOcol = A.add(ocol.size() * 4 + 4),
               oOval = A.add(oval.size() * 16 + 16), oORe = A.add(oRe.size() * 4 + 4), oOIm = A.add(oIm.size() * 4 + 4), oOS = A.add(oS.size() * 4 + 4),
               oOF = A.add(oF.size() * 4 + 4), oFW = A.add(L.fourierW.size() * 8 + 8),
               oFreq = A.add(H.freq.size() * 16 + 16), oLambda = A.add(L.lambda.size() * 16 + 16),
               oFIdx = A.add(fIdx.size() * 2 + 16), oFDist = A.add(fDist.size() * 16 + 16),
               oDiagD = A.add(H.diag.size() * 16 + 16), oValD = A.add(H.val.size() * 16 + 16),
               oJvalD = A.add(jval.size() * 16 + 16), oDiagF = A.add(H.diag.size() * 8 + 8),
               oValF = A.add(H.val.size() * 8 + 8), oJvalF = A.add(jval.size() * 8 + 8);
  ck(cudaMalloc(&s.dmem, A.total), "cudaMalloc(system)");
  char* b = static_cast<char*>(s.dmem);
  upload(b, oCol, H.col);
  upload(b, oJcol, jcol);
  upload(b, oJw, jw);
  upload(b, oJHasW, jHasW);
  upload(b, oOcol, ocol);
  upload(b, oOval, toD2(oval));
  upload(b, oORe, oRe);
  upload(b, oOIm, oIm);
  upload(b, oOS, oS);
  upload(b, oOF, oF);
  upload(b, oFW, L.fourierW);
  upload(b, oFreq, toD2(H.freq));
  upload(b, oFIdx, fIdx);
  upload(b, oFDist, toD2(fDist));
  upload(b, oLambda, toD2(L.lambda));
  upload(b, oDiagD, toD2(H.diag));
  upload(b, oValD, toD2(H.val));
  upload(b, oJvalD, toD2(jval));
  upload(b, oDiagF, toF2(H.diag));
  upload(b, oValF, toF2(H.val));
  upload(b, oJvalF, toF2(jval));
  upload(b, oCtaWord, ctaWord);
  upload(b, oCtaRecF, ctaRecF);
  upload(b, oWcol, wcol);
  upload(b, oWdiagD, toD2(wdiag));
  upload(b, oWvalD, toD2(wval));
  upload(b, oWdiagF, toF2(wdiag));
  upload(b, oWvalF, toF2(wval));
  upload(b, oWjw, wjw);
  upload(b, oWlambda, toD2(wlambda));
  upload(b, oWfIdx, wfIdx);
  upload(b, oWfreq, toD2(wfreq));
  auto& sd = s.sd;
  sd.D = int(D);
  sd.S = S;
  sd.SJ = SJ;
  sd.SO = SO;
  sd.nJ = nJ;
  sd.nObs = nObs;
  sd.nAvr = L.nAvr;
  sd.hasH = L.hasH ? 1 : 0;
  sd.hasEx = L.hasEx ? 1 : 0;
  sd.hasFreq = H.freq.empty() ? 0 : 1;
  sd.col = reinterpret_cast<const int*>(b + oCol);
  sd.jcol = reinterpret_cast<const int*>(b + oJcol);
  sd.jw = reinterpret_cast<const double*>(b + oJw);
  sd.jHasW = reinterpret_cast<const int*>(b + oJHasW);
  sd.ocol = reinterpret_cast<const int*>(b + oOcol);
  sd.oval = reinterpret_cast<const double2*>(b + oOval);
  sd.oRe = reinterpret_cast<const int*>(b + oORe);
  sd.oIm = reinterpret_cast<const int*>(b + oOIm);
  sd.oS = reinterpret_cast<const int*>(b + oOS);
  sd.oFourier = reinterpret_cast<const int*>(b + oOF);
  sd.fW = reinterpret_cast<const double*>(b + oFW);
  sd.nF = int(L.fourierObs.size());
  sd.fN = int(L.fourierN);
  sd.fStride = int(L.fourierStride);
  sd.fLog2 = 0;
  while ((int64_t(1) << sd.fLog2) < L.fourierN) ++sd.fLog2;
  for (int k = 0; k < 4; ++k) sd.fObs[k] = k < sd.nF ? L.fourierObs[size_t(k)] : -1;
  sd.freq = H.freq.empty() ? nullptr : reinterpret_cast<const double2*>(b + oFreq);
  sd.nFD = int(fDist.size());
  sd.fIdx = fIdx.empty() ? nullptr : reinterpret_cast<const unsigned short*>(b + oFIdx);
  sd.fDist = fDist.empty() ? nullptr : reinterpret_cast<const double2*>(b + oFDist);
  sd.lambda = L.lambda.empty() ? nullptr : reinterpret_cast<const double2*>(b + oLambda);
  sd.diagD = reinterpret_cast<const double2*>(b + oDiagD);
  sd.valD = reinterpret_cast<const double2*>(b + oValD);
  sd.jvalD = reinterpret_cast<const double2*>(b + oJvalD);
  sd.diagF = reinterpret_cast<const float2*>(b + oDiagF);
  sd.valF = reinterpret_cast<const float2*>(b + oValF);
  sd.jvalF = reinterpret_cast<const float2*>(b + oJvalF);
  sd.diagZero = 1;
  for (const auto& v : H.diag)
    if (v != dcomp(0, 0)) sd.diagZero = 0;
  sd.ctaWord = ctaWord.empty() ? nullptr : reinterpret_cast<const int*>(b + oCtaWord);
  sd.ctaRecF = ctaRecF.empty() ? nullptr : reinterpret_cast<const int4*>(b + oCtaRecF);
  sd.Dp = warpTables ? int(Dp) : 0;
  sd.wcol = warpTables ? reinterpret_cast<const int*>(b + oWcol) : nullptr;
  sd.wdiagD = warpTables ? reinterpret_cast<const double2*>(b + oWdiagD) : nullptr;
  sd.wvalD = warpTables ? reinterpret_cast<const double2*>(b + oWvalD) : nullptr;
  sd.wdiagF = warpTables ? reinterpret_cast<const float2*>(b + oWdiagF) : nullptr;
  sd.wvalF = warpTables ? reinterpret_cast<const float2*>(b + oWvalF) : nullptr;
  sd.wjw = warpTables ? reinterpret_cast<const double*>(b + oWjw) : nullptr;
  sd.wlambda = wlambda.empty() ? nullptr : reinterpret_cast<const double2*>(b + oWlambda);
  sd.wfIdx = wfIdx.empty() ? nullptr : reinterpret_cast<const unsigned short*>(b + oWfIdx);
  sd.wfreq = wfreq.empty() ? nullptr : reinterpret_cast<const double2*>(b + oWfreq);
  sd.fTw = nullptr;
  if (nTw > 0) {
    double2* tw = reinterpret_cast<double2*>(b + oFTw);
    twiddleKernel<<<1, 256>>>(tw, int(L.fourierN));
    ck(cudaGetLastError(), "twiddle kernel launch");
    ck(cudaStreamSynchronize(0), "twiddle kernel");
    sd.fTw = tw;
  }
}

// ---- kernel dispatch -------------------------------------------------------------

using KernelFn = void (*)(dev::TrajDev, dev::RunArgs);

}  // namespace

namespace cqg {
namespace dev {
KernelFn pick_double_e1_ip0(int smax, bool highOccupancy);
KernelFn pick_double_e1_ip1(int smax, bool highOccupancy);
KernelFn pick_double_e2_ip0(int smax, bool highOccupancy);
KernelFn pick_double_e2_ip1(int smax, bool highOccupancy);
KernelFn pick_double_e3_ip0(int smax, bool highOccupancy);
KernelFn pick_double_e3_ip1(int smax, bool highOccupancy);
KernelFn pick_double_e4_ip0(int smax, bool highOccupancy);
KernelFn pick_double_e4_ip1(int smax, bool highOccupancy);
KernelFn pick_float_e1_ip0(int smax, bool highOccupancy);
KernelFn pick_float_e1_ip1(int smax, bool highOccupancy);
KernelFn pick_float_e2_ip0(int smax, bool highOccupancy);
KernelFn pick_float_e2_ip1(int smax, bool highOccupancy);
KernelFn pick_float_e3_ip0(int smax, bool highOccupancy);
KernelFn pick_float_e3_ip1(int smax, bool highOccupancy);
KernelFn pick_float_e4_ip0(int smax, bool highOccupancy);
KernelFn pick_float_e4_ip1(int smax, bool highOccupancy);
}  // namespace dev
}  // namespace cqg

namespace {

}  // namespace

namespace cqg {
namespace dev {
using BlockKernelFn = void (*)(TrajDev, RunArgs, BlockScratch, int);
BlockKernelFn pick_block(bool fp64, bool ip);
}  // namespace dev
}  // namespace cqg

namespace {


int tunedThreads(const cqg_ensemble& e, size_t gi, const cqg_system* const* systems, int nSys,
                 const cqg_complex* psi0s, const int64_t* psi0Off, const cqg_mcwf_pars& pars);
bool sharedVectorsFit(const KernelGroup& g, size_t elemBytes, int device);

KernelFn pickKernel(bool fp64, int E, int SMAX, bool ip, bool hi) {
  using P = KernelFn (*)(int, bool);
  static const P table[2][4][2] = {
      {{dev::pick_double_e1_ip0, dev::pick_double_e1_ip1}, {dev::pick_double_e2_ip0, dev::pick_double_e2_ip1},
       {dev::pick_double_e3_ip0, dev::pick_double_e3_ip1}, {dev::pick_double_e4_ip0, dev::pick_double_e4_ip1}},
      {{dev::pick_float_e1_ip0, dev::pick_float_e1_ip1}, {dev::pick_float_e2_ip0, dev::pick_float_e2_ip1},
       {dev::pick_float_e3_ip0, dev::pick_float_e3_ip1}, {dev::pick_float_e4_ip0, dev::pick_float_e4_ip1}}};
  return table[fp64 ? 0 : 1][std::min(std::max(E, 1), 4) - 1][ip ? 1 : 0](SMAX, hi);
}

__global__ void reduceAveragesKernel(const double* __restrict__ avr, int nTraj, int nAvrStride, int nAvr,
                                     double* __restrict__ sums) {
  // one block per (output, column): fixed-order strided sums then a fixed tree
  const int k = blockIdx.x / nAvr, c = blockIdx.x % nAvr;
  __shared__ double part[256];
  double acc = 0.;
  for (int i = threadIdx.x; i < nTraj; i += blockDim.x) acc += avr[((size_t)k * nTraj + i) * nAvrStride + c];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[(size_t)k * nAvr + c] = part[0];
}

// Initial states: trajectory i's slot (dimension from the slot offsets) receives a copy of its
// distinct initial state, which the host uploaded once; 8-byte words.
__global__ void replicateStatesKernel(const unsigned long long* __restrict__ uniq, const long long* __restrict__ uOff,
                                      const long long* __restrict__ psiOff, long long nTraj, long long psiElems,
                                      int wordsPerElem, unsigned long long* __restrict__ psi) {
  for (long long i = blockIdx.x; i < nTraj; i += gridDim.x) {
    const long long D = (i + 1 < nTraj ? psiOff[i + 1] : psiElems) - psiOff[i];
    const long long n = D * wordsPerElem;
    const unsigned long long* src = uniq + uOff[i] * wordsPerElem;
    unsigned long long* dst = psi + psiOff[i] * wordsPerElem;
    for (long long k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
  }
}

__global__ void statusOrKernel(const unsigned* __restrict__ st, int n, unsigned* out) {
  unsigned v = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v |= st[i];
  v = __reduce_or_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && v) atomicOr(out, v);
}

int createEnsemble(const cqg_system* const* systems, int nSys, const int32_t* sysIndex, const cqg_complex* psi0s,
                   const int64_t* psi0Off, int64_t nTraj, const cqg_mcwf_pars* pars, cqg_ensemble** out) {
  if (!systems || nSys < 1 || !psi0s || nTraj < 1 || !pars || !out)
    return fail(CQG_E_INVALID, "ensemble: null argument or empty ensemble");
  if (nTraj > (int64_t(1) << 30)) return fail(CQG_E_INVALID, "ensemble: too many trajectories");
  if (pars->precision != CQG_FP64 && pars->precision != CQG_FP32) return fail(CQG_E_INVALID, "ensemble: bad precision");
  if (pars->rng != CQG_RNG_PCG64 && pars->rng != CQG_RNG_PHILOX) return fail(CQG_E_INVALID, "ensemble: bad rng");
  if (!(pars->eps_rel > 0) || !(pars->eps_abs >= 0) || !(pars->dp_limit > 0) || !(pars->overshoot_tolerance >= 1))
    return fail(CQG_E_INVALID, "ensemble: eps_rel > 0, eps_abs >= 0, dp_limit > 0, overshoot_tolerance >= 1 required");
  auto e = std::make_unique<cqg_ensemble>();
  e->nTraj = nTraj;
  e->pars = *pars;
  if (e->pars.max_attempts <= 0) e->pars.max_attempts = 100000;
  for (int s = 0; s < nSys; ++s) {
    if (!systems[s]) return fail(CQG_E_INVALID, "ensemble: null system");
    e->systems.push_back(systems[s]);
    e->Dmax = std::max<int>(e->Dmax, int(systems[s]->L.D));
    e->Smax = std::max<int>(e->Smax, systems[s]->sd.S);
    e->nAvrMax = std::max<int>(e->nAvrMax, systems[s]->L.nAvr);
    if (int(systems[s]->L.jumps.size()) > dev::MAX_JUMPS)
      return fail(CQG_E_UNSUPPORTED, "ensemble: more than 8 jump operators");
  }
  if (int64_t(e->Dmax) * 2 * (pars->precision == CQG_FP64 ? 16 : 8) > 200 * 1024)
    return fail(CQG_E_UNSUPPORTED, "ensemble: the stage vectors of a trajectory exceed shared memory");
  if (e->Smax > kMaxSlots) return fail(CQG_E_UNSUPPORTED, "ensemble: more than 64 off-diagonal entries per row");
  e->device = systems[0]->device;
  ck(cudaSetDevice(e->device), "cudaSetDevice");
  ck(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaEventCreate(&e->ev0), "cudaEventCreate");
  ck(cudaEventCreate(&e->ev1), "cudaEventCreate");
  ck(cudaEventCreate(&e->evRun0), "cudaEventCreate");
  ck(cudaEventCreate(&e->evRun1), "cudaEventCreate");
  ck(cudaEventCreateWithFlags(&e->evFork, cudaEventDisableTiming), "cudaEventCreate");
  e->elemBytes = pars->precision == CQG_FP64 ? 16 : 8;

  e->sysIdx.resize(nTraj);
  e->psiOff.resize(nTraj);
  long long off = 0;
  for (int64_t i = 0; i < nTraj; ++i) {
    const int si = sysIndex ? sysIndex[i] : 0;
    if (si < 0 || si >= nSys) return fail(CQG_E_INVALID, "ensemble: system index out of range");
    e->sysIdx[i] = si;
    e->psiOff[i] = off;
    off += systems[si]->L.D;
  }
  const long long psiElems = off;

  // Distinct initial states: one for a single-state ensemble, one per distinct (offset,
  // dimension) in a batch.  Each is converted and sent once; a kernel copies it into the
  // slots of its trajectories.
  std::vector<int> uId(nTraj);          // trajectory i's distinct state
  std::vector<long long> uOff(nTraj);   // element offset of trajectory i's state in the list
  std::vector<int64_t> uFirst;          // a trajectory of each distinct state
  std::vector<long long> uStart;        // element offset of each distinct state in the list
  long long uniqElems = 0;
  if (!psi0Off && nSys == 1) {  // one state for the whole ensemble
    uFirst.push_back(0);
    uStart.push_back(0);
    uniqElems = systems[0]->L.D;
  } else {
    std::map<std::pair<int64_t, int64_t>, int> seen;
    for (int64_t i = 0; i < nTraj; ++i) {
      const int64_t D = systems[e->sysIdx[i]]->L.D;
      const std::pair<int64_t, int64_t> key(psi0Off ? psi0Off[i] : 0, D);
      auto it = seen.find(key);
      if (it == seen.end()) {
        it = seen.emplace(key, int(uFirst.size())).first;
        uFirst.push_back(i);
        uStart.push_back(uniqElems);
        uniqElems += D;
      }
      uId[i] = it->second;
    }
  }
  for (int64_t i = 0; i < nTraj; ++i) uOff[i] = uStart[size_t(uId[i])];

  Arena A;
  const size_t oPsi = A.add(size_t(psiElems) * e->elemBytes), oOff = A.add(nTraj * 8), oIdx = A.add(nTraj * 4),
               oT = A.add(nTraj * 8), oT0 = A.add(nTraj * 8), oTry = A.add(nTraj * 8), oDid = A.add(nTraj * 8),
               oRng = A.add(nTraj * 32), oCnt = A.add(nTraj * 64), oUOff = A.add(nTraj * 8),
               oUniq = A.add(size_t(uniqElems) * e->elemBytes), oMax = A.add(nTraj * 24), oSt = A.add(nTraj * 4),
               oJT = A.add(nTraj * e->jumpCap * 8), oJL = A.add(nTraj * e->jumpCap * 4), oJN = A.add(nTraj * 8),
               oSys = A.add(nSys * sizeof(dev::SysDev)), oQ = A.add(kMaxGroups * sizeof(int)), oOrd = A.add(nTraj * 4), oSOr = A.add(16);
  e->dmem = deviceAlloc(A.total, "cudaMalloc(ensemble)");
  e->dmemBytes = A.total;
  char* b = static_cast<char*>(e->dmem);

  // Host image of the arena from the slot offsets to the distinct initial states (offsets,
  // indices, times, random streams, counters, the states) in a pinned staging buffer, sent in
  // one copy; the trajectories' slots are filled on the device, the rest is zeroed there.
  {  // the staging buffer is held only for this block (the autotuner below creates ensembles)
  HostStaging staging(oMax - oOff);
  char* const h0 = staging.data();
  auto H = [&](size_t o) { return h0 + (o - oOff); };  // host address of arena offset o
  const long long* offs = e->psiOff.data();
  std::memcpy(H(oOff), offs, size_t(nTraj) * 8);
  std::memcpy(H(oUOff), uOff.data(), size_t(nTraj) * 8);
  std::memcpy(H(oIdx), e->sysIdx.data(), size_t(nTraj) * 4);
  auto* ht = reinterpret_cast<double*>(H(oT));
  auto* ht0 = reinterpret_cast<double*>(H(oT0));
  auto* hTry = reinterpret_cast<double*>(H(oTry));
  auto* hDid = reinterpret_cast<double*>(H(oDid));
  auto* hRng = reinterpret_cast<unsigned long long*>(H(oRng));
  auto* hCnt = reinterpret_cast<unsigned long long*>(H(oCnt));
  std::memset(hRng, 0, size_t(nTraj) * 32);
  std::memset(hCnt, 0, size_t(nTraj) * 64);
  // per distinct state: the converted state and the initial dtTry (with its overshoot flag)
  std::vector<double> uDt0(uFirst.size());
  std::vector<char> uOvershot(uFirst.size());
  {
    std::vector<dcomp> psi;
    for (size_t u = 0; u < uFirst.size(); ++u) {
      const int64_t i = uFirst[u];
      const cqg_system* s = systems[e->sysIdx[i]];
      const int64_t D = s->L.D;
      const cqg_complex* p = psi0s + (psi0Off ? psi0Off[i] : 0);
      psi.resize(D);
      for (int64_t k = 0; k < D; ++k) psi[k] = dcomp(p[k].re, p[k].im);
      char* dst = H(oUniq) + size_t(uOff[i]) * e->elemBytes;
      for (int64_t k = 0; k < D; ++k) {
        if (e->elemBytes == 16) {
          const double2 v = make_double2(psi[k].real(), psi[k].imag());
          std::memcpy(dst + k * 16, &v, 16);
        } else {
          const float2 v = make_float2(float(psi[k].real()), float(psi[k].imag()));
          std::memcpy(dst + k * 8, &v, 8);
        }
      }
      bool ov = false;
      uDt0[u] = initialDtTry(*s, psi, *pars, &ov);
      uOvershot[u] = ov ? 1 : 0;
    }
  }
  for (int64_t i = 0; i < nTraj; ++i) {
    const size_t u = size_t(uId[i]);
    const double dt0Shared = uDt0[u];
    const bool overshotShared = uOvershot[u] != 0;
    if (pars->rng == CQG_RNG_PCG64) {
      const auto g = dev::Pcg64::seeded(pars->seed, pars->prng_stream + uint64_t(i));
      hRng[4 * i + 0] = g.state.hi;
      hRng[4 * i + 1] = g.state.lo;
      hRng[4 * i + 2] = g.inc.hi;
      hRng[4 * i + 3] = g.inc.lo;
    }
    if (overshotShared) hCnt[8 * i + 4] = 1;
    ht[i] = 0.;
    ht0[i] = 0.;
    hTry[i] = dt0Shared;
    hDid[i] = 0.;
  }
  ck(cudaMemcpy(b + oOff, h0, oMax - oOff, cudaMemcpyHostToDevice), "cudaMemcpy(ensemble)");
  }
  {
    const int grid = int(std::min<int64_t>(nTraj, 148 * 8));
    replicateStatesKernel<<<grid, 128, 0, e->stream>>>(
        reinterpret_cast<const unsigned long long*>(b + oUniq), reinterpret_cast<const long long*>(b + oUOff),
        reinterpret_cast<const long long*>(b + oOff), nTraj, psiElems, int(e->elemBytes / 8),
        reinterpret_cast<unsigned long long*>(b + oPsi));
    ck(cudaGetLastError(), "replicateStatesKernel");
    ck(cudaStreamSynchronize(e->stream), "cudaStreamSynchronize");
  }
  ck(cudaMemset(b + oMax, 0, A.total - oMax), "cudaMemset");
  std::vector<dev::SysDev> sds;
  for (auto* s : e->systems) sds.push_back(s->sd);
  upload(b, oSys, sds);

  auto& td = e->td;
  td.nTraj = int(nTraj);
  td.sysIdx = reinterpret_cast<const int*>(b + oIdx);
  td.systems = reinterpret_cast<const dev::SysDev*>(b + oSys);
  td.psi = b + oPsi;
  td.psiOff = reinterpret_cast<const long long*>(b + oOff);
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
  td.jumpCap = e->jumpCap;
  e->dSystems = reinterpret_cast<dev::SysDev*>(b + oSys);
  e->dQueue = reinterpret_cast<int*>(b + oQ);
  e->dOrder = reinterpret_cast<int*>(b + oOrd);
  e->dStatusOr = reinterpret_cast<unsigned*>(b + oSOr);
  // kernel groups: CTA-per-trajectory for D > 128, else warp-per-trajectory by rows per
  // lane; heavier groups first, and inside a group the longest trajectories first
  // (dimension as the cost proxy) for its work queue
  auto trajKey = [&](int64_t i) {
    const cqg_system* sy = systems[e->sysIdx[i]];
    return groupKey(sy->L.D, sy->sd.S);
  };
  std::vector<int> order(nTraj);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
    const int ka = trajKey(a), kc = trajKey(c);
    if (ka != kc) return ka > kc;
    return systems[e->sysIdx[a]]->L.D > systems[e->sysIdx[c]]->L.D;
  });
  for (int64_t k = 0; k < nTraj;) {
    KernelGroup g;
    const int key = trajKey(order[k]);
    g.kind = key == kMaxGroups ? 1 : 0;
    g.E = g.kind ? 0 : key;
    g.first = k;
    for (; k < nTraj && trajKey(order[k]) == key; ++k) {
      const cqg_system* s = systems[e->sysIdx[order[k]]];
      g.Dmax = std::max<int>(g.Dmax, int(s->L.D));
      g.smax = std::max(g.smax, s->sd.S);
      g.anyFreq |= s->sd.hasFreq != 0;
      g.phaseElems = std::max(g.phaseElems, blockPhaseElems(s->sd));
    }
    g.count = k - g.first;
    e->groups.push_back(g);
  }
  upload(b, oOrd, order);
  for (auto& g : e->groups) {
    if (e->groups.size() > 1) {
      ck(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking), "cudaStreamCreate");
      ck(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming), "cudaEventCreate");
    }
    g.threads = pars->cta_threads > 0 ? pars->cta_threads : defaultThreads(g);
    if (g.threads % 32 || g.threads < 32 || g.threads > (g.kind ? 512 : 128))
      return fail(CQG_E_INVALID, "ensemble: cta_threads must be a multiple of 32, at most 128 (warp kernel) or 512");
    g.smemVectors = pars->cta_threads > 0 && pars->cta_shared_vectors && sharedVectorsFit(g, e->elemBytes, e->device);
    g.highOccupancy = g.kind == 0 && pars->cta_threads > 0 && pars->cta_shared_vectors &&
                      dev::warpHighOccupancyVariant(g.E, g.smax <= 2 ? 2 : g.smax <= 3 ? 3 : g.smax <= 4 ? 4 : 8,
                                                    g.anyFreq);
    g.phaseTable = pars->ip_phase_table >= 0;
    if (!g.phaseTable || g.kind == 0) g.phaseElems = 0;
  }
  if (pars->autotune && pars->cta_threads <= 0)
    for (size_t gi = 0; gi < e->groups.size(); ++gi) {
      const int shape = tunedThreads(*e, gi, systems, nSys, psi0s, psi0Off, *pars);
      e->groups[gi].threads = shape & 0xffff;
      e->groups[gi].smemVectors = (shape & (1 << 16)) != 0;
      e->groups[gi].highOccupancy = (shape & kHighOccupancyFlag) != 0 && e->groups[gi].kind == 0 &&
                                    !e->groups[gi].anyFreq;
    }
  *out = e.release();
  return CQG_OK;
}

}  // namespace

namespace cqg {
namespace engine {

void launchGroup(bool fp64, size_t elemBytes, const dev::TrajDev& td, KernelGroup& g, dev::RunArgs ra, int nSM,
                 cudaStream_t st) {
  dev::TrajDev tdArg = td;
  if (g.kind == 0) {
    KernelFn fn = pickKernel(fp64, g.E, g.smax, g.anyFreq, g.highOccupancy);
    const int warps = g.threads / 32;
    // stage vectors, warp scratch, and for interaction-picture systems the phase tables
    ra.phaseCache = g.anyFreq && g.phaseTable ? 1 : 0;
    const size_t smem = size_t(warps) * dev::warpSmemVectors(g.E) * 32 * g.E * elemBytes +
                        size_t(warps) * sizeof(dev::WarpScratch) +
                        (ra.phaseCache ? size_t(warps) * dev::kWarpPhaseElems * sizeof(double2) : 0);
    ck(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
       "cudaFuncSetAttribute");
    int perSM = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, reinterpret_cast<const void*>(fn), g.threads, smem),
       "occupancy");
    int grid = int(std::min<int64_t>(int64_t(std::max(perSM, 1)) * nSM, (g.count + warps - 1) / warps));
    grid = std::max(grid, 1);
    if (g.count <= int64_t(grid) * warps) ra.yieldSteps = 0;  // one wave: nothing to balance
    void* args[] = {&tdArg, &ra};
    ck(cudaLaunchKernel(reinterpret_cast<const void*>(fn), dim3(grid), dim3(g.threads), args, smem, st),
       "kernel launch");
  } else {
    // one CTA per trajectory: stage vectors in shared memory, stage derivatives in a
    // per-CTA scratch slab or, when the group says so, in shared memory too
    dev::BlockKernelFn fn = dev::pick_block(fp64, g.anyFreq);
    int smemD = g.Dmax;
    if (g.phaseElems > 0) {  // a phase table that does not fit leaves the phases per row and slot
      int device = 0, optin = 0;
      ck(cudaGetDevice(&device), "cudaGetDevice");
      ck(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device), "attribute");
      if (blockSmemBytes(g.Dmax, elemBytes, g.smemVectors, g.phaseElems) > size_t(optin)) g.phaseElems = 0;
    }
    const size_t smem = blockSmemBytes(g.Dmax, elemBytes, g.smemVectors, g.phaseElems);
    ck(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
       "cudaFuncSetAttribute");
    int perSM = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, reinterpret_cast<const void*>(fn), g.threads, smem),
       "occupancy");
    int grid = int(std::min<int64_t>(int64_t(std::max(perSM, 1)) * nSM, g.count));
    grid = std::max(grid, 1);
    dev::BlockScratch bsc;
    bsc.stride = (g.Dmax + 31) / 32 * 32;
    bsc.base = nullptr;
    bsc.phaseElems = g.phaseElems;
    if (!g.smemVectors) {
      const size_t need = size_t(grid) * dev::kBlockVectors * size_t(bsc.stride) * elemBytes;
      if (need > g.scratchBytes) {
        int device = 0;
        ck(cudaGetDevice(&device), "cudaGetDevice");
        if (g.scratch) {
          ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
          deviceRelease(device, g.scratch, g.scratchBytes);
        }
        g.scratch = nullptr;
        g.scratchBytes = 0;
        g.scratch = deviceAlloc(need, "cudaMalloc(block scratch)");
        g.scratchBytes = need;
      }
      bsc.base = g.scratch;
    }
    void* args[] = {&tdArg, &ra, &bsc, &smemD};
    ck(cudaLaunchKernel(reinterpret_cast<const void*>(fn), dim3(grid), dim3(g.threads), args, smem, st),
       "kernel launch");
  }
}

}  // namespace engine
}  // namespace cqg

namespace {

int launchRun(cqg_ensemble* e, dev::RunArgs ra, int nOut, double* avrHost) {
  ck(cudaSetDevice(e->device), "cudaSetDevice");
  const int nAvr = e->nAvrMax + 1;  // the linear averages, then dtDid
  const size_t need = size_t(std::max(nOut, 1)) * e->nTraj * nAvr;
  if (need > e->avrCap) {
    ck(cudaStreamSynchronize(e->stream), "cudaStreamSynchronize");
    cqg::engine::deviceRelease(e->device, e->dAvr, e->avrCap * sizeof(double));
    e->dAvr = nullptr;
    e->avrCap = 0;
    e->dAvr = static_cast<double*>(cqg::engine::deviceAlloc(need * sizeof(double), "cudaMalloc(averages)"));
    e->avrCap = need;
  }
  const size_t needS = size_t(std::max(nOut, 1)) * nAvr;
  if (needS > e->sumsCap) {
    ck(cudaStreamSynchronize(e->stream), "cudaStreamSynchronize");
    cqg::engine::deviceRelease(e->device, e->dSums, e->sumsCap * sizeof(double));
    e->dSums = nullptr;
    e->sumsCap = 0;
    e->dSums = static_cast<double*>(cqg::engine::deviceAlloc(needS * sizeof(double), "cudaMalloc(sums)"));
    e->sumsCap = needS;
  }
  ck(cudaEventRecord(e->evRun0, e->stream), "cudaEventRecord");
  ck(cudaMemsetAsync(e->dAvr, 0, need * sizeof(double), e->stream), "cudaMemsetAsync");
  ck(cudaMemsetAsync(e->dQueue, 0, kMaxGroups * sizeof(int), e->stream), "cudaMemsetAsync");
  ck(cudaMemsetAsync(e->dStatusOr, 0, sizeof(unsigned), e->stream), "cudaMemsetAsync");
  ra.avrOut = e->dAvr;
  ra.nAvrStride = nAvr;
  ra.absSlot = e->pars.eps_rel;  // make_controlled(epsRel, epsAbs, ...) (ODE.h:205)
  ra.relSlot = e->pars.eps_abs;
  ra.dpLimit = e->pars.dp_limit;
  ra.overTol = e->pars.overshoot_tolerance;
  ra.maxAttempts = e->pars.max_attempts;
  ra.noise = e->pars.noise;
  ra.rng = e->pars.rng;
  ra.seed = e->pars.seed;
  ra.maxStepsPerInterval = 2000000000LL;
  ra.timeLimitNs = 120ull * 1000000000ull;

  int nSM = 0;
  ck(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, e->device), "attribute");
  // warp groups hand their trajectories back to the queue every yield_steps MCWF steps
  const int yieldSteps = ra.mode == dev::RUN_STEPS || e->pars.yield_steps < 0 ? 0
                         : e->pars.yield_steps > 0                           ? e->pars.yield_steps
                                                                              : kDefaultYieldSteps;
  if (yieldSteps > 0 && !e->dYield) {
    size_t off = 0;
    const size_t nG = e->groups.size();
    e->yieldHead.assign(nG, 0);
    e->yieldSeq.assign(nG, 0);
    e->yieldEntry.assign(nG, 0);
    e->yieldCap.assign(nG, 0);
    for (size_t gi = 0; gi < nG; ++gi) {
      e->yieldCap[gi] = int(std::min<int64_t>(e->groups[gi].count * kYieldSlotsPerTrajectory, int64_t(1) << 28));
      e->yieldHead[gi] = off;
      off += 16;
    }
    for (size_t gi = 0; gi < nG; ++gi) {
      e->yieldSeq[gi] = off;
      off += size_t(e->yieldCap[gi]) * 4;
    }
    off = (off + 15) / 16 * 16;
    e->yieldResume = off;
    off += size_t(e->nTraj) * sizeof(dev::ResumeInfo);
    e->yieldZeroBytes = off;
    for (size_t gi = 0; gi < nG; ++gi) {
      e->yieldEntry[gi] = off;
      off += size_t(e->yieldCap[gi]) * 4;
    }
    e->dYield = deviceAlloc(off, "cudaMalloc(yield queues)");
    e->yieldBytes = off;
  }
  if (yieldSteps > 0) ck(cudaMemsetAsync(e->dYield, 0, e->yieldZeroBytes, e->stream), "cudaMemsetAsync");
  ck(cudaEventRecord(e->ev0, e->stream), "cudaEventRecord");
  const bool fork = e->groups.size() > 1;
  if (fork) ck(cudaEventRecord(e->evFork, e->stream), "cudaEventRecord");
  for (size_t gi = 0; gi < e->groups.size(); ++gi) {
    KernelGroup& g = e->groups[gi];
    cudaStream_t st = fork ? g.stream : e->stream;
    if (fork) ck(cudaStreamWaitEvent(st, e->evFork, 0), "cudaStreamWaitEvent");
    ra.order = e->dOrder + g.first;
    ra.nTasks = int(g.count);
    ra.queue = e->dQueue + gi;
    // by default only the Schroedinger-picture instance yields: the interaction-picture one
    // measured 4.5 % slower with yielding on (qubit-mode 2x40, detuned), even with chunks
    // longer than its trajectories' steps per launch
    ra.yieldSteps = g.kind == 0 && (e->pars.yield_steps > 0 || !g.anyFreq) ? yieldSteps : 0;
    if (ra.yieldSteps > 0) {
      char* y = static_cast<char*>(e->dYield);
      int* head = reinterpret_cast<int*>(y + e->yieldHead[gi]);
      ra.yieldTail = head;
      ra.doneCount = head + 1;
      ra.queueError = reinterpret_cast<unsigned*>(head + 2);
      ra.yieldSeq = reinterpret_cast<int*>(y + e->yieldSeq[gi]);
      ra.yieldEntry = reinterpret_cast<int*>(y + e->yieldEntry[gi]);
      ra.yieldCap = e->yieldCap[gi];
      ra.resume = reinterpret_cast<dev::ResumeInfo*>(y + e->yieldResume);
    }
    launchGroup(e->pars.precision == CQG_FP64, e->elemBytes, e->td, g, ra, nSM, st);
    if (fork) {
      ck(cudaEventRecord(g.done, st), "cudaEventRecord");
      ck(cudaStreamWaitEvent(e->stream, g.done, 0), "cudaStreamWaitEvent");
    }
  }
  ck(cudaEventRecord(e->ev1, e->stream), "cudaEventRecord");
  if (nAvr > 0 && nOut > 0) {
    reduceAveragesKernel<<<nOut * nAvr, 256, 0, e->stream>>>(e->dAvr, int(e->nTraj), ra.nAvrStride, nAvr, e->dSums);
    ck(cudaGetLastError(), "reduce launch");
  }
  statusOrKernel<<<std::max(1, std::min(148, int((e->nTraj + 255) / 256))), 256, 0, e->stream>>>(
      e->td.status, int(e->nTraj), e->dStatusOr);
  ck(cudaGetLastError(), "status launch");
  unsigned bits = 0;
  ck(cudaMemcpyAsync(&bits, e->dStatusOr, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream), "cudaMemcpyAsync");
  std::vector<int> yieldHeads(yieldSteps > 0 ? 4 * e->groups.size() : 0);
  for (size_t gi = 0; gi < e->groups.size() && yieldSteps > 0; ++gi)
    ck(cudaMemcpyAsync(&yieldHeads[4 * gi], static_cast<char*>(e->dYield) + e->yieldHead[gi], 16,
                       cudaMemcpyDeviceToHost, e->stream),
       "cudaMemcpyAsync");
  std::vector<double> sums;
  if (avrHost && nAvr > 0 && nOut > 0) {
    ck(cudaMemcpyAsync(avrHost, e->dSums, size_t(nOut) * nAvr * sizeof(double), cudaMemcpyDeviceToHost, e->stream),
       "cudaMemcpyAsync");
  }
  ck(cudaEventRecord(e->evRun1, e->stream), "cudaEventRecord");
  ck(cudaStreamSynchronize(e->stream), "kernel execution");
  ck(cudaEventElapsedTime(&e->lastMs, e->ev0, e->ev1), "cudaEventElapsedTime");
  ck(cudaEventElapsedTime(&e->lastRunMs, e->evRun0, e->evRun1), "cudaEventElapsedTime");
  if (bits & 3u) return fail(CQG_E_NONFINITE, "a trajectory produced a non-finite norm or rate");
  if (bits & 12u) return fail(CQG_E_STALLED, "a trajectory exhausted its step-size or attempt budget");
  for (size_t gi = 0; 4 * gi < yieldHeads.size(); ++gi)
    if (yieldHeads[4 * gi + 2])
      return fail(CQG_E_STALLED, "a yielded trajectory was not resumed within the time limit");
  return CQG_OK;
}

// Autotuner of the CTA shape of a kernel group (its size and, for CTA-per-trajectory groups,
// whether the stage derivatives live in shared memory or in a global scratch slab): the
// candidates are timed on a sample of the group's trajectories (a scratch ensemble from the
// same initial states, so the ensemble itself is not advanced) over a fixed number of MCWF
// steps each, and the fastest is kept.  Results are cached per (device, precision, kernel kind, rows per lane, slot
// bound, largest dimension) for the life of the process.
// Candidate shapes, encoded as CTA threads | (shared-memory stage vectors << 16) | (the warp
// kernel's high-occupancy instance << 17).
std::vector<int> threadCandidates(const KernelGroup& g, bool vectorsFit) {
  std::vector<int> c;
  if (g.kind == 0) {  // warp kernel: CTA size, and the high-occupancy instance where there is one
    c = {64, 128};
    if (dev::warpHighOccupancyVariant(g.E, g.smax <= 2 ? 2 : g.smax <= 3 ? 3 : g.smax <= 4 ? 4 : 8, g.anyFreq))
      c.insert(c.end(), {64 | kHighOccupancyFlag, 128 | kHighOccupancyFlag});
    return c;
  }
  for (int q = 1; q <= 4; ++q) {  // rows per thread
    const int t = std::min(512, std::max(64, ((g.Dmax + q - 1) / q + 31) / 32 * 32));
    if (std::find(c.begin(), c.end(), t) == c.end()) c.push_back(t);
  }
  if (std::find(c.begin(), c.end(), 256) == c.end()) c.push_back(256);
  if (vectorsFit) {
    const size_t n = c.size();
    for (size_t k = 0; k < n; ++k) c.push_back(c[k] | (1 << 16));
  }
  return c;
}

bool sharedVectorsFit(const KernelGroup& g, size_t elemBytes, int device) {
  int optin = 0;
  ck(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device), "attribute");
  return g.kind == 1 && blockSmemBytes(g.Dmax, elemBytes, true, g.phaseElems) <= size_t(optin);
}

int tunedThreads(const cqg_ensemble& e, size_t gi, const cqg_system* const* systems, int nSys,
                 const cqg_complex* psi0s, const int64_t* psi0Off, const cqg_mcwf_pars& pars) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int, int, int, bool>, int> cache;
  const KernelGroup& g = e.groups[gi];
  const auto key = std::make_tuple(e.device, pars.precision, g.kind, g.E, g.smax, g.Dmax, g.anyFreq);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  const std::vector<int> cands = threadCandidates(g, sharedVectorsFit(g, e.elemBytes, e.device));
  int nSM = 0;
  ck(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, e.device), "attribute");
  // the group itself up to a few fills of the device: the number of waves the resident CTAs
  // take decides as much as their speed, so the sample has the group's own count where it can
  const int64_t want = g.kind ? int64_t(nSM) * 16 : int64_t(nSM) * 64;
  if (g.count < (g.kind ? int64_t(nSM) * 2 : int64_t(nSM) * 8)) return defaultThreads(g);  // too small to time
  const int64_t n = std::min<int64_t>(g.count, want);
  std::vector<int> order(e.nTraj);
  ck(cudaMemcpy(order.data(), e.dOrder, order.size() * sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(order)");
  std::vector<int32_t> sIdx(n);
  std::vector<int64_t> sOff(n);
  for (int64_t k = 0; k < n; ++k) {
    const int ti = order[g.first + k];
    sIdx[k] = e.sysIdx[ti];
    sOff[k] = psi0Off ? psi0Off[ti] : 0;
  }
  cqg_mcwf_pars tp = pars;
  tp.autotune = 0;
  tp.cta_threads = cands[0] & 0xffff;
  tp.cta_shared_vectors = 0;
  cqg_ensemble* tmp = nullptr;
  if (createEnsemble(systems, nSys, sIdx.data(), psi0s, psi0Off ? sOff.data() : nullptr, n, &tp, &tmp) != CQG_OK)
    return defaultThreads(g);
  std::unique_ptr<cqg_ensemble> hold(tmp);
  if (tmp->groups.size() != 1) return defaultThreads(g);
  dev::RunArgs ra{};
  ra.mode = dev::RUN_STEPS;
  ra.nIntervals = 1;
  ra.T = 1e300;
  int best = defaultThreads(g);
  float bestMs = 0;
  auto setShape = [&](int c) {
    tmp->groups[0].threads = c & 0xffff;
    tmp->groups[0].smemVectors = (c & (1 << 16)) != 0;
    tmp->groups[0].highOccupancy = (c & kHighOccupancyFlag) != 0;
  };
  // Warm-up: every candidate advances the sample by 8 MCWF steps (which also moves it away
  // from its initial state).  The candidates are then timed as the ensemble runs: every
  // trajectory advanced over the same interval of simulated time (a varying number of steps
  // each, the interval sized for about 48 steps), twice, keeping each candidate's faster time.
  for (int c : cands) {
    setShape(c);
    ra.nSteps = 8;
    if (launchRun(tmp, ra, 0, nullptr) != CQG_OK) return defaultThreads(g);
  }
  std::vector<double> tt(size_t(tmp->nTraj));
  ck(cudaMemcpy(tt.data(), tmp->td.t, tt.size() * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy(times)");
  double tNow = *std::max_element(tt.begin(), tt.end());
  const double interval = tNow / (8. * double(cands.size())) * 48.;
  std::vector<float> ms(cands.size(), 0.f);
  for (int pass = 1; pass <= 2; ++pass)
    for (size_t ci = 0; ci < cands.size(); ++ci) {
      setShape(cands[ci]);
      if (interval > 0 && std::isfinite(interval)) {
        ra.mode = dev::RUN_TO;
        ra.tEnd = tNow + interval;
        tNow = ra.tEnd;
      } else {
        ra.nSteps = 48;
      }
      if (launchRun(tmp, ra, 0, nullptr) != CQG_OK) return defaultThreads(g);
      ms[ci] = pass == 1 ? tmp->lastMs : std::min(ms[ci], tmp->lastMs);
    }
  for (size_t ci = 0; ci < cands.size(); ++ci)
    if (bestMs == 0 || ms[ci] < bestMs) {
      bestMs = ms[ci];
      best = cands[ci];
    }
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = best;
  return best;
}

}  // namespace

namespace {

// FMA-chain probe: each thread runs `iters` dependent-free FMA groups on 8 accumulators
template <typename R>
__global__ void fmaProbeKernel(R* out, int iters, R a, R b) {
  R x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = R(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  }
  R s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == R(-1.2345)) out[threadIdx.x] = s;  // keeps the loop alive
}

template <typename R>
double probe(int device) {
  int nSM = 0;
  ck(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, device), "attribute");
  R* out = nullptr;
  ck(cudaMalloc(&out, 1024 * sizeof(R)), "cudaMalloc");
  cudaEvent_t a, b;
  ck(cudaEventCreate(&a), "event");
  ck(cudaEventCreate(&b), "event");
  const int blocks = nSM * 8, threads = 256, iters = 4096;
  fmaProbeKernel<R><<<blocks, threads>>>(out, iters, R(0.999999), R(1e-7));
  ck(cudaEventRecord(a), "event");
  const int reps = 5;
  for (int r = 0; r < reps; ++r) fmaProbeKernel<R><<<blocks, threads>>>(out, iters, R(0.999999), R(1e-7));
  ck(cudaEventRecord(b), "event");
  ck(cudaEventSynchronize(b), "sync");
  float ms = 0;
  ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  const double flops = 2.0 * 8 * double(iters) * blocks * threads * reps;
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

namespace cqg {
namespace dev {
// accessors for the allocation-free averages entry point (noalloc.cu)
const SysDev* systemDescriptor(const cqg_system* sys) { return &sys->sd; }
int systemDevice(const cqg_system* sys) { return sys->device; }
}  // namespace dev
}  // namespace cqg

extern "C" {

int cqg_device_count(int* count) {
  if (!count) return fail(CQG_E_INVALID, "null argument");
  int n = 0;
  const cudaError_t err = cudaGetDeviceCount(&n);
  if (err != cudaSuccess) {
    *count = 0;
    cudaGetLastError();
    return fail(CQG_E_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(err));
  }
  *count = n;
  return CQG_OK;
}

int cqg_system_create(const cqg_system_desc* desc, cqg_system** out) {
  return guardedCuda([&] {
    if (!desc || !out) return fail(CQG_E_INVALID, "cqg_system_create: null argument");
    int n = 0;
    if (cqg_device_count(&n) != CQG_OK || n < 1) return fail(CQG_E_NODEVICE, "cqg_system_create: no CUDA device");
    auto s = std::make_unique<cqg_system>();
    s->L = cqg::lowerSystem(*desc);
    if (!(s->L.highestFrequency > 0) && s->L.hasH)
      return fail(CQG_E_INVALID, "cqg_system_create: highest_frequency must be positive");
    ck(cudaGetDevice(&s->device), "cudaGetDevice");
    buildSystemDevice(*s);
    *out = s.release();
    return CQG_OK;
  });
}

int cqg_system_dimension(const cqg_system* sys, int64_t* d) {
  if (!sys || !d) return fail(CQG_E_INVALID, "null argument");
  *d = sys->L.D;
  return CQG_OK;
}

int cqg_system_destroy(cqg_system* sys) {
  delete sys;
  return CQG_OK;
}

int cqg_ensemble_create(const cqg_system* sys, const cqg_complex* psi0, int64_t n_traj, const cqg_mcwf_pars* pars,
                        cqg_ensemble** out) {
  return guardedCuda([&] { return createEnsemble(&sys, 1, nullptr, psi0, nullptr, n_traj, pars, out); });
}

int cqg_batch_create(const cqg_system* const* systems, int32_t n_systems, const int32_t* sys_index,
                     const cqg_complex* psi0s, const int64_t* psi0_offsets, int64_t n_traj, const cqg_mcwf_pars* pars,
                     cqg_ensemble** out) {
  return guardedCuda([&] {
    if (!sys_index || !psi0_offsets) return fail(CQG_E_INVALID, "cqg_batch_create: null index arrays");
    return createEnsemble(systems, n_systems, sys_index, psi0s, psi0_offsets, n_traj, pars, out);
  });
}

int cqg_ensemble_run(cqg_ensemble* ens, double Dt, int32_t n_intervals, double* avr_out) {
  return guardedCuda([&] {
    if (!ens || !(Dt > 0) || n_intervals < 1) return fail(CQG_E_INVALID, "cqg_ensemble_run: Dt > 0 and n_intervals >= 1 required");
    dev::RunArgs ra{};
    ra.mode = dev::RUN_INTERVALS;
    ra.Dt = Dt;
    ra.nIntervals = n_intervals;
    return launchRun(ens, ra, n_intervals, avr_out);
  });
}

int cqg_ensemble_advance_to(cqg_ensemble* ens, double t_end, double* avr_out) {
  return guardedCuda([&] {
    if (!ens) return fail(CQG_E_INVALID, "null ensemble");
    dev::RunArgs ra{};
    ra.mode = dev::RUN_TO;
    ra.tEnd = t_end;
    ra.nIntervals = 1;
    return launchRun(ens, ra, 1, avr_out);
  });
}

int cqg_ensemble_steps(cqg_ensemble* ens, int32_t n_steps, double T, double* avr_out) {
  return guardedCuda([&] {
    if (!ens || n_steps < 0) return fail(CQG_E_INVALID, "cqg_ensemble_steps: n_steps >= 0 required");
    dev::RunArgs ra{};
    ra.mode = dev::RUN_STEPS;
    ra.nSteps = n_steps;
    ra.T = T;
    ra.nIntervals = 1;
    return launchRun(ens, ra, 1, avr_out);
  });
}

int cqg_ensemble_traj_averages(cqg_ensemble* ens, double* out) {
  return guardedCuda([&] {
    if (!ens || !out) return fail(CQG_E_INVALID, "null argument");
    // the per-trajectory slots of the last output of the last run
    if (!ens->dAvr) return fail(CQG_E_INVALID, "cqg_ensemble_traj_averages: no run yet");
    ck(cudaMemcpy(out, ens->dAvr, size_t(ens->nTraj) * (ens->nAvrMax + 1) * sizeof(double), cudaMemcpyDeviceToHost),
       "cudaMemcpy");
    return CQG_OK;
  });
}

namespace {

constexpr char kCheckpointMagic[8] = {'C', 'Q', 'G', 'C', 'K', 'P', 'T', '1'};

struct CheckpointHeader {
  char magic[8];
  uint32_t elemBytes, jumpCap;
  int64_t nTraj, psiElems;
  uint64_t layoutHash;  // dimensions and system index of every trajectory
};

// the device arrays of a checkpoint, in order: (pointer, bytes)
std::vector<std::pair<void*, size_t>> checkpointParts(const cqg_ensemble& e, int64_t psiElems) {
  const size_t n = size_t(e.nTraj);
  const auto& td = e.td;
  return {{td.psi, size_t(psiElems) * e.elemBytes},
          {td.t, n * 8},
          {td.t0, n * 8},
          {td.dtTry, n * 8},
          {td.dtDid, n * 8},
          {td.rng, n * 32},
          {td.cnt, n * 64},
          {td.maxima, n * 24},
          {td.status, n * 4},
          {td.jumpT, n * size_t(td.jumpCap) * 8},
          {td.jumpL, n * size_t(td.jumpCap) * 4},
          {td.jumpN, n * 8}};
}

CheckpointHeader checkpointHeader(const cqg_ensemble& e) {
  CheckpointHeader h{};
  std::memcpy(h.magic, kCheckpointMagic, 8);
  h.elemBytes = uint32_t(e.elemBytes);
  h.jumpCap = uint32_t(e.td.jumpCap);
  h.nTraj = e.nTraj;
  uint64_t hash = 1469598103934665603ull, elems = 0;  // FNV-1a over (D, system index)
  for (int64_t i = 0; i < e.nTraj; ++i) {
    const uint64_t D = uint64_t(e.systems[e.sysIdx[i]]->L.D), words[2] = {D, uint64_t(e.sysIdx[i])};
    for (uint64_t w : words)
      for (int b = 0; b < 8; ++b) hash = (hash ^ ((w >> (8 * b)) & 0xff)) * 1099511628211ull;
    elems += D;
  }
  h.psiElems = int64_t(elems);
  h.layoutHash = hash;
  return h;
}

}  // namespace

int cqg_ensemble_save(const cqg_ensemble* ens, void* buf, uint64_t cap, uint64_t* size) {
  return guardedCuda([&] {
    if (!ens || !size) return fail(CQG_E_INVALID, "cqg_ensemble_save: null argument");
    const CheckpointHeader h = checkpointHeader(*ens);
    const auto parts = checkpointParts(*ens, h.psiElems);
    uint64_t total = sizeof(h);
    for (auto& p : parts) total += p.second;
    *size = total;
    if (!buf || cap < total) return CQG_OK;
    ck(cudaStreamSynchronize(ens->stream), "cudaStreamSynchronize");
    char* out = static_cast<char*>(buf);
    std::memcpy(out, &h, sizeof(h));
    out += sizeof(h);
    for (auto& p : parts) {
      ck(cudaMemcpy(out, p.first, p.second, cudaMemcpyDeviceToHost), "cudaMemcpy(checkpoint)");
      out += p.second;
    }
    return CQG_OK;
  });
}

int cqg_ensemble_load(cqg_ensemble* ens, const void* buf, uint64_t size) {
  return guardedCuda([&] {
    if (!ens || !buf) return fail(CQG_E_INVALID, "cqg_ensemble_load: null argument");
    if (size < sizeof(CheckpointHeader)) return fail(CQG_E_INVALID, "cqg_ensemble_load: truncated checkpoint");
    CheckpointHeader h;
    std::memcpy(&h, buf, sizeof(h));
    const CheckpointHeader mine = checkpointHeader(*ens);
    if (std::memcmp(h.magic, kCheckpointMagic, 8) != 0) return fail(CQG_E_INVALID, "cqg_ensemble_load: not a checkpoint");
    if (h.elemBytes != mine.elemBytes || h.jumpCap != mine.jumpCap || h.nTraj != mine.nTraj ||
        h.psiElems != mine.psiElems || h.layoutHash != mine.layoutHash)
      return fail(CQG_E_INVALID, "cqg_ensemble_load: checkpoint of a different ensemble (systems, size or precision)");
    const auto parts = checkpointParts(*ens, h.psiElems);
    uint64_t total = sizeof(h);
    for (auto& p : parts) total += p.second;
    if (size != total) return fail(CQG_E_INVALID, "cqg_ensemble_load: checkpoint size mismatch");
    ck(cudaStreamSynchronize(ens->stream), "cudaStreamSynchronize");
    const char* in = static_cast<const char*>(buf) + sizeof(h);
    for (auto& p : parts) {
      ck(cudaMemcpy(p.first, in, p.second, cudaMemcpyHostToDevice), "cudaMemcpy(checkpoint)");
      in += p.second;
    }
    return CQG_OK;
  });
}

int cqg_ensemble_plan(const cqg_ensemble* ens, int32_t* n_groups, int32_t* plan, int32_t cap) {
  if (!ens || !n_groups || (cap > 0 && !plan)) return fail(CQG_E_INVALID, "cqg_ensemble_plan: null argument");
  *n_groups = int32_t(ens->groups.size());
  for (int32_t g = 0; g < std::min<int32_t>(cap, *n_groups); ++g) {
    const KernelGroup& k = ens->groups[g];
    int32_t* o = plan + 5 * g;
    o[0] = k.kind == 1 && k.smemVectors ? 2 : k.kind == 0 && k.highOccupancy ? 3 : k.kind;
    o[1] = k.E;
    o[2] = k.smax;
    o[3] = k.threads;
    o[4] = int32_t(k.count);
  }
  return CQG_OK;
}

int cqg_ensemble_size(const cqg_ensemble* ens, int64_t* n_traj, int32_t* n_avr) {
  if (!ens) return fail(CQG_E_INVALID, "null ensemble");
  if (n_traj) *n_traj = ens->nTraj;
  if (n_avr) *n_avr = ens->nAvrMax;
  return CQG_OK;
}

int cqg_ensemble_get_state(const cqg_ensemble* ens, int64_t i, cqg_complex* psi) {
  return guardedCuda([&] {
    if (!ens || !psi || i < 0 || i >= ens->nTraj) return fail(CQG_E_INVALID, "cqg_ensemble_get_state: bad index");
    const int64_t D = ens->systems[ens->sysIdx[i]]->L.D;
    std::vector<unsigned char> b(D * ens->elemBytes);
    ck(cudaMemcpy(b.data(), static_cast<char*>(ens->td.psi) + ens->psiOff[i] * ens->elemBytes, b.size(),
                  cudaMemcpyDeviceToHost),
       "cudaMemcpy");
    for (int64_t k = 0; k < D; ++k) {
      if (ens->elemBytes == 16) {
        double2 v;
        std::memcpy(&v, &b[k * 16], 16);
        psi[k] = {v.x, v.y};
      } else {
        float2 v;
        std::memcpy(&v, &b[k * 8], 8);
        psi[k] = {double(v.x), double(v.y)};
      }
    }
    return CQG_OK;
  });
}

int cqg_ensemble_set_state(cqg_ensemble* ens, int64_t i, const cqg_complex* psi) {
  return guardedCuda([&] {
    if (!ens || !psi || i < 0 || i >= ens->nTraj) return fail(CQG_E_INVALID, "cqg_ensemble_set_state: bad index");
    const int64_t D = ens->systems[ens->sysIdx[i]]->L.D;
    std::vector<unsigned char> b(D * ens->elemBytes);
    for (int64_t k = 0; k < D; ++k) {
      if (ens->elemBytes == 16) {
        double2 v = make_double2(psi[k].re, psi[k].im);
        std::memcpy(&b[k * 16], &v, 16);
      } else {
        float2 v = make_float2(float(psi[k].re), float(psi[k].im));
        std::memcpy(&b[k * 8], &v, 8);
      }
    }
    ck(cudaMemcpy(static_cast<char*>(ens->td.psi) + ens->psiOff[i] * ens->elemBytes, b.data(), b.size(),
                  cudaMemcpyHostToDevice),
       "cudaMemcpy");
    return CQG_OK;
  });
}

int cqg_ensemble_get_times(const cqg_ensemble* ens, double* t, double* dt_did, double* dt_try) {
  return guardedCuda([&] {
    if (!ens) return fail(CQG_E_INVALID, "null ensemble");
    const size_t n = size_t(ens->nTraj) * sizeof(double);
    if (t) ck(cudaMemcpy(t, ens->td.t, n, cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (dt_did) ck(cudaMemcpy(dt_did, ens->td.dtDid, n, cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (dt_try) ck(cudaMemcpy(dt_try, ens->td.dtTry, n, cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CQG_OK;
  });
}

int cqg_ensemble_get_counters(const cqg_ensemble* ens, uint64_t* counters) {
  return guardedCuda([&] {
    if (!ens || !counters) return fail(CQG_E_INVALID, "null argument");
    ck(cudaMemcpy(counters, ens->td.cnt, size_t(ens->nTraj) * 64, cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CQG_OK;
  });
}

int cqg_ensemble_get_logger_maxima(const cqg_ensemble* ens, double* max_overshoot, double* max_tolerance_overshoot,
                                   double* max_norm_dev) {
  return guardedCuda([&] {
    if (!ens) return fail(CQG_E_INVALID, "null ensemble");
    std::vector<double> m(3 * ens->nTraj);
    ck(cudaMemcpy(m.data(), ens->td.maxima, m.size() * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (int64_t i = 0; i < ens->nTraj; ++i) {
      if (max_overshoot) max_overshoot[i] = m[3 * i];
      if (max_tolerance_overshoot) max_tolerance_overshoot[i] = m[3 * i + 1];
      if (max_norm_dev) max_norm_dev[i] = m[3 * i + 2];
    }
    return CQG_OK;
  });
}

int cqg_ensemble_get_jumps(const cqg_ensemble* ens, int64_t i, int32_t cap, double* times, int32_t* lindblads,
                           int32_t* n_out) {
  return guardedCuda([&] {
    if (!ens || i < 0 || i >= ens->nTraj || cap < 0) return fail(CQG_E_INVALID, "cqg_ensemble_get_jumps: bad argument");
    unsigned long long n = 0;
    ck(cudaMemcpy(&n, ens->td.jumpN + i, 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    const int J = ens->jumpCap;
    std::vector<double> tt(J);
    std::vector<int> ll(J);
    ck(cudaMemcpy(tt.data(), ens->td.jumpT + size_t(i) * J, J * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    ck(cudaMemcpy(ll.data(), ens->td.jumpL + size_t(i) * J, J * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    const unsigned long long kept = std::min<unsigned long long>(n, J);
    const unsigned long long first = n - kept;
    int32_t w = 0;
    for (unsigned long long k = first; k < n && w < cap; ++k, ++w) {
      if (times) times[w] = tt[k % J];
      if (lindblads) lindblads[w] = ll[k % J];
    }
    if (n_out) *n_out = w;
    return CQG_OK;
  });
}

int cqg_ensemble_get_jump_rings(const cqg_ensemble* ens, int32_t* cap, uint64_t* counts, double* times,
                                int32_t* lindblads) {
  return guardedCuda([&] {
    if (!ens) return fail(CQG_E_INVALID, "null ensemble");
    ck(cudaSetDevice(ens->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(ens->stream), "cudaStreamSynchronize");
    const size_t n = size_t(ens->nTraj), J = size_t(ens->jumpCap);
    if (cap) *cap = ens->jumpCap;
    if (counts) ck(cudaMemcpy(counts, ens->td.jumpN, n * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (times) ck(cudaMemcpy(times, ens->td.jumpT, n * J * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (lindblads) ck(cudaMemcpy(lindblads, ens->td.jumpL, n * J * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    return CQG_OK;
  });
}

int cqg_ensemble_set_jump_capacity(cqg_ensemble* ens, int32_t cap) {
  return guardedCuda([&] {
    if (!ens || cap < 1) return fail(CQG_E_INVALID, "cqg_ensemble_set_jump_capacity: capacity >= 1 required");
    if (cap == ens->jumpCap) return CQG_OK;
    ck(cudaSetDevice(ens->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(ens->stream), "cudaStreamSynchronize");
    const size_t n = size_t(ens->nTraj), J0 = size_t(ens->jumpCap), J1 = size_t(cap);
    if (n * J1 > (size_t(1) << 31)) return fail(CQG_E_NOMEM, "cqg_ensemble_set_jump_capacity: capacity too large");
    std::vector<unsigned long long> cnt(n);
    std::vector<double> t0(n * J0), t1(n * J1, 0.);
    std::vector<int> l0(n * J0), l1(n * J1, 0);
    ck(cudaMemcpy(cnt.data(), ens->td.jumpN, n * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    ck(cudaMemcpy(t0.data(), ens->td.jumpT, n * J0 * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    ck(cudaMemcpy(l0.data(), ens->td.jumpL, n * J0 * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    // the most recent records that both rings hold, each at its slot (k mod capacity)
    for (size_t i = 0; i < n; ++i) {
      const unsigned long long keep = std::min<unsigned long long>(cnt[i], std::min(J0, J1));
      for (unsigned long long k = cnt[i] - keep; k < cnt[i]; ++k) {
        t1[i * J1 + k % J1] = t0[i * J0 + k % J0];
        l1[i * J1 + k % J1] = l0[i * J0 + k % J0];
      }
    }
    const size_t bytes = n * J1 * 12;
    void* ring = cqg::engine::deviceAlloc(bytes, "cudaMalloc(jump rings)");
    char* r = static_cast<char*>(ring);
    ck(cudaMemcpy(r, t1.data(), n * J1 * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
    ck(cudaMemcpy(r + n * J1 * 8, l1.data(), n * J1 * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
    cqg::engine::deviceRelease(ens->device, ens->dJumpRing, ens->jumpRingBytes);
    ens->dJumpRing = ring;
    ens->jumpRingBytes = bytes;
    ens->jumpCap = cap;
    ens->td.jumpT = reinterpret_cast<double*>(r);
    ens->td.jumpL = reinterpret_cast<int*>(r + n * J1 * 8);
    ens->td.jumpCap = cap;
    return CQG_OK;
  });
}

int cqg_ensemble_status(const cqg_ensemble* ens, uint32_t* bits) {
  return guardedCuda([&] {
    if (!ens || !bits) return fail(CQG_E_INVALID, "null argument");
    std::vector<unsigned> st(ens->nTraj);
    ck(cudaMemcpy(st.data(), ens->td.status, st.size() * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    unsigned b = 0;
    for (auto v : st) b |= v;
    *bits = b;
    if (b & 3u) return fail(CQG_E_NONFINITE, "a trajectory produced a non-finite norm or rate");
    if (b & 12u) return fail(CQG_E_STALLED, "a trajectory exhausted its step-size or attempt budget");
    return CQG_OK;
  });
}

int cqg_ensemble_last_kernel_ms(const cqg_ensemble* ens, double* kernel_ms, double* run_ms) {
  if (!ens) return fail(CQG_E_INVALID, "null argument");
  if (kernel_ms) *kernel_ms = ens->lastMs;
  if (run_ms) *run_ms = ens->lastRunMs;
  return CQG_OK;
}

int cqg_probe_fma_peaks(double* fp64_tflops, double* fp32_tflops) {
  return guardedCuda([&] {
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    if (fp64_tflops) *fp64_tflops = probe<double>(dev);
    if (fp32_tflops) *fp32_tflops = probe<float>(dev);
    return CQG_OK;
  });
}

int cqg_ensemble_destroy(cqg_ensemble* ens) {
  delete ens;
  return CQG_OK;
}

}  // extern "C"
