// MCWF trajectory kernel for large Hilbert spaces (D > 128), one CTA per trajectory.
//
// The warp kernel keeps a trajectory's state and stage derivatives in registers, which
// limits it to D <= 128.  Here a CTA owns one trajectory at a time (persistent CTAs pull
// trajectories from the same work queue) and each thread walks rows r = tid + blockDim*j.
// The state lives in two buffers, the trajectory's slot in device memory and one vector of a
// per-CTA scratch slab: an ODE attempt writes its candidate solution into the buffer the
// state is not in, an accepted attempt makes that buffer the state, and the other one still
// holds the state of the step's start, which is all a step-back needs.  The stage
// derivatives k0..k4 live in the scratch slab too (L2-resident for the CTAs in flight); k5
// is consumed row by row by the solution and the error norm as the last right-hand side
// produces it.  Only the stage vector that the banded H/i gather reads is staged in shared
// memory (double-buffered, one __syncthreads per right-hand side).  Every row is touched by
// the same thread in every pass, so the scratch vectors need no synchronisation.  The
// algorithm, step by step, is the one of the warp kernel (mcwf_kernel.cuh) and of the
// reference's MCWF_Trajectory::step.
#pragma once

#include "mcwf_kernel.cuh"

namespace cqg {
namespace dev {

constexpr int kBlockVectors = 6;  // k0..k4, the second state buffer

// Cash-Karp stage tableau for the (not unrolled) stage loop
__constant__ double kBlockA[5][5] = {{1. / 5, 0, 0, 0, 0},
                                     {3. / 40, 9. / 40, 0, 0, 0},
                                     {3. / 10, -9. / 10, 6. / 5, 0, 0},
                                     {-11. / 54, 5. / 2, -70. / 27, 35. / 27, 0},
                                     {1631. / 55296, 175. / 512, 575. / 13824, 44275. / 110592, 253. / 4096}};
__constant__ double kBlockC[5] = {1. / 5, 3. / 10, 3. / 5, 1., 7. / 8};

struct BlockScratch {
  void* base;           // [gridDim.x][kBlockVectors][stride] Real2, or null: the vectors
                        // follow the broadcast words in dynamic shared memory
  long long stride;     // elements per vector (>= max D)
  int phaseElems;       // IP: capacity of the shared-memory phase table (0: none)
};

// block-wide sums of n <= N uniform values; red holds 32 * N doubles of shared memory
template <int N>
__device__ __forceinline__ void blockSumN(double (&v)[N], int n, double* red) {
  warpSumN(v, n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  // loops over the compile-time bound, so that v stays in registers
  if (lane == 0)
#pragma unroll
    for (int m = 0; m < N; ++m)
      if (m < n) red[warp * N + m] = v[m];
  __syncthreads();
#pragma unroll
  for (int m = 0; m < N; ++m)
    if (m < n) {
      double s = 0.;
      for (int w = 0; w < nw; ++w) s += red[w * N + m];
      v[m] = s;
    }
}

__device__ __forceinline__ double blockMax(double v, double* red) {
  v = warpMax(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double m = 0.;
  for (int w = 0; w < nw; ++w) m = fmax(m, red[w]);
  return m;
}

// IP: the instance serves interaction-picture systems; the IP = false instance has no
// phase code.
template <typename R, bool IP>
struct BlockWorker {
  using C2 = typename CT<R>::T;
  static constexpr int NR = MAX_JUMPS + 1;

  const SysDev* sysp;
  const RunArgs& ra;
  int D, S, nJ;
  bool hasH, hasEx, hasFreq, anySpecial;
  const int* col;
  const C2* val;
  const C2* diag;
  const double2* freq;
  const unsigned short* fIdx;  // IP: distinct-frequency index per slot and row, or null
  const double2* fDist;
  int nFD;
  double2* phTab;  // IP: shared-memory phases of the distinct frequencies, or null
  const int* word;    // packed slot words (SysDev::ctaWord) or null
  const int4* recF;   // FP32 packed records (SysDev::ctaRecF) or null
  bool diagZero;      // the fused main diagonal is zero: not read
  C2* x;       // the state: the trajectory's slot or the second buffer
  C2* xalt;    // the other one (an attempt's candidate; after a step, the step's start)
  C2* xslot;   // the trajectory's slot in device memory
  C2* vec;     // this CTA's scratch vectors
  long long stride;
  C2* ys0;     // shared stage buffers
  C2* ys1;
  double* red; // shared reduction scratch [32][NR]
  unsigned long long* bcast;  // shared broadcast words

  double t, t0, dtTry, dtDid;
  unsigned long long ti;
  unsigned nSteps, nAttempts, nFailed, nRhs, nOvershot, nBacks, nJumps;
  double maxOvershoot, maxTolOvershoot, maxNormDev;
  unsigned status;

  __device__ __forceinline__ C2* K(int j) const { return vec + j * stride; }
  __device__ __forceinline__ C2* second() const { return vec + 5 * stride; }

  // sink(r, ((H/i) y)[r]) for every row r of this thread, y in shared memory, at picture
  // time tau
  template <class Sink>
  __device__ __forceinline__ void rhs(const C2* ys, double tau, Sink&& sink) {
    ++nRhs;
    bool tab = false;
    if constexpr (IP) {
      // exp(tau f) once per distinct frequency into shared memory: the same values, bit for
      // bit, as one exponential per row and slot
      tab = phTab && hasFreq && tau != 0.;
      if (tab) {
        __syncthreads();
        for (int k = threadIdx.x; k < nFD; k += blockDim.x) phTab[k] = cexpScaledInline(tau, __ldg(&fDist[k]));
        __syncthreads();
      }
    }
    // The operator tables are shared by all trajectories and live in L2 (L1 is mostly given
    // to shared memory here).  The slot loops are unrolled by four and free of calls, so that
    // the loads of several slots are in flight together; the products are accumulated in
    // slot order in every variant.
    // With the packed records (SysDev::ctaWord) a slot's column and phase index come in one
    // word, and in FP32 with the coefficient in one 16-byte load.
    for (int r = threadIdx.x; r < D; r += blockDim.x) {
      C2 acc = diagZero ? mk<C2>(0, 0) : cmul(diag[r], ys[r]);
      if (IP && tab && word) {
#pragma unroll 4
        for (int s = 0; s < S; ++s) {
          C2 c;
          unsigned w;
          slotRecord(s, r, c, w);
          const unsigned k = w >> 16;
          if (k != kNoPhase) {
            const double2 ph = phTab[k];
            c = mk<C2>(double(c.x) * ph.x - double(c.y) * ph.y, double(c.x) * ph.y + double(c.y) * ph.x);
          }
          acc = cfma(c, ys[r + int(short(w & 0xffffu))], acc);
        }
      } else if (IP && tab) {
#pragma unroll 4
        for (int s = 0; s < S; ++s) {
          C2 c = __ldg(&val[s * D + r]);
          const unsigned k = __ldg(&fIdx[s * D + r]);
          if (k != kNoPhase) {
            const double2 ph = phTab[k];
            c = mk<C2>(double(c.x) * ph.x - double(c.y) * ph.y, double(c.x) * ph.y + double(c.y) * ph.x);
          }
          acc = cfma(c, ys[__ldg(&col[s * D + r])], acc);
        }
      } else if (IP && hasFreq && tau != 0.) {
        for (int s = 0; s < S; ++s) {
          C2 c = __ldg(&val[s * D + r]);
          const double2 f = __ldg(&freq[s * D + r]);
          if (f.x != 0. || f.y != 0.) {  // exp(0 f) = 1 exactly
            const double2 ph = cexpScaled(tau, f);
            c = mk<C2>(double(c.x) * ph.x - double(c.y) * ph.y, double(c.x) * ph.y + double(c.y) * ph.x);
          }
          acc = cfma(c, ys[__ldg(&col[s * D + r])], acc);
        }
      } else if (word) {
#pragma unroll 4
        for (int s = 0; s < S; ++s) {
          C2 c;
          unsigned w;
          slotRecord(s, r, c, w);
          acc = cfma(c, ys[r + int(short(w & 0xffffu))], acc);
        }
      } else {
#pragma unroll 4
        for (int s = 0; s < S; ++s) acc = cfma(__ldg(&val[s * D + r]), ys[__ldg(&col[s * D + r])], acc);
      }
      sink(r, acc);
    }
  }

  // coefficient and packed word of slot s of row r (SysDev::ctaWord / ctaRecF)
  __device__ __forceinline__ void slotRecord(int s, int r, C2& c, unsigned& w) const {
    if constexpr (sizeof(C2) == sizeof(float2)) {
      const int4 q = __ldg(&recF[s * D + r]);
      c = mk<C2>(__int_as_float(q.x), __int_as_float(q.y));
      w = unsigned(q.z);
    } else {
      c = __ldg(&val[s * D + r]);
      w = unsigned(__ldg(&word[s * D + r]));
    }
  }

  __device__ __forceinline__ bool odeStep(double deltaT) {
    const double timeBefore = t;
    const double nextDtTry = fabs(deltaT) < fabs(dtTry / 10.) ? dtTry : 0.;
    if (fabs(dtTry) > fabs(deltaT)) dtTry = deltaT;
    __syncthreads();
    for (int r = threadIdx.x; r < D; r += blockDim.x) ys0[r] = x[r];
    __syncthreads();
    {
      C2* const k0 = K(0);
      rhs(ys0, t - t0, [&](int r, C2 v) { k0[r] = v; });
    }
    for (int attempt = 0;; ++attempt) {
      if (attempt >= ra.maxAttempts) {
        status |= 8u;
        return false;
      }
      ++nAttempts;
      const double dt = dtTry;
      for (int st = 1; st <= 5; ++st) {
        C2* ys = (st & 1) ? ys1 : ys0;
        R a[5];  // this stage's tableau row times dt (unrolled below: all loads of a row at once)
#pragma unroll
        for (int j = 0; j < 5; ++j) a[j] = j < st ? R(dt * kBlockA[st - 1][j]) : R(0);
        for (int r = threadIdx.x; r < D; r += blockDim.x) {
          C2 y = x[r];
#pragma unroll
          for (int j = 0; j < 5; ++j)
            if (j < st) y = axpy(a[j], K(j)[r], y);
          ys[r] = y;
        }
        __syncthreads();
        if (st == 5) break;  // the last right-hand side feeds the solution below
        C2* const ks = K(st);
        rhs(ys, t + kBlockC[st - 1] * dt - t0, [&](int r, C2 v) { ks[r] = v; });
      }
      const R b0 = R(dt * CK::b0), b2 = R(dt * CK::b2), b3 = R(dt * CK::b3), b5 = R(dt * CK::b5);
      const R e0 = R(dt * CK::e0), e2 = R(dt * CK::e2), e3 = R(dt * CK::e3), e4 = R(dt * CK::e4),
              e5 = R(dt * CK::e5);
      const double adt = fabs(dt);
      ErrNormMax errLocal;
      // k5 row by row: the 5th-order solution into the other state buffer and the rows' part
      // of the error norm
      {
        const C2* const xs = x;
        C2* const cand = xalt;
        rhs(ys1, t + kBlockC[4] * dt - t0, [&](int r, C2 k5) {
          const C2 xr = xs[r], k0 = K(0)[r], k2 = K(2)[r], k3 = K(3)[r], k4 = K(4)[r];
          cand[r] = axpy(b5, k5, axpy(b3, k3, axpy(b2, k2, axpy(b0, k0, xr))));
          C2 xe = mk<C2>(0, 0);
          xe = axpy(e5, k5, axpy(e4, k4, axpy(e3, k3, axpy(e2, k2, axpy(e0, k0, xe)))));
          errLocal.add(abs2(xe), ra.absSlot + ra.relSlot * (cabs(xr) + adt * cabs(k0)));
        });
      }
      const double err = blockMax(errLocal.value(), red);
      if (!(err == err)) {
        status |= 1u;
        return false;
      }
      if (err > 1.0) {
        dtTry = decreasedStep(dt, err);
        ++nFailed;
        if (!(dtTry > 0.) || t + dtTry == t) {
          status |= 4u;
          return false;
        }
        continue;
      }
      t += dt;
      dtTry = err < 0.5 ? increasedStep(dt, err) : dt;
      C2* const start = x;  // the candidate becomes the state; the step's start stays behind
      x = xalt;
      xalt = start;
      break;
    }
    dtDid = t - timeBefore;
    if (nextDtTry != 0.) dtTry = nextDtTry;
    return true;
  }

  // J_m applied to the state staged in ys0 (caller synchronised), result into out
  __device__ __forceinline__ void applyJump(int m, C2* out) const {
    const int SJ = sysp->SJ;
    const C2* jv = Tables<R>::jval(*sysp) + size_t(m) * SJ * D;
    const int* jc = sysp->jcol + size_t(m) * SJ * D;
    for (int r = threadIdx.x; r < D; r += blockDim.x) {
      C2 acc = mk<C2>(0, 0);
      for (int s = 0; s < SJ; ++s) acc = cfma(jv[s * D + r], ys0[jc[s * D + r]], acc);
      out[r] = acc;
    }
  }

  __device__ __forceinline__ bool coherentAndRates(double Dt, bool li, double (&rates)[MAX_JUMPS]) {
    if (hasH) {
      if (!odeStep(Dt)) return false;
    } else {
      const double stepToDo = li ? fmin(dtTry, Dt) : Dt;
      t += stepToDo;
      dtDid = stepToDo;
      if (li) {  // the state is changed in place below: keep the step's start for a step-back
        for (int r = threadIdx.x; r < D; r += blockDim.x) xalt[r] = x[r];
        C2* const start = x;
        x = xalt;
        xalt = start;
      }
    }
    // One pass over the state: the exact part (Exact::actWithU), the state staged for the
    // special jumps, the norm and the closed-form rates, each sum over this thread's rows in
    // row order.
    double v[NR];
    for (int m = 0; m < NR; ++m) v[m] = 0.;
    const bool stage = li && anySpecial;
    if (stage) __syncthreads();
    {
      const double tau = t - t0;
      unsigned wMask = 0u;  // jumps with closed-form rate weights
      if (li)
        for (int m = 0; m < nJ; ++m)
          if (sysp->jHasW[m]) wMask |= 1u << m;
      const double* const jw = sysp->jw;
      for (int r = threadIdx.x; r < D; r += blockDim.x) {
        C2 a = x[r];
        if (hasEx) {
          const double2 u = cexpScaledInline(tau, __ldg(&sysp->lambda[r]));
          a = mk<C2>(double(a.x) * u.x - double(a.y) * u.y, double(a.x) * u.y + double(a.y) * u.x);
          x[r] = a;
        }
        if (stage) ys0[r] = a;
        const double a2 = abs2(a);
        v[0] += a2;
#pragma unroll
        for (int m = 0; m < MAX_JUMPS; ++m)
          if (wMask >> m & 1u) v[m + 1] += __ldg(&jw[size_t(m) * D + r]) * a2;
      }
    }
    if (hasEx) t0 = t;
    if (stage) __syncthreads();
    int nRed = 1;
    if (li) {
      for (int m = 0; m < nJ; ++m) {
        if (sysp->jHasW[m]) continue;  // summed in the pass above
        // special jump: rate |J_m psi|^2 from the staged state
        double acc = 0.;
        const int SJ = sysp->SJ;
        const C2* jv = Tables<R>::jval(*sysp) + size_t(m) * SJ * D;
        const int* jc = sysp->jcol + size_t(m) * SJ * D;
        for (int r = threadIdx.x; r < D; r += blockDim.x) {
          C2 a = mk<C2>(0, 0);
          for (int s = 0; s < SJ; ++s) a = cfma(jv[s * D + r], ys0[jc[s * D + r]], a);
          acc += abs2(a);
        }
#pragma unroll
        for (int q = 0; q < MAX_JUMPS; ++q)
          if (q == m) v[q + 1] = acc;
      }
      nRed = 1 + nJ;
    }
    blockSumN(v, nRed, red);
    const double n = sqrt(v[0]);
    if (!(n > 0.) || !isfinite(n)) {
      status |= 1u;
      return false;
    }
    const double inv = 1. / n;
    for (int r = threadIdx.x; r < D; r += blockDim.x) {
      const C2 a = x[r];
      x[r] = mk<C2>(double(a.x) * inv, double(a.y) * inv);
    }
    maxNormDev = fmax(maxNormDev, fabs(1. - n));
    if (li) {
      bool ok = true;
      const double inv2 = 1. / v[0];
#pragma unroll
      for (int m = 0; m < MAX_JUMPS; ++m) {
        rates[m] = m < nJ ? v[m + 1] * inv2 : 0.;
        ok &= isfinite(rates[m]);
      }
      if (!ok) {
        status |= 2u;
        return false;
      }
    }
    return true;
  }

  __device__ __forceinline__ bool manageTimeStep(const double (&rates)[MAX_JUMPS], double tCache, double dtDidCache) {
    double totalRate = 0.;
#pragma unroll
    for (int m = 0; m < MAX_JUMPS; ++m)
      if (m < nJ) totalRate += rates[m];
    const double suggested = ra.dpLimit / totalRate;
    if (totalRate * dtDid > ra.overTol * ra.dpLimit) {
      maxTolOvershoot = fmax(maxTolOvershoot, totalRate * dtDid);
      t = tCache;
      dtDid = dtDidCache;
      dtTry = suggested;
      ++nBacks;
      return true;
    } else if (totalRate * dtTry > ra.dpLimit) {
      ++nOvershot;
      maxOvershoot = fmax(maxOvershoot, totalRate * dtTry);
    }
    dtTry = hasH ? fmin(dtTry, suggested) : suggested;
    return false;
  }

  __device__ __forceinline__ double uniform() {
    __syncthreads();
    if (threadIdx.x == 0) {
      double u;
      if (ra.rng == 0) {
        Pcg64 g;
        g.state.hi = bcast[0];
        g.state.lo = bcast[1];
        g.inc.hi = bcast[2];
        g.inc.lo = bcast[3];
        u = canonicalFromU64(g.next());
        bcast[0] = g.state.hi;
        bcast[1] = g.state.lo;
      } else {
        u = philoxUniform(ra.seed, ti, bcast[0]++);
      }
      reinterpret_cast<double*>(bcast)[4] = u;
    }
    __syncthreads();
    return reinterpret_cast<double*>(bcast)[4];
  }

  __device__ __forceinline__ bool performJump(const double (&rates)[MAX_JUMPS], const TrajDev& td) {
    double random = uniform() / dtDid;
    int lindbladNo = -1;
    double rate = 0.;
#pragma unroll
    for (int m = 0; m < MAX_JUMPS; ++m)
      if (m < nJ && lindbladNo < 0 && random > 0) {
        random -= rates[m];
        if (!(random > 0)) {
          lindbladNo = m;
          rate = rates[m];
        }
      }
    if (random < 0) {
      for (int r = threadIdx.x; r < D; r += blockDim.x) ys0[r] = x[r];
      __syncthreads();
      const double normFactor = sqrt(rate);
      if (!isfinite(normFactor) || !(normFactor > 0.)) {
        status |= 1u;
        return false;
      }
      applyJump(lindbladNo, x);
      const double inv = 1. / normFactor;
      for (int r = threadIdx.x; r < D; r += blockDim.x) {
        const C2 a = x[r];
        x[r] = mk<C2>(double(a.x) * inv, double(a.y) * inv);
      }
      if (threadIdx.x == 0 && td.jumpCap > 0) {
        const unsigned long long total = td.jumpN[ti] + nJumps;
        const unsigned long long slot = total % (unsigned long long)td.jumpCap;
        td.jumpT[ti * td.jumpCap + slot] = t;
        td.jumpL[ti * td.jumpCap + slot] = lindbladNo;
      }
      ++nJumps;
    }
    return true;
  }

  __device__ __forceinline__ bool step(double Dt, const TrajDev& td) {
    const bool li = ra.noise && nJ > 0;
    const double tCache = t, dtDidCache = dtDid;
    double rates[MAX_JUMPS];
    // with jumps, coherentAndRates leaves the step's start untouched in xalt
    if (!coherentAndRates(Dt, li, rates)) return false;
    if (li) {
      int backs = 0;
      while (manageTimeStep(rates, tCache, dtDidCache)) {
        if (++backs > 10000) {
          status |= 8u;
          return false;
        }
        C2* const discarded = x;  // back to the step's start
        x = xalt;
        xalt = discarded;
        if (!coherentAndRates(Dt, li, rates)) return false;
      }
      if (!performJump(rates, td)) return false;
    }
    ++nSteps;
    return true;
  }

  // Observables sum_slices sum_x w_k[x] |(F psi_slice)_x|^2 with F the k -> x transform of
  // quantumdata::ffTransform (LazyDensityOperatorFFT.cc:12-31): radix-2 backward DFT of each
  // slice along the axis (one warp per slice, in the second stage buffer), then
  // (F psi)_x = (-1)^x y_{(x + N/2) mod N} / sqrt(N), whose sign does not enter |.|^2.
  // The state is staged in ys0 by the caller.
  __device__ __noinline__ void fourierAverages(double* out) {
    const int N = sysp->fN, logN = sysp->fLog2, stride = sysp->fStride, nF = sysp->nF;
    const int nSlices = D / N, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double v[4] = {0., 0., 0., 0.};
    if (warp < nSlices) {
      C2* buf = ys1 + size_t(warp) * N;  // nSlices * N = D elements, one slice per warp
      for (int j = warp; j < nSlices; j += nw) {
        const int base = (j / stride) * (N * stride) + (j % stride);
        for (int m = lane; m < N; m += 32) buf[__brev(unsigned(m)) >> (32 - logN)] = ys0[base + m * stride];
        __syncwarp();
        for (int len = 2; len <= N; len <<= 1) {
          const int half = len >> 1;
          for (int bf = lane; bf < (N >> 1); bf += 32) {
            const int pos = bf % half, i0 = (bf / half) * len + pos, i1 = i0 + half;
            const double2 tw = __ldg(&sysp->fTw[pos * (N / len)]);  // exp(+2 pi i pos / len)
            const double sw = tw.y, cw = tw.x;
            const C2 a = buf[i0], bb = buf[i1];
            const R tx = R(cw) * bb.x - R(sw) * bb.y, ty = R(cw) * bb.y + R(sw) * bb.x;
            buf[i0] = mk<C2>(double(a.x + tx), double(a.y + ty));
            buf[i1] = mk<C2>(double(a.x - tx), double(a.y - ty));
          }
          __syncwarp();
        }
        for (int m = lane; m < N; m += 32) {
          const C2 yv = buf[(m + (N >> 1)) & (N - 1)];
          const double p = (double(yv.x) * double(yv.x) + double(yv.y) * double(yv.y)) / double(N);
#pragma unroll
          for (int f = 0; f < 4; ++f)  // over the compile-time bound: v stays in registers
            if (f < nF) v[f] += __ldg(&sysp->fW[size_t(f) * N + m]) * p;
        }
        __syncwarp();
      }
    }
    blockSumN(v, nF, red);
    if (threadIdx.x == 0 && out)
      for (int f = 0; f < nF; ++f) {
        const int k = sysp->fObs[f];
        if (sysp->oRe[k] >= 0) out[sysp->oRe[k]] = v[f];
      }
  }

  __device__ __forceinline__ void averages(double* out) {
    __syncthreads();
    for (int r = threadIdx.x; r < D; r += blockDim.x) ys0[r] = x[r];
    __syncthreads();
    const int nObs = sysp->nObs, SO = sysp->SO, nF = sysp->nF;
    if (nF) fourierAverages(out);
    for (int k = 0; k < nObs; ++k) {
      if (nF && sysp->oFourier[k]) continue;
      const double2* ov = sysp->oval + size_t(k) * SO * D;
      const int* oc = sysp->ocol + size_t(k) * SO * D;
      const int nSk = sysp->oS[k];
      double v[2] = {0., 0.};
      for (int r = threadIdx.x; r < D; r += blockDim.x) {
        double2 acc = make_double2(0., 0.);
        for (int s = 0; s < nSk; ++s) {
          const C2 y = ys0[oc[s * D + r]];
          acc = cfma(ov[s * D + r], make_double2(double(y.x), double(y.y)), acc);
        }
        const C2 xr = ys0[r];
        v[0] += double(xr.x) * acc.x + double(xr.y) * acc.y;
        v[1] += double(xr.x) * acc.y - double(xr.y) * acc.x;
      }
      blockSumN(v, 2, red);
      if (threadIdx.x == 0 && out) {
        const int cr = sysp->oRe[k], ci = sysp->oIm[k];
        if (cr >= 0) out[cr] = v[0];
        if (ci >= 0) out[ci] = v[1];
      }
    }
  }

  __device__ __forceinline__ void run(const TrajDev& td, int trajIndex) {
    ti = (unsigned long long)trajIndex;
    xslot = reinterpret_cast<C2*>(td.psi) + td.psiOff[trajIndex];
    x = xslot;
    xalt = second();
    t = td.t[ti];
    t0 = td.t0[ti];
    dtTry = td.dtTry[ti];
    dtDid = td.dtDid[ti];
    if (threadIdx.x < 4) bcast[threadIdx.x] = td.rng[4 * ti + threadIdx.x];
    nSteps = nAttempts = nFailed = nRhs = nOvershot = nBacks = nJumps = 0;
    maxOvershoot = td.maxima[3 * ti];
    maxTolOvershoot = td.maxima[3 * ti + 1];
    maxNormDev = td.maxima[3 * ti + 2];
    status = td.status[ti];
    __syncthreads();

    const int nOut = ra.mode == RUN_TO ? 1 : ra.nIntervals;
    const unsigned long long tStart = globalTimerNs();
    for (int k = 0; k < nOut && status == 0u; ++k) {
      long long guard = 0;
      if (ra.mode == RUN_STEPS) {
        for (int s = 0; s < ra.nSteps && t < ra.T; ++s)
          if (!step(ra.T - t, td)) break;
      } else {
        const double endTime = ra.mode == RUN_TO ? (ra.tEndPer ? ra.tEndPer[ti] : ra.tEnd) : t + ra.Dt;
        double dt;
        while ((dt = endTime - t) != 0.) {
          if (dt < 0. || ++guard > ra.maxStepsPerInterval ||
              ((guard & 63) == 0 && globalTimerNs() - tStart > ra.timeLimitNs)) {
            status |= 8u;
            break;
          }
          if (!step(dt, td)) break;
        }
      }
      if (ra.avrOut) {
        double* slot = ra.avrOut + ((size_t)k * td.nTraj + ti) * ra.nAvrStride;
        averages(slot);
        if (threadIdx.x == 0) slot[ra.nAvrStride - 1] = dtDid;
      }
    }
    if (x != xslot)  // the state ended in the second buffer (each thread copies its own rows)
      for (int r = threadIdx.x; r < D; r += blockDim.x) xslot[r] = x[r];
    __syncthreads();
    if (threadIdx.x < 4) td.rng[4 * ti + threadIdx.x] = bcast[threadIdx.x];
    if (threadIdx.x == 0) {
      td.t[ti] = t;
      td.t0[ti] = t0;
      td.dtTry[ti] = dtTry;
      td.dtDid[ti] = dtDid;
      unsigned long long* cw = td.cnt + 8 * ti;
      cw[0] += nSteps;
      cw[1] += nAttempts;
      cw[2] += nFailed;
      cw[3] += nRhs;
      cw[4] += nOvershot;
      cw[5] += nBacks;
      cw[6] += nJumps;
      cw[7] = status;
      td.maxima[3 * ti] = maxOvershoot;
      td.maxima[3 * ti + 1] = maxTolOvershoot;
      td.maxima[3 * ti + 2] = maxNormDev;
      td.status[ti] = status;
      td.jumpN[ti] += nJumps;
    }
    __syncthreads();
  }
};

// Dynamic shared memory: two stage buffers of `smemD` elements, the reduction scratch,
// 8 broadcast words, the interaction-picture phase table (bsc.phaseElems double2), then
// (without a scratch slab) the stage derivatives.
template <typename R, bool IP>
__global__ void __launch_bounds__(512, 1) mcwfBlockKernel(TrajDev td, RunArgs ra, BlockScratch bsc, int smemD) {
  using C2 = typename CT<R>::T;
  extern __shared__ __align__(16) unsigned char blockSmem[];
  C2* ys0 = reinterpret_cast<C2*>(blockSmem);
  C2* ys1 = ys0 + smemD;
  double* red = reinterpret_cast<double*>(ys1 + smemD);
  unsigned long long* bcast = reinterpret_cast<unsigned long long*>(red + 32 * (MAX_JUMPS + 1));
  __shared__ int task;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) task = atomicAdd(ra.queue, 1);
    __syncthreads();
    if (task >= ra.nTasks) return;
    const int ti = ra.order[task];
    const SysDev* s = td.systems + td.sysIdx[ti];
    BlockWorker<R, IP> w{s, ra};
    w.D = s->D;
    w.S = s->S;
    w.nJ = s->nJ;
    w.hasH = s->hasH != 0;
    w.hasEx = s->hasEx != 0;
    w.hasFreq = s->hasFreq != 0;
    w.anySpecial = false;
    for (int m = 0; m < w.nJ; ++m) w.anySpecial |= !s->jHasW[m];
    w.col = s->col;
    w.val = Tables<R>::val(*s);
    w.diag = Tables<R>::diag(*s);
    w.word = s->ctaWord;
    w.recF = s->ctaRecF;
    w.diagZero = s->diagZero != 0;
    w.freq = s->freq;
    // the phase table follows the broadcast words; shared-memory vectors follow the table
    double2* phTab = reinterpret_cast<double2*>(bcast + 8);
    w.fIdx = s->fIdx;
    w.fDist = s->fDist;
    w.nFD = s->nFD;
    w.phTab = IP && s->fIdx && s->nFD <= bsc.phaseElems ? phTab : nullptr;
    w.vec = bsc.base ? reinterpret_cast<C2*>(bsc.base) + size_t(blockIdx.x) * kBlockVectors * bsc.stride
                     : reinterpret_cast<C2*>(phTab + bsc.phaseElems);
    w.stride = bsc.stride;
    w.ys0 = ys0;
    w.ys1 = ys1;
    w.red = red;
    w.bcast = bcast;
    w.run(td, ti);
  }
}

}  // namespace dev
}  // namespace cqg
