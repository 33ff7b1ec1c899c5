// Fused MCWF trajectory kernel for sm_100a.
//
// One warp owns one trajectory at a time (persistent CTAs pull trajectories from a
// device work queue).  Lane l owns state rows r = l + 32 e, e < E; the state, the
// six Cash-Karp stage derivatives and the row's operator coefficients stay in
// registers for the whole run.  The only cross-lane traffic is the banded H/i gather
// (the stage vector is staged in a double-buffered shared-memory slab, one __syncwarp
// per right-hand side) and the warp-shuffle reductions for the error norm, the norm,
// the jump rates and the observables.  Everything the reference does per MCWF step
// is fused here:
//   ode_engine::Base::step + controlled Cash-Karp (ODE.h:234-262, Boost.Odeint)
//   Exact::actWithU, renormalisation           (MCWF_Trajectory.h:250-276)
//   rates, dpLimit control with step-back       (MCWF_Trajectory.h:279-317, 357-365)
//   jump selection and J_m psi / sqrt(rate)     (MCWF_Trajectory.h:320-344)
//   linear averages at every output time        (MCWF_Trajectory.h:406-420)
#pragma once

#include <cstdint>

#include "rng.cuh"

namespace cqg {
namespace dev {

constexpr int MAX_JUMPS = 8;
// Interaction-picture frequency tables: a system's distinct nonzero frequencies when there
// are at most kPhaseTableMax of them (the CTA kernel's shared-memory table); the warp kernel
// uses a table of at most kWarpPhaseTableMax.  kNoPhase indexes a zero frequency.
constexpr int kPhaseTableMax = 1024;
constexpr int kWarpPhaseTableMax = 128;
constexpr unsigned short kNoPhase = 0xffff;
// per-warp phase region of the warp kernel (double2 elements): the five Cash-Karp stage
// phases of each distinct frequency of the table, stage-major
constexpr int kWarpPhaseElems = 5 * kWarpPhaseTableMax;
constexpr unsigned FULL = 0xffffffffu;
// off-diagonal slots of the warp kernel's padded tables
constexpr int kWarpSlots = 8;
// Stage derivatives k1..k4 of the warp kernel live in shared memory (each lane touches only
// its own rows, so no synchronisation) when a lane holds three or four rows: their registers
// would otherwise cap the resident warps and spill.
__host__ __device__ constexpr bool warpStagesInShared(int E) { return E >= 3; }
// per-warp shared-memory vectors of DMAX elements: two stage-vector slabs, the step-back
// cache, and k1..k4 when they are kept there
__host__ __device__ constexpr int warpSmemVectors(int E) { return warpStagesInShared(E) ? 7 : 3; }

// ---- complex helpers ---------------------------------------------------------
template <typename R>
struct CT;
template <>
struct CT<double> {
  using T = double2;
};
template <>
struct CT<float> {
  using T = float2;
};

template <typename C2>
__device__ __forceinline__ C2 mk(double x, double y) {
  C2 r;
  r.x = x;
  r.y = y;
  return r;
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {  // acc + a*b
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 acc) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
  return acc;
}
template <typename C2>
__device__ __forceinline__ C2 cmul(C2 a, C2 b) {
  C2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C2, typename S>
__device__ __forceinline__ C2 axpy(S s, C2 v, C2 acc) {  // acc + s*v, s real
  acc.x = fma(s, v.x, acc.x);
  acc.y = fma(s, v.y, acc.y);
  return acc;
}
template <typename C2>
__device__ __forceinline__ double abs2(C2 a) {
  return double(a.x) * double(a.x) + double(a.y) * double(a.y);
}
template <typename C2>
__device__ __forceinline__ double cabs(C2 a) {
  return sqrt(double(a.x) * double(a.x) + double(a.y) * double(a.y));
}
// exp(tau * f) for complex f, in double.  cexpScaled is kept out of line: sincos/exp expand
// to a lot of code and are only needed in the interaction picture; the CTA kernel's per-row
// loops take the inline form (same operations, same results), where a call would save and
// restore the loop's live registers through local memory on every row.
__device__ __forceinline__ double2 cexpScaledInline(double tau, double2 f) {
  double s, c;
  sincos(tau * f.y, &s, &c);
  const double m = exp(tau * f.x);
  return make_double2(m * c, m * s);
}
static __device__ __noinline__ double2 cexpScaled(double tau, double2 f) { return cexpScaledInline(tau, f); }

// complex product with explicit roundings (no contraction choices left to the compiler)
__device__ __forceinline__ double2 cmulD(double2 a, double2 b) {
  return make_double2(__fma_rn(a.x, b.x, -__dmul_rn(a.y, b.y)), __fma_rn(a.x, b.y, __dmul_rn(a.y, b.x)));
}
// Interaction-picture phases of the Cash-Karp stages from one exponential per attempt: with
// E = exp(dt f / 40), stage s (c_s = 1/5, 3/10, 3/5, 1, 7/8) needs exp(c_s dt f) = E^n,
// n = 8, 12, 24, 40, 35, by repeated squaring (relative error ~ n ulp).
__device__ __forceinline__ void stagePhases(double2 E, double2* out, int stride) {
  const double2 e2 = cmulD(E, E), e4 = cmulD(e2, e2), e8 = cmulD(e4, e4);
  const double2 e12 = cmulD(e8, e4);
  const double2 e16 = cmulD(e8, e8), e32 = cmulD(e16, e16);
  out[0] = e8;
  out[stride] = e12;
  out[2 * stride] = cmulD(e12, e12);
  out[3 * stride] = cmulD(e32, e8);
  out[4 * stride] = cmulD(cmulD(e32, e2), E);
}

// ---- warp reductions -----------------------------------------------------------
__device__ __forceinline__ unsigned long long globalTimerNs() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
// sums of n <= N warp-uniform values at once (independent shuffles pipeline)
template <int N>
__device__ __forceinline__ void warpSumN(double (&v)[N], int n) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
#pragma unroll
    for (int m = 0; m < N; ++m)
      if (m < n) v[m] += __shfl_xor_sync(FULL, v[m], o);
  }
}

// Odeint's default step adjuster (decrease: max(0.9 err^(-1/(error order - 1)), 0.2);
// increase below err 0.5: 0.9 max(err, 5^-5)^(-1/stepper order)).  The decrease (a double
// pow, after a rejected attempt only) is out of line for code size.  The increase follows
// nearly every accepted attempt and is a few instructions: inline, since a call makes the
// caller save and restore its live registers through local memory on every attempt.
static __device__ __noinline__ double decreasedStep(double dt, double err) {
  return dt * fmax(0.9 * pow(err, -1. / 3.), 0.2);
}
// err^(-1/5) on [5^-5, 0.5] (the only range increasedStep sees) by Newton's method on
// f(y) = y^5 err - 1 started from a single-precision power: y <- y (1 + (1 - y^5 err) / 5).
// The start is good to ~1e-7 relative, the iteration converges quadratically, so two steps
// reach double precision (a few ulp, as pow) for a fraction of pow's instructions.
__device__ __forceinline__ double invFifthRoot(double err) {
  double y = double(__powf(float(err), -0.2f));
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double y2 = y * y;
    const double r = fma(-(y2 * y2 * y), err, 1.);
    y = fma(y * 0.2, r, y);
  }
  return y;
}
__device__ __forceinline__ double increasedStep(double dt, double err) {
  err = fmax(3.2e-4, err);  // 5^-5
  return dt * 0.9 * invFifthRoot(err);
}

// Running maximum over rows of |e_n| / den_n (the Odeint error norm) with no square root
// or division per row: a row replaces the current maximum when |e|^2 den_max^2 >
// |e_max|^2 den^2, and the maximum's ratio is formed once, by the same expression a direct
// evaluation uses.  Like fmax, rows whose ratio is NaN never become the maximum.
struct ErrNormMax {
  double n2 = 0., den = 1.;
  __device__ __forceinline__ void add(double e2, double d) {
    if (e2 * (den * den) > n2 * (d * d)) {
      n2 = e2;
      den = d;
    }
  }
  __device__ __forceinline__ double value() const { return sqrt(n2) / den; }
};

__device__ __forceinline__ double warpMax(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// ---- device-side system tables (see lowering.hpp) -----------------------------------
struct SysDev {
  int D, S, SJ, SO, nJ, nObs, nAvr;
  int hasH, hasEx, hasFreq;
  const int* col;        // [S][D]
  const int* jcol;       // [nJ][SJ][D]
  const double* jw;      // [nJ][D] rate weights
  const int* jHasW;      // [nJ]
  const int* ocol;       // [nObs][SO][D]
  const double2* oval;   // [nObs][SO][D]
  const int* oRe;        // [nObs]
  const int* oIm;        // [nObs]
  const int* oS;         // [nObs] slots used by each observable (<= SO; the rest is padding)
  // observables that the CTA kernel evaluates with a fast k -> x transform along one axis
  int nF;                // how many (0: none)
  int fN, fLog2, fStride;
  int fObs[4];           // their observable indices
  const int* oFourier;   // [nObs] 1: evaluated by the transform (CTA kernel), else 0
  const double* fW;      // [nF][fN] weights
  const double2* fTw;    // [fN / 2] twiddle factors exp(2 pi i k / fN) of the transform
  const double2* freq;   // [S][D] (IP) or null
  int nFD;               // IP with a table: distinct nonzero values of freq
  const unsigned short* fIdx;  // [S][D] index of freq into fDist (kNoPhase: zero), or null
  const double2* fDist;  // [nFD]
  const double2* lambda; // [D] (Exact) or null
  // Warp-kernel copies of the hot tables (D <= 128, S <= 8; null otherwise): rows padded to
  // Dp = 32 ceil(D / 32), slots padded to kWarpSlots, padding with zero coefficients, its own
  // row as column, no interaction-picture phase and zero rate weight and Exact exponent, so
  // that a warp's rows and slots need no validity tests.
  int Dp;
  const int* wcol;             // [kWarpSlots][Dp]
  const double2* wdiagD;       // [Dp]
  const double2* wvalD;        // [kWarpSlots][Dp]
  const float2* wdiagF;
  const float2* wvalF;
  const double* wjw;           // [nJ][Dp]
  const double2* wlambda;      // [Dp] (Exact) or null
  const unsigned short* wfIdx; // [kWarpSlots][Dp] (IP with a table) or null
  const double2* wfreq;        // [kWarpSlots][Dp] (IP) or null
  // CTA-kernel records of the ELL tables (D < 32768; null otherwise): per slot and row one
  // word, the column offset col - row as int16 in the low half and the distinct-frequency
  // index (kNoPhase without one) in the high half; for FP32 the word rides in one 16-byte
  // record with the coefficient {re, im, word, 0}, so a slot is one load
  int diagZero;                // the fused main diagonal is all zero
  const int* ctaWord;          // [S][D]
  const int4* ctaRecF;         // [S][D]
  // precision-specific copies
  const double2* diagD;
  const double2* valD;
  const double2* jvalD;
  const float2* diagF;
  const float2* valF;
  const float2* jvalF;
};

template <typename R>
struct Tables;
template <>
struct Tables<double> {
  __device__ static const double2* diag(const SysDev& s) { return s.diagD; }
  __device__ static const double2* val(const SysDev& s) { return s.valD; }
  __device__ static const double2* jval(const SysDev& s) { return s.jvalD; }
  __device__ static const double2* wdiag(const SysDev& s) { return s.wdiagD; }
  __device__ static const double2* wval(const SysDev& s) { return s.wvalD; }
};
template <>
struct Tables<float> {
  __device__ static const float2* diag(const SysDev& s) { return s.diagF; }
  __device__ static const float2* val(const SysDev& s) { return s.valF; }
  __device__ static const float2* jval(const SysDev& s) { return s.jvalF; }
  __device__ static const float2* wdiag(const SysDev& s) { return s.wdiagF; }
  __device__ static const float2* wval(const SysDev& s) { return s.wvalF; }
};

struct TrajDev {
  int nTraj;
  const int* sysIdx;
  const SysDev* systems;
  void* psi;                   // Real2 states
  const long long* psiOff;     // element offset of each trajectory's state
  double* t;
  double* t0;
  double* dtTry;
  double* dtDid;
  unsigned long long* rng;     // 4 words per trajectory
  unsigned long long* cnt;     // 8 counters per trajectory
  double* maxima;              // 3 per trajectory: dp overshoot, dp tolerance overshoot, |norm-1|
  unsigned* status;
  double* jumpT;               // [nTraj][jumpCap] ring
  int* jumpL;
  unsigned long long* jumpN;   // total jumps recorded per trajectory
  int jumpCap;
};

enum RunMode { RUN_INTERVALS = 0, RUN_TO = 1, RUN_STEPS = 2 };

struct RunArgs {
  int mode;
  double Dt;        // RUN_INTERVALS
  int nIntervals;   // RUN_INTERVALS / RUN_STEPS
  double tEnd;      // RUN_TO
  const double* tEndPer;  // RUN_TO: per-trajectory end times (indexed like the trajectory arrays) or null
  int nSteps;       // RUN_STEPS: steps per interval
  double T;         // RUN_STEPS: end time
  double absSlot, relSlot;  // Odeint error-checker slots (eps_abs, eps_rel after the swap)
  double dpLimit, overTol;
  int maxAttempts;
  int noise;
  int rng;
  unsigned long long seed;
  long long maxStepsPerInterval;
  unsigned long long timeLimitNs;  // wall-clock watchdog per trajectory task
  double* avrOut;   // [nOut][nTraj][nAvrStride] or null
  int nAvrStride;
  int* queue;
  const int* order;  // the launch's trajectories (a segment of the ensemble's order)
  int nTasks;        // how many
  int phaseCache;    // warp kernel: shared memory holds a per-warp interaction-picture phase table
  // Warp kernel, RUN_INTERVALS / RUN_TO: a warp yields its trajectory after yieldSteps MCWF
  // steps (0: never) and takes the next task, so that the end of a launch is one chunk of
  // steps long rather than one whole trajectory.  A yielding warp saves the trajectory with
  // its place in the run (ResumeInfo), reserves the next push slot (yieldTail) and publishes
  // the trajectory there (yieldEntry, then yieldSeq = slot + 1); tasks past nTasks are these
  // pushes in order.  When the slots run out (yieldCap) trajectories run on without yielding.
  int yieldSteps;
  int yieldCap;
  int* yieldTail;
  int* yieldEntry;
  int* yieldSeq;
  int* doneCount;     // trajectories of the launch that finished
  unsigned* queueError;  // set when a wait for a published push ran past the time limit
  struct ResumeInfo* resume;  // [trajectory] place of a yielded trajectory in the run
};

// Where a yielded trajectory resumes: output interval k, the end time and step count of the
// interval it is in (mid != 0).  Zeroed before every launch.
struct ResumeInfo {
  double endTime;
  long long guard;
  int k;
  int mid;
};

// Cash-Karp tableau (published coefficients)
struct CK {
  static constexpr double c1 = 1. / 5, c2 = 3. / 10, c3 = 3. / 5, c4 = 1., c5 = 7. / 8;
  static constexpr double a10 = 1. / 5;
  static constexpr double a20 = 3. / 40, a21 = 9. / 40;
  static constexpr double a30 = 3. / 10, a31 = -9. / 10, a32 = 6. / 5;
  static constexpr double a40 = -11. / 54, a41 = 5. / 2, a42 = -70. / 27, a43 = 35. / 27;
  static constexpr double a50 = 1631. / 55296, a51 = 175. / 512, a52 = 575. / 13824, a53 = 44275. / 110592,
                          a54 = 253. / 4096;
  static constexpr double b0 = 37. / 378, b2 = 250. / 621, b3 = 125. / 594, b5 = 512. / 1771;
  static constexpr double e0 = 37. / 378 - 2825. / 27648, e2 = 250. / 621 - 18575. / 48384,
                          e3 = 125. / 594 - 13525. / 55296, e4 = -277. / 14336, e5 = 512. / 1771 - 1. / 4;
};

// Per-warp shared scratch next to the state slabs.
// The rarely changed logger counters and maxima live here rather than in registers; the
// registers they free shorten the spills of the hot loops.  Lane 0 keeps them (every lane
// holds the same warp-uniform values).
struct alignas(16) WarpScratch {
  unsigned long long pcg[4];  // state hi, lo, increment hi, lo (pcg64); word 0 = draw count (philox)
  double mx[3];               // maximal dpLimit overshoot, maximal tolerance overshoot, norm deviation
  unsigned cnt[4];            // failed attempts, dpLimit overshoots, step-backs, jumps
};

// IP: the instance serves interaction-picture systems (rows with frequencies); Schroedinger-
// picture groups run the IP = false instance, which has no phase code at all.
template <typename R, int E, int SMAX, bool IP>
struct Worker {
  using C2 = typename CT<R>::T;

  // hot system fields in registers; the rest is read through sysp on rare paths
  const SysDev* sysp;
  const RunArgs& ra;
  const int lane;
  int D, S, nJ;
  bool hasH, hasEx, hasFreq, anySpecial;
  // the padded warp tables (SysDev::wcol ...): row stride DMAX, no validity tests
  static constexpr int DMAX = 32 * E;
  const int* col;
  const C2* val;
  const double2* freq;
  const double* jw;
  C2* buf0;
  C2* buf1;
  C2* cache;
  C2* kst;  // k1..k4, each DMAX elements (warpStagesInShared(E))
  static constexpr bool KSMEM = warpStagesInShared(E);
  WarpScratch* ws;
  double2* phs;  // per-warp phase region [5][kWarpPhaseTableMax] or null
  bool phsOn;    // this attempt's stage phases come from phs
  bool phsTab;   // the system's distinct frequencies fit the per-warp table
  const unsigned short* fIdx;  // with phsTab: distinct-frequency index per slot and row

  // Coefficients live in registers when E * SMAX is small (CREG), else they are
  // re-read per right-hand side through L1 (shared by all trajectories of the system).
  static constexpr bool CREG = E * SMAX <= 8;
  C2 diag[E];
  C2 cval[CREG ? SMAX : 1][E];
  int ccol[CREG ? SMAX : 1][E];
  // Otherwise the column indices still live in registers, one byte per slot (a warp's rows
  // are < 128), so that the gather from the staged state does not wait for a table load.
  static constexpr int CPACK = CREG ? 1 : (SMAX + 3) / 4;
  unsigned cpack[CPACK][E];

  // trajectory state
  C2 x[E];
  double t, t0, dtTry, dtDid;
  unsigned long long ti;
  // per-launch counter increments
  unsigned nSteps, nAttempts, nRhs;
  unsigned status;
  // rare logger counter c += 1, maximum c = max(maximum c, v) (WarpScratch::cnt / mx)
  __device__ __forceinline__ void bump(int c) {
    if (lane == 0) ws->cnt[c] += 1u;
  }
  __device__ __forceinline__ void maxTo(int c, double v) {
    if (lane == 0) ws->mx[c] = fmax(ws->mx[c], v);
  }

  __device__ __forceinline__ Worker(const SysDev* s, const RunArgs& a, int l, C2* b0, C2* b1, C2* c, WarpScratch* w,
                                    double2* ph)
      : sysp(s), ra(a), lane(l), buf0(b0), buf1(b1), cache(c), kst(c + DMAX), ws(w), phs(ph), phsOn(false),
        phsTab(false) {
    D = s->D;
    S = s->S;
    nJ = s->nJ;
    hasH = s->hasH != 0;
    hasEx = s->hasEx != 0;
    hasFreq = s->hasFreq != 0;
    col = s->wcol;
    val = Tables<R>::wval(*s);
    freq = s->wfreq;
    phsTab = ph && s->wfIdx && s->nFD <= kWarpPhaseTableMax;
    fIdx = s->wfIdx;
    jw = s->wjw;
    anySpecial = false;
    for (int m = 0; m < nJ; ++m) anySpecial |= !s->jHasW[m];
  }

  __device__ __forceinline__ int row(int e) const { return lane + 32 * e; }
  __device__ __forceinline__ bool valid(int e) const { return row(e) < D; }

  __device__ __forceinline__ void loadOperator() {
    const C2* dg = Tables<R>::wdiag(*sysp);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int r = row(e);
      diag[e] = dg[r];
      if constexpr (CREG) {
#pragma unroll
        for (int s = 0; s < SMAX; ++s) {
          ccol[s][e] = col[s * DMAX + r];
          cval[s][e] = val[s * DMAX + r];
        }
      } else {
#pragma unroll
        for (int w = 0; w < CPACK; ++w) {
          unsigned p = 0u;
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int s = 4 * w + b;
            if (s < SMAX) p |= unsigned(col[s * DMAX + r]) << (8 * b);
          }
          cpack[w][e] = p;
        }
      }
    }
  }

  // The stage phases exp(c_s dt f) of this attempt for every distinct frequency f of the
  // system (t == t0: the stage times are c_s dt past the picture's reference time): lane k
  // takes frequencies k, k + 32, ..., forms E = exp(dt f / 40) and its stage powers.  One
  // shared table per warp keeps the unrolled right-hand sides small (a per-row-and-slot phase
  // path beside it overflowed the instruction cache: ncu no_instruction stalls 2.7 -> 6.5
  // per issued instruction).
  __device__ __forceinline__ void preparePhases(double dt) {
    const double q = dt / 40.;
    __syncwarp();  // every lane is done with the previous attempt's table
    for (int k = lane; k < sysp->nFD; k += 32) {
      const double2 f = __ldg(&sysp->fDist[k]);
      stagePhases(cexpScaled(q, f), phs + k, kWarpPhaseTableMax);
    }
    __syncwarp();
  }

  // out = (H/i) y at picture time tau; y staged through `buf`

  // out = (H/i) y at picture time tau = stage time - t0 (stage 0..5 of the attempt)
  // Every row and slot of the padded tables is read: padding rows hold zeros and padding
  // slots a zero coefficient on the row itself, so there is no branch in the slot loops and
  // the loads of a right-hand side can all be issued ahead of their FMAs.
  __device__ __forceinline__ void rhs(const C2 (&y)[E], C2 (&out)[E], double tau, int stage, C2* buf) {
#pragma unroll
    for (int e = 0; e < E; ++e) buf[row(e)] = y[e];
    __syncwarp();
    ++nRhs;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      C2 acc = cmul(diag[e], y[e]);
      const int r = row(e);
#pragma unroll
      for (int s = 0; s < SMAX; ++s) {
        C2 c;
        int cc;
        if constexpr (CREG) {
          c = cval[s][e];
          cc = ccol[s][e];
        } else {
          c = __ldg(&val[s * DMAX + r]);
          cc = int((cpack[s >> 2][e] >> (8 * (s & 3))) & 0xffu);
        }
        if (IP && hasFreq) {
          if (phsOn) {
            if (stage) {
              const unsigned k = __ldg(&fIdx[s * DMAX + r]);
              const double2 ph = k == kNoPhase ? make_double2(1., 0.) : phs[(stage - 1) * kWarpPhaseTableMax + k];
              c = mk<C2>(double(c.x) * ph.x - double(c.y) * ph.y, double(c.x) * ph.y + double(c.y) * ph.x);
            }
          } else {
            const double2 f = __ldg(&freq[s * DMAX + r]);
            if ((f.x != 0. || f.y != 0.) && tau != 0.) {  // exp(0 f) = 1 exactly
              const double2 ph = cexpScaled(tau, f);
              c = mk<C2>(double(c.x) * ph.x - double(c.y) * ph.y, double(c.x) * ph.y + double(c.y) * ph.x);
            }
          }
        }
        acc = cfma(c, buf[cc], acc);
      }
      out[e] = acc;
    }
  }

  // The five further Cash-Karp stages of one attempt from k0 = (H/i) x, then the 5th-order
  // solution (into y) and the rows' part of Odeint's error norm.  Both variants compute the
  // same expressions in the same order (bit-identical): stagesRegisters keeps k1..k5 in
  // registers, stagesShared keeps k1..k4 in the warp's shared memory, each lane reading back
  // only the rows it wrote.
  __device__ __forceinline__ void stagesRegisters(double dt, const C2 (&k0)[E], C2 (&y)[E], ErrNormMax& errLocal) {
    C2 k1[E], k2[E], k3[E], k4[E], k5[E];
    {
      const R s0 = R(dt * CK::a10);
#pragma unroll
      for (int e = 0; e < E; ++e) y[e] = axpy(s0, k0[e], x[e]);
    }
    rhs(y, k1, t + CK::c1 * dt - t0, 1, buf1);
    {
      const R s0 = R(dt * CK::a20), s1 = R(dt * CK::a21);
#pragma unroll
      for (int e = 0; e < E; ++e) y[e] = axpy(s1, k1[e], axpy(s0, k0[e], x[e]));
    }
    rhs(y, k2, t + CK::c2 * dt - t0, 2, buf0);
    {
      const R s0 = R(dt * CK::a30), s1 = R(dt * CK::a31), s2 = R(dt * CK::a32);
#pragma unroll
      for (int e = 0; e < E; ++e) y[e] = axpy(s2, k2[e], axpy(s1, k1[e], axpy(s0, k0[e], x[e])));
    }
    rhs(y, k3, t + CK::c3 * dt - t0, 3, buf1);
    {
      const R s0 = R(dt * CK::a40), s1 = R(dt * CK::a41), s2 = R(dt * CK::a42), s3 = R(dt * CK::a43);
#pragma unroll
      for (int e = 0; e < E; ++e) y[e] = axpy(s3, k3[e], axpy(s2, k2[e], axpy(s1, k1[e], axpy(s0, k0[e], x[e]))));
    }
    rhs(y, k4, t + CK::c4 * dt - t0, 4, buf0);
    {
      const R s0 = R(dt * CK::a50), s1 = R(dt * CK::a51), s2 = R(dt * CK::a52), s3 = R(dt * CK::a53),
              s4 = R(dt * CK::a54);
#pragma unroll
      for (int e = 0; e < E; ++e)
        y[e] = axpy(s4, k4[e], axpy(s3, k3[e], axpy(s2, k2[e], axpy(s1, k1[e], axpy(s0, k0[e], x[e])))));
    }
    rhs(y, k5, t + CK::c5 * dt - t0, 5, buf1);
    solutionAndError(dt, k0, k2, k3, k4, k5, y, errLocal);
  }

  __device__ __forceinline__ void stagesShared(double dt, const C2 (&k0)[E], C2 (&y)[E], ErrNormMax& errLocal) {
    C2* const K1 = kst;
    C2* const K2 = kst + DMAX;
    C2* const K3 = kst + 2 * DMAX;
    C2* const K4 = kst + 3 * DMAX;
    C2 kc[E];
    {
      const R s0 = R(dt * CK::a10);
#pragma unroll
      for (int e = 0; e < E; ++e) y[e] = axpy(s0, k0[e], x[e]);
    }
    rhs(y, kc, t + CK::c1 * dt - t0, 1, buf1);
    {
      const R s0 = R(dt * CK::a20), s1 = R(dt * CK::a21);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        K1[row(e)] = kc[e];
        y[e] = axpy(s1, kc[e], axpy(s0, k0[e], x[e]));
      }
    }
    rhs(y, kc, t + CK::c2 * dt - t0, 2, buf0);
    {
      const R s0 = R(dt * CK::a30), s1 = R(dt * CK::a31), s2 = R(dt * CK::a32);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        K2[row(e)] = kc[e];
        y[e] = axpy(s2, kc[e], axpy(s1, K1[row(e)], axpy(s0, k0[e], x[e])));
      }
    }
    rhs(y, kc, t + CK::c3 * dt - t0, 3, buf1);
    {
      const R s0 = R(dt * CK::a40), s1 = R(dt * CK::a41), s2 = R(dt * CK::a42), s3 = R(dt * CK::a43);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        K3[row(e)] = kc[e];
        y[e] = axpy(s3, kc[e], axpy(s2, K2[row(e)], axpy(s1, K1[row(e)], axpy(s0, k0[e], x[e]))));
      }
    }
    rhs(y, kc, t + CK::c4 * dt - t0, 4, buf0);
    {
      const R s0 = R(dt * CK::a50), s1 = R(dt * CK::a51), s2 = R(dt * CK::a52), s3 = R(dt * CK::a53),
              s4 = R(dt * CK::a54);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        K4[row(e)] = kc[e];
        y[e] = axpy(s4, kc[e],
                    axpy(s3, K3[row(e)], axpy(s2, K2[row(e)], axpy(s1, K1[row(e)], axpy(s0, k0[e], x[e])))));
      }
    }
    rhs(y, kc, t + CK::c5 * dt - t0, 5, buf1);
    C2 k2[E], k3[E], k4[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      k2[e] = K2[row(e)];
      k3[e] = K3[row(e)];
      k4[e] = K4[row(e)];
    }
    solutionAndError(dt, k0, k2, k3, k4, kc, y, errLocal);
  }

  // 5th-order solution into y, embedded error and the rows' part of the Odeint error norm
  __device__ __forceinline__ void solutionAndError(double dt, const C2 (&k0)[E], const C2 (&k2)[E], const C2 (&k3)[E],
                                                   const C2 (&k4)[E], const C2 (&k5)[E], C2 (&y)[E],
                                                   ErrNormMax& errLocal) {
    const R b0 = R(dt * CK::b0), b2 = R(dt * CK::b2), b3 = R(dt * CK::b3), b5 = R(dt * CK::b5);
    const R e0 = R(dt * CK::e0), e2 = R(dt * CK::e2), e3 = R(dt * CK::e3), e4 = R(dt * CK::e4), e5 = R(dt * CK::e5);
    const double adt = fabs(dt);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      y[e] = axpy(b5, k5[e], axpy(b3, k3[e], axpy(b2, k2[e], axpy(b0, k0[e], x[e]))));
      C2 xe = mk<C2>(0, 0);
      xe = axpy(e5, k5[e], axpy(e4, k4[e], axpy(e3, k3[e], axpy(e2, k2[e], axpy(e0, k0[e], xe)))));
      // a padding row (all zero) never raises the maximum
      errLocal.add(abs2(xe), ra.absSlot + ra.relSlot * (cabs(x[e]) + adt * cabs(k0[e])));
    }
  }

  // one adaptive ODE step towards at most deltaT (ode_engine::Base::step, ODE.h:234-262,
  // with Boost.Odeint's controlled_runge_kutta<runge_kutta_cash_karp54>::try_step)
  __device__ __forceinline__ bool odeStep(double deltaT) {
    const double timeBefore = t;
    const double nextDtTry = fabs(deltaT) < fabs(dtTry / 10.) ? dtTry : 0.;
    if (fabs(dtTry) > fabs(deltaT)) dtTry = deltaT;
    C2 k0[E], y[E];
    // dxdt at the start is the same for every attempt (Odeint recomputes it per try)
    rhs(x, k0, t - t0, 0, buf0);
    for (int attempt = 0;; ++attempt) {
      if (attempt >= ra.maxAttempts) {
        status |= 8u;  // CQG_TRAJ_ATTEMPT_LIMIT
        return false;
      }
      ++nAttempts;
      const double dt = dtTry;
      if constexpr (IP) {
        phsOn = phsTab && hasFreq && t == t0;
        if (phsOn) preparePhases(dt);
      }
      ErrNormMax errLocal;
      if constexpr (KSMEM)
        stagesShared(dt, k0, y, errLocal);
      else
        stagesRegisters(dt, k0, y, errLocal);
      double err = warpMax(errLocal.value());
      if (!(err == err)) {  // NaN error norm
        status |= 1u;
        return false;
      }
      if (err > 1.0) {
        dtTry = decreasedStep(dt, err);
        bump(0);
        if (!(dtTry > 0.) || t + dtTry == t) {
          status |= 4u;  // CQG_TRAJ_DT_UNDERFLOW
          return false;
        }
        __syncwarp();  // the retry rewrites the buffer the last stage read
        continue;
      }
      t += dt;
      dtTry = err < 0.5 ? increasedStep(dt, err) : dt;
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = y[e];
      break;
    }
    dtDid = t - timeBefore;
    if (nextDtTry != 0.) dtTry = nextDtTry;
    return true;
  }

  // (J_m psi) rows into out; psi staged in buf (caller synchronised)
  __device__ __forceinline__ void applyJump(int m, const C2* buf, C2 (&out)[E]) const {
    const int SJ = sysp->SJ;
    const C2* jv = Tables<R>::jval(*sysp) + size_t(m) * SJ * D;
    const int* jc = sysp->jcol + size_t(m) * SJ * D;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      C2 acc = mk<C2>(0, 0);
      if (valid(e))
        for (int s = 0; s < SJ; ++s) acc = cfma(jv[s * D + row(e)], buf[jc[s * D + row(e)]], acc);
      out[e] = acc;
    }
  }

  // Coherent part of MCWF_Trajectory::step (coherentTimeDevelopment, MCWF_Trajectory.h:250-276)
  // fused with the rates of the renormalised state (:357-358): one warp reduction yields
  // ||psi||^2 and every sum_n w_n |psi_n|^2 (or ||J psi||^2), and rate = raw / ||psi||^2.
  __device__ __forceinline__ bool coherentAndRates(double Dt, bool li, double (&rates)[MAX_JUMPS]) {
    if (hasH) {
      if (!odeStep(Dt)) return false;
    } else {
      const double stepToDo = li ? fmin(dtTry, Dt) : Dt;
      t += stepToDo;
      dtDid = stepToDo;
    }
    if (hasEx) {
      // Exact::actWithU.  FP64 states: the factors exp(tau lambda) of this lane's rows are
      // formed by one inline copy of the exponential in a rolled loop and parked in the warp's
      // first stage buffer (free between steps), then applied; an out-of-line call here, even
      // never taken (Schroedinger-picture systems have no exact part), made the whole FP64
      // kernel's register allocation worse (qubit-mode 2x40 FP64: +1.2 % without it).  The
      // FP32 kernel measured 3 % slower that way and keeps one call per row.
      const double tau = t - t0;
      if constexpr (sizeof(R) == sizeof(double)) {
        double2* const u = reinterpret_cast<double2*>(buf0);
        __syncwarp();  // every lane is done with the last stage's gathers
#pragma unroll 1
        for (int e = 0; e < E; ++e) u[row(e)] = cexpScaledInline(tau, __ldg(&sysp->wlambda[row(e)]));
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const double2 ue = u[row(e)];
          x[e] = mk<C2>(double(x[e].x) * ue.x - double(x[e].y) * ue.y, double(x[e].x) * ue.y + double(x[e].y) * ue.x);
        }
        __syncwarp();
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const double2 u = cexpScaled(tau, __ldg(&sysp->wlambda[row(e)]));
          x[e] = mk<C2>(double(x[e].x) * u.x - double(x[e].y) * u.y, double(x[e].x) * u.y + double(x[e].y) * u.x);
        }
      }
      t0 = t;
    }
    double red[MAX_JUMPS + 1];
    red[0] = 0.;
#pragma unroll
    for (int e = 0; e < E; ++e) red[0] += abs2(x[e]);
    int nRed = 1;
    if (li) {
      if (anySpecial) {
#pragma unroll
        for (int e = 0; e < E; ++e) buf0[row(e)] = x[e];
        __syncwarp();
      }
#pragma unroll
      for (int m = 0; m < MAX_JUMPS; ++m) {
        red[m + 1] = 0.;
        if (m < nJ) {
          if (!anySpecial || sysp->jHasW[m]) {
            const double* w = jw + size_t(m) * DMAX;
#pragma unroll
            for (int e = 0; e < E; ++e) red[m + 1] += __ldg(&w[row(e)]) * abs2(x[e]);
          } else {
            C2 jx[E];
            applyJump(m, buf0, jx);
#pragma unroll
            for (int e = 0; e < E; ++e) red[m + 1] += abs2(jx[e]);
          }
        }
      }
      if (anySpecial) __syncwarp();
      nRed = 1 + nJ;
    }
    warpSumN(red, nRed);
    const double n = sqrt(red[0]);
    if (!(n > 0.) || !isfinite(n)) {
      status |= 1u;  // CQG_TRAJ_NONFINITE_NORM
      return false;
    }
    const double inv = 1. / n;
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = mk<C2>(double(x[e].x) * inv, double(x[e].y) * inv);
    maxTo(2, fabs(1. - n));
    if (li) {
      bool ok = true;
      const double inv2 = 1. / red[0];
#pragma unroll
      for (int m = 0; m < MAX_JUMPS; ++m) {
        rates[m] = m < nJ ? red[m + 1] * inv2 : 0.;
        ok &= isfinite(rates[m]);
      }
      if (!ok) {
        status |= 2u;  // CQG_TRAJ_NONFINITE_RATE
        return false;
      }
    }
    return true;
  }

  // MCWF_Trajectory::manageTimeStep (MCWF_Trajectory.h:294-317); true = step back
  __device__ __forceinline__ bool manageTimeStep(const double (&rates)[MAX_JUMPS], double tCache, double dtDidCache) {
    double totalRate = 0.;
#pragma unroll
    for (int m = 0; m < MAX_JUMPS; ++m)
      if (m < nJ) totalRate += rates[m];
    const double liouvilleanSuggestedDtTry = ra.dpLimit / totalRate;
    if (totalRate * dtDid > ra.overTol * ra.dpLimit) {
      maxTo(1, totalRate * dtDid);
      t = tCache;
      dtDid = dtDidCache;
      dtTry = liouvilleanSuggestedDtTry;
      bump(2);
      return true;
    } else if (totalRate * dtTry > ra.dpLimit) {
      bump(1);
      maxTo(0, totalRate * dtTry);
    }
    dtTry = hasH ? fmin(dtTry, liouvilleanSuggestedDtTry) : liouvilleanSuggestedDtTry;
    return false;
  }

  __device__ __forceinline__ double uniform() {
    double u = 0.;
    if (lane == 0) {
      if (ra.rng == 0) {
        Pcg64 g;
        g.state.hi = ws->pcg[0];
        g.state.lo = ws->pcg[1];
        g.inc.hi = ws->pcg[2];
        g.inc.lo = ws->pcg[3];
        u = canonicalFromU64(g.next());
        ws->pcg[0] = g.state.hi;
        ws->pcg[1] = g.state.lo;
      } else {
        u = philoxUniform(ra.seed, ti, ws->pcg[0]++);
      }
    }
    return __shfl_sync(FULL, u, 0);
  }

  // MCWF_Trajectory::performJump (MCWF_Trajectory.h:320-344)
  __device__ __forceinline__ bool performJump(const double (&rates)[MAX_JUMPS], const TrajDev& td) {
    double random = uniform() / dtDid;
    // for (; random > 0 && lindbladNo != nJ; random -= rates[lindbladNo++]) with static indices
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
#pragma unroll
      for (int e = 0; e < E; ++e) buf0[row(e)] = x[e];
      __syncwarp();
      C2 jx[E];
      applyJump(lindbladNo, buf0, jx);
      __syncwarp();
      const double normFactor = sqrt(rate);
      if (!isfinite(normFactor) || !(normFactor > 0.)) {
        status |= 1u;
        return false;
      }
      const double inv = 1. / normFactor;
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = mk<C2>(double(jx[e].x) * inv, double(jx[e].y) * inv);
      if (lane == 0 && td.jumpCap > 0) {
        const unsigned long long total = __ldcg(&td.jumpN[ti]) + ws->cnt[3];
        const unsigned long long slot = total % (unsigned long long)td.jumpCap;
        td.jumpT[ti * td.jumpCap + slot] = t;
        td.jumpL[ti * td.jumpCap + slot] = lindbladNo;
      }
      bump(3);
    }
    return true;
  }

  // MCWF_Trajectory::step (MCWF_Trajectory.h:347-374)
  __device__ __forceinline__ bool step(double Dt, const TrajDev& td) {
    const bool li = ra.noise && nJ > 0;
    const double tCache = t, dtDidCache = dtDid;
    if (li) {
#pragma unroll
      for (int e = 0; e < E; ++e) cache[row(e)] = x[e];
    }
    double rates[MAX_JUMPS];
    if (!coherentAndRates(Dt, li, rates)) return false;
    if (li) {
      int backs = 0;
      while (manageTimeStep(rates, tCache, dtDidCache)) {
        if (++backs > 10000) {
          status |= 8u;
          return false;
        }
#pragma unroll
        for (int e = 0; e < E; ++e) x[e] = cache[row(e)];
        if (!coherentAndRates(Dt, li, rates)) return false;
      }
      if (!performJump(rates, td)) return false;
    }
    ++nSteps;
    return true;
  }

  // per-trajectory linear averages <psi|O_k|psi> (output times only)
  __device__ __forceinline__ void averages(double* out) {
#pragma unroll
    for (int e = 0; e < E; ++e) buf0[row(e)] = x[e];
    __syncwarp();
    const int nObs = sysp->nObs, SO = sysp->SO;
    for (int k = 0; k < nObs; ++k) {
      const double2* ov = sysp->oval + size_t(k) * SO * D;
      const int* oc = sysp->ocol + size_t(k) * SO * D;
      const int nSk = sysp->oS[k];
      double re = 0., im = 0.;
#pragma unroll
      for (int e = 0; e < E; ++e)
        if (valid(e)) {
          double2 acc = make_double2(0., 0.);
          for (int s = 0; s < nSk; ++s) {
            const C2 v = buf0[oc[s * D + row(e)]];
            acc = cfma(ov[s * D + row(e)], make_double2(double(v.x), double(v.y)), acc);
          }
          const double xr = double(x[e].x), xi = double(x[e].y);
          re += xr * acc.x + xi * acc.y;  // conj(x) * acc
          im += xr * acc.y - xi * acc.x;
        }
      re = warpSum(re);
      im = warpSum(im);
      if (lane == 0 && out) {
        const int cr = sysp->oRe[k], ci = sysp->oIm[k];
        if (cr >= 0) out[cr] = re;
        if (ci >= 0) out[ci] = im;
      }
    }
    __syncwarp();
  }

  // One task: advances the trajectory through the run (its output intervals, or to its end
  // time), or, with ra.yieldSteps > 0, until it has taken that many MCWF steps and a push slot
  // was reserved for it: then it saves its place (ResumeInfo), writes *pushSlot and returns
  // false.  A trajectory may resume on another SM, so its state is read past L1 (__ldcg).
  __device__ __forceinline__ bool run(const TrajDev& td, int trajIndex, int* pushSlot) {
    ti = (unsigned long long)trajIndex;
    C2* psi = reinterpret_cast<C2*>(td.psi) + td.psiOff[trajIndex];
    loadOperator();
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = valid(e) ? __ldcg(&psi[row(e)]) : mk<C2>(0, 0);
    t = __ldcg(&td.t[ti]);
    t0 = __ldcg(&td.t0[ti]);
    dtTry = __ldcg(&td.dtTry[ti]);
    dtDid = __ldcg(&td.dtDid[ti]);
    if (lane < 4) ws->pcg[lane] = __ldcg(&td.rng[4 * ti + lane]);
    __syncwarp();
    nSteps = nAttempts = nRhs = 0;
    if (lane == 0) {
      ws->cnt[0] = ws->cnt[1] = ws->cnt[2] = ws->cnt[3] = 0u;
      ws->mx[0] = __ldcg(&td.maxima[3 * ti]);
      ws->mx[1] = __ldcg(&td.maxima[3 * ti + 1]);
      ws->mx[2] = __ldcg(&td.maxima[3 * ti + 2]);
    }
    status = __ldcg(&td.status[ti]);
    ResumeInfo rs{0., 0, 0, 0};
    if (ra.resume) {
      rs.endTime = __ldcg(&ra.resume[ti].endTime);
      rs.guard = __ldcg(&ra.resume[ti].guard);
      rs.k = __ldcg(&ra.resume[ti].k);
      rs.mid = __ldcg(&ra.resume[ti].mid);
    }

    const int nOut = ra.mode == RUN_TO ? 1 : ra.nIntervals;
    const unsigned long long tStart = globalTimerNs();
    bool yielded = false, mayYield = ra.yieldSteps > 0 && ra.mode != RUN_STEPS;
    int chunkSteps = 0;
    int k = rs.k;
    for (; k < nOut && status == 0u; ++k) {
      long long guard = rs.mid ? rs.guard : 0;
      if (ra.mode == RUN_STEPS) {
        for (int s = 0; s < ra.nSteps && t < ra.T; ++s)
          if (!step(ra.T - t, td)) break;
      } else {
        const double endTime =
            rs.mid ? rs.endTime : ra.mode == RUN_TO ? (ra.tEndPer ? ra.tEndPer[ti] : ra.tEnd) : t + ra.Dt;
        rs.mid = 0;
        double dt;
        while ((dt = endTime - t) != 0.) {
          if (mayYield && chunkSteps >= ra.yieldSteps) {
            int slot = 0;
            if (lane == 0) slot = atomicAdd(ra.yieldTail, 1);
            slot = __shfl_sync(FULL, slot, 0);
            if (slot < ra.yieldCap) {
              rs = ResumeInfo{endTime, guard, k, 1};
              *pushSlot = slot;
              yielded = true;
              break;
            }
            mayYield = false;  // no push slot left: run on
          }
          // bounded: a negative remainder, a step budget, or the wall-clock watchdog
          // end the trajectory with an error status instead of spinning
          if (dt < 0. || ++guard > ra.maxStepsPerInterval ||
              ((guard & 63) == 0 && globalTimerNs() - tStart > ra.timeLimitNs)) {
            status |= 8u;
            break;
          }
          if (!step(dt, td)) break;
          ++chunkSteps;
        }
      }
      if (yielded) break;
      if (ra.avrOut) {
        double* slot = ra.avrOut + ((size_t)k * td.nTraj + ti) * ra.nAvrStride;
        averages(slot);
        if (lane == 0) slot[ra.nAvrStride - 1] = dtDid;
      }
    }

#pragma unroll
    for (int e = 0; e < E; ++e)
      if (valid(e)) psi[row(e)] = x[e];
    __syncwarp();
    if (lane < 4) td.rng[4 * ti + lane] = ws->pcg[lane];
    if (lane == 0) {
      td.t[ti] = t;
      td.t0[ti] = t0;
      td.dtTry[ti] = dtTry;
      td.dtDid[ti] = dtDid;
      unsigned long long* cw = td.cnt + 8 * ti;
      cw[0] = __ldcg(&cw[0]) + nSteps;
      cw[1] = __ldcg(&cw[1]) + nAttempts;
      cw[2] = __ldcg(&cw[2]) + ws->cnt[0];
      cw[3] = __ldcg(&cw[3]) + nRhs;
      cw[4] = __ldcg(&cw[4]) + ws->cnt[1];
      cw[5] = __ldcg(&cw[5]) + ws->cnt[2];
      cw[6] = __ldcg(&cw[6]) + ws->cnt[3];
      cw[7] = status;
      td.maxima[3 * ti] = ws->mx[0];
      td.maxima[3 * ti + 1] = ws->mx[1];
      td.maxima[3 * ti + 2] = ws->mx[2];
      td.status[ti] = status;
      td.jumpN[ti] = __ldcg(&td.jumpN[ti]) + ws->cnt[3];
      if (yielded) ra.resume[ti] = rs;
    }
    __syncwarp();
    return !yielded;
    __syncwarp();
  }
};

// CTAs of 128 threads the compiler must fit on one SM.  Three (at most 170 registers per
// thread, some spills) for the Schroedinger-picture instance with three rows per lane, where
// the 12 resident warps hide more latency than the spills cost (qubit-mode 2x40: FP64 113.0
// -> 117.8 M steps/s, FP32 122.7 -> 141.2 M, with the stage derivatives in registers); one
// (255 registers, 8 warps) elsewhere, where three or four measured slower (pumped lossy mode
// E = 1: -1 % / -12 %; interaction-picture E = 3: -6 % / -14 %).
template <int E, bool IP>
struct WarpMinBlocks {
  static constexpr int value = (!IP && E == 3) ? 3 : 1;
};
// A second instance with more resident CTAs (fewer registers) for Schroedinger-picture groups
// with three or four rows per lane and at most four slots, whose stage derivatives k1..k4 sit
// in shared memory; the autotuner times both and keeps the faster.
__host__ __device__ constexpr bool warpHighOccupancyVariant(int E, int SMAX, bool IP) {
  return !IP && E >= 3 && SMAX <= 4;
}
template <int E>
struct WarpMinBlocksHigh {
  static constexpr int value = E == 3 ? 4 : 3;
};

template <typename R, int E, int SMAX, bool IP, int MINB>
__global__ void __launch_bounds__(128, MINB) mcwfWarpKernel(TrajDev td, RunArgs ra) {
  using C2 = typename CT<R>::T;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int DMAX = 32 * E;
  constexpr int NV = warpSmemVectors(E);
  C2* base = reinterpret_cast<C2*>(smem) + size_t(warp) * NV * DMAX;
  WarpScratch* ws =
      reinterpret_cast<WarpScratch*>(smem + size_t(blockDim.x / 32) * NV * DMAX * sizeof(C2)) + warp;
  // optional phase tables after every warp's scratch: [warps][kWarpPhaseElems] double2
  double2* phs = IP && ra.phaseCache ? reinterpret_cast<double2*>(reinterpret_cast<WarpScratch*>(
                                     smem + size_t(blockDim.x / 32) * NV * DMAX * sizeof(C2)) +
                                 blockDim.x / 32) +
                                     size_t(warp) * kWarpPhaseElems
                               : nullptr;
  while (true) {
    int task = 0;
    if (lane == 0) task = atomicAdd(ra.queue, 1);
    task = __shfl_sync(FULL, task, 0);
    int ti;
    if (task < ra.nTasks) {
      ti = ra.order[task];
    } else {
      // Tasks past nTasks are the yielded trajectories in push order.  Wait until push p is
      // published, or every trajectory of the launch is done (no push will come), or the
      // wall-clock limit passes (an error the host reports).
      const int p = task - ra.nTasks;
      if (ra.yieldSteps <= 0 || p >= ra.yieldCap) return;
      int got = -1;
      if (lane == 0) {
        const unsigned long long tw = globalTimerNs();
        volatile int* seq = ra.yieldSeq;
        volatile int* done = ra.doneCount;
        // the polls back off (128 ns doubling to 4 us): the waiting warps of a launch's tail
        // would otherwise keep the queue's few cache lines busy for the warps that still run
        unsigned sleepNs = 128;
        while (true) {
          if (seq[p] == p + 1) {
            __threadfence();
            got = reinterpret_cast<volatile int*>(ra.yieldEntry)[p];
            break;
          }
          if (*done >= ra.nTasks) break;
          if (globalTimerNs() - tw > ra.timeLimitNs) {
            atomicOr(ra.queueError, 1u);
            break;
          }
          __nanosleep(sleepNs);
          if (sleepNs < 4096) sleepNs <<= 1;
        }
      }
      got = __shfl_sync(FULL, got, 0);
      if (got < 0) return;
      ti = got;
    }
    Worker<R, E, SMAX, IP> w(td.systems + td.sysIdx[ti], ra, lane, base, base + DMAX, base + 2 * DMAX, ws, phs);
    int slot = -1;
    const bool finished = w.run(td, ti, &slot);
    if (ra.yieldSteps > 0) {  // the queue's counters and marks exist only when yielding is on
      __threadfence();        // the trajectory's state is visible before it is counted or published
      __syncwarp();
      if (lane == 0) {
        if (finished) {
          atomicAdd(ra.doneCount, 1);
        } else {
          ra.yieldEntry[slot] = ti;
          __threadfence();
          atomicExch(&ra.yieldSeq[slot], slot + 1);
        }
      }
    }
  }
}

}  // namespace dev
}  // namespace cqg
