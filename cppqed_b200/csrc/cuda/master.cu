// Master equation on the device (cqg_master_*): the reference's Master trajectory
// (quantumtrajectory::Master, Master.h:153-208) for the same lowered system.
//
//   drho/dt = A rho + (A rho)^+ + sum_m J_m rho J_m^+,     A = H/i (non-Hermitian H_eff / i)
//
// A acts on every column of rho (fullRange<Left>), the Hermitian part is taken
// (calculateTwoTimesRealPartOfSelf), and each jump term is J on the columns, a Hermitian
// conjugate, J on the columns again.  The step is the same controlled Cash-Karp as the MCWF
// trajectories (ode_engine::Base::step with Odeint's error checker and step adjuster) over
// all D^2 elements; after each step the exact part acts as rho -> U rho U^+, t0 = t, and rho
// is made exactly Hermitian and normalised.
//
// Layout: rho column-major (element (i, j) at j*D + i), so that every column is a contiguous
// state and A is the batched H/i application of apply.cu over the D columns.  Elementwise
// work (stage combinations, error norm, exact factors) streams the D^2 elements; the
// Hermitian parts and conjugate transposes go through 32 x 32 shared-memory tiles.  Step
// control runs on the host: one 8-byte read-back of the error norm per attempt.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "engine_internal.cuh"

using cqg::fail;
using namespace cqg::engine;
namespace dev = cqg::dev;

namespace {

constexpr int kTile = 32;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// h(i, j) = a(i, j) + conj(a(j, i)), diagonal 2 Re a(i, i)   (calculateTwoTimesRealPartOfSelf)
// or, with conjTransposeOnly, h(i, j) = conj(a(j, i)).  Block (32, 8) per 32 x 32 tile.
__global__ void tileKernel(const double2* __restrict__ a, double2* __restrict__ h, int D, bool conjTransposeOnly) {
  __shared__ double2 t[kTile][kTile + 1];
  const int i0 = blockIdx.x * kTile, j0 = blockIdx.y * kTile;
  // transposed tile: rows j0.., columns i0.. of a, i.e. a(j, i) for this tile's (i, j)
  for (int k = threadIdx.y; k < kTile; k += blockDim.y) {
    const int r = j0 + threadIdx.x, c = i0 + k;  // a(r, c), column-major: c * D + r
    if (r < D && c < D) t[k][threadIdx.x] = a[size_t(c) * D + r];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < kTile; k += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + k;
    if (i >= D || j >= D) continue;
    const double2 aji = t[threadIdx.x][k];  // a(j, i)
    double2 v;
    if (conjTransposeOnly)
      v = cconj(aji);
    else if (i == j)
      v = make_double2(2. * aji.x, 0.);
    else
      v = cadd(a[size_t(j) * D + i], cconj(aji));
    h[size_t(j) * D + i] = v;
  }
}

// out(:, j) (+)= J_m in(:, j) for every column j (mcwf jump tables [M][SJ][D])
__global__ void jumpColumnsKernel(dev::SysDev sd, int m, const double2* __restrict__ in, double2* __restrict__ out,
                                  bool accumulate) {
  const long long D = sd.D, total = D * D;
  const double2* jv = sd.jvalD + size_t(m) * sd.SJ * D;
  const int* jc = sd.jcol + size_t(m) * sd.SJ * D;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    const long long j = g / D, i = g - j * D;
    const double2* col = in + j * D;
    double2 acc = make_double2(0., 0.);
    for (int s = 0; s < sd.SJ; ++s) acc = cqg::dev::cfma(__ldg(&jv[s * D + i]), col[__ldg(&jc[s * D + i])], acc);
    out[g] = accumulate ? cadd(out[g], acc) : acc;
  }
}

// y = x + sum_k c_k K_k (k < n), and optionally the embedded error e = sum_k d_k K_k with
// Odeint's error norm max |e| / (abs + rel (|x| + |dt| |K_0|)) into errMax (as ordered bits)
struct Combo {
  const double2* K[6];
  double c[6], d[6];
  int n;
  double absSlot, relSlot, adt;
};

__global__ void comboKernel(const double2* __restrict__ x, double2* __restrict__ y, Combo cb, long long total,
                            unsigned long long* errMax) {
  double local = 0.;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    double2 acc = x[g];
    double2 e = make_double2(0., 0.);
    for (int k = 0; k < cb.n; ++k) {
      const double2 v = cb.K[k][g];
      acc.x = fma(cb.c[k], v.x, acc.x);
      acc.y = fma(cb.c[k], v.y, acc.y);
      if (errMax) {
        e.x = fma(cb.d[k], v.x, e.x);
        e.y = fma(cb.d[k], v.y, e.y);
      }
    }
    y[g] = acc;
    if (errMax) {
      const double2 xv = x[g], k0 = cb.K[0][g];
      const double w = cb.absSlot + cb.relSlot * (hypot(xv.x, xv.y) + cb.adt * hypot(k0.x, k0.y));
      const double q = hypot(e.x, e.y) / w;
      local = q == q ? fmax(local, q) : INFINITY;  // a NaN anywhere makes the norm infinite
    }
  }
  if (errMax) {
    for (int o = 16; o; o >>= 1) local = fmax(local, __shfl_xor_sync(0xffffffffu, local, o));
    // non-negative doubles order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(errMax, __double_as_longlong(local));
  }
}

// U_i = exp(lambda_i tau) (Exact::actWithU's diagonal)
__global__ void exactFactorsKernel(const double2* __restrict__ lambda, double tau, int D, double2* __restrict__ u) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D; i += gridDim.x * blockDim.x)
    u[i] = cqg::dev::cexpScaled(tau, lambda[i]);
}

// rho(i, j) <- conj(U_j) (U_i rho(i, j)) (actWithU on the columns, then on the rows of the
// conjugate)
__global__ void exactKernel(double2* __restrict__ r, const double2* __restrict__ u, int D) {
  const long long total = (long long)D * D;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    const long long j = g / D, i = g - j * D;
    r[g] = cmul(cconj(u[j]), cmul(u[i], r[g]));
  }
}

// trace, then rho /= Re tr (StateVector-like renorm of the density operator)
__global__ void traceKernel(const double2* __restrict__ r, int D, double* out) {
  __shared__ double part[256];
  double acc = 0.;
  for (int i = threadIdx.x; i < D; i += blockDim.x) acc += r[size_t(i) * D + i].x;
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = part[0];
}

__global__ void scaleKernel(double2* __restrict__ r, long long total, const double* tr) {
  const double s = *tr;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    r[g].x /= s;
    r[g].y /= s;
  }
}

// Tr(O_k rho) = sum_i sum_s O[k][s][i] rho(col, i): one block per observable, fixed order
__global__ void averagesKernel(dev::SysDev sd, const double2* __restrict__ r, double* __restrict__ out) {
  const int k = blockIdx.x, D = sd.D;
  const double2* ov = sd.oval + size_t(k) * sd.SO * D;
  const int* oc = sd.ocol + size_t(k) * sd.SO * D;
  const int nS = sd.oS[k];
  __shared__ double re[256], im[256];
  double a = 0., b = 0.;
  for (int i = threadIdx.x; i < D; i += blockDim.x) {
    double2 acc = make_double2(0., 0.);
    for (int s = 0; s < nS; ++s) acc = cqg::dev::cfma(ov[s * D + i], r[size_t(i) * D + oc[s * D + i]], acc);
    a += acc.x;
    b += acc.y;
  }
  re[threadIdx.x] = a;
  im[threadIdx.x] = b;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if (threadIdx.x < o) {
      re[threadIdx.x] += re[threadIdx.x + o];
      im[threadIdx.x] += im[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (sd.oRe[k] >= 0) out[sd.oRe[k]] = re[0];
    if (sd.oIm[k] >= 0) out[sd.oIm[k]] = im[0];
  }
}

// Cash-Karp tableau (published coefficients)
const double kA[5][5] = {{1. / 5},
                         {3. / 40, 9. / 40},
                         {3. / 10, -9. / 10, 6. / 5},
                         {-11. / 54, 5. / 2, -70. / 27, 35. / 27},
                         {1631. / 55296, 175. / 512, 575. / 13824, 44275. / 110592, 253. / 4096}};
const double kC[6] = {0., 1. / 5, 3. / 10, 3. / 5, 1., 7. / 8};
const double kB5[6] = {37. / 378, 0., 250. / 621, 125. / 594, 0., 512. / 1771};
const double kB4[6] = {2825. / 27648, 0., 18575. / 48384, 13525. / 55296, 277. / 14336, 1. / 4};

}  // namespace

struct cqg_master {
  const cqg_system* sys = nullptr;
  int device = 0, nSM = 0;
  int64_t D = 0;
  cqg_mcwf_pars pars{};
  cudaStream_t stream = nullptr;
  void* dmem = nullptr;
  double2* rho = nullptr;
  double2* K[6] = {};
  double2* y = nullptr;
  double2* xout = nullptr;
  double2* t1 = nullptr;
  double2* t2 = nullptr;
  unsigned long long* dErr = nullptr;
  double* dScalar = nullptr;
  double* dAvr = nullptr;
  double2* u = nullptr;  // exact factors [D]
  double t = 0, t0 = 0, dtTry = 0, dtDid = 0;
  uint64_t nSteps = 0, nAttempts = 0, nFailed = 0;
  ~cqg_master() {
    if (dmem) cudaFree(dmem);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

unsigned gridFor(long long total, int nSM) {
  return unsigned(std::max<long long>(1, std::min<long long>((total + 255) / 256, (long long)nSM * 8)));
}

// drho = A rho + (A rho)^+ + sum_m J_m rho J_m^+ at time tt
void derivs(cqg_master& m, const double2* r, double2* dr, double tt) {
  const dev::SysDev& sd = m.sys->sd;
  const long long D = m.D, total = D * D;
  cudaStream_t st = m.stream;
  const dim3 tiles(unsigned((D + kTile - 1) / kTile), unsigned((D + kTile - 1) / kTile)), tb(kTile, 8);
  ck(cudaMemsetAsync(m.t1, 0, size_t(total) * sizeof(double2), st), "cudaMemsetAsync");
  ck(applyHamiltonian(sd, r, m.t1, D, tt - m.t0, st, m.nSM), "master: H/i on the columns");
  tileKernel<<<tiles, tb, 0, st>>>(m.t1, dr, int(D), false);
  ck(cudaGetLastError(), "master: Hermitian part");
  for (int j = 0; j < sd.nJ; ++j) {
    jumpColumnsKernel<<<gridFor(total, m.nSM), 256, 0, st>>>(sd, j, r, m.t1, false);
    tileKernel<<<tiles, tb, 0, st>>>(m.t1, m.t2, int(D), true);
    jumpColumnsKernel<<<gridFor(total, m.nSM), 256, 0, st>>>(sd, j, m.t2, dr, true);
    ck(cudaGetLastError(), "master: jump terms");
  }
}

// one try of the controlled Cash-Karp step of size dt; returns the error norm
double tryStep(cqg_master& m, double dt) {
  const long long total = m.D * m.D;
  cudaStream_t st = m.stream;
  derivs(m, m.rho, m.K[0], m.t);
  for (int s = 1; s < 6; ++s) {
    Combo cb{};
    cb.n = s;
    for (int k = 0; k < s; ++k) {
      cb.K[k] = m.K[k];
      cb.c[k] = dt * kA[s - 1][k];
    }
    comboKernel<<<gridFor(total, m.nSM), 256, 0, st>>>(m.rho, m.y, cb, total, nullptr);
    ck(cudaGetLastError(), "master: stage");
    derivs(m, m.y, m.K[s], m.t + kC[s] * dt);
  }
  Combo cb{};
  cb.n = 6;
  for (int k = 0; k < 6; ++k) {
    cb.K[k] = m.K[k];
    cb.c[k] = dt * kB5[k];
    cb.d[k] = dt * (kB5[k] - kB4[k]);
  }
  cb.absSlot = m.pars.eps_rel;  // make_controlled(epsRel, epsAbs, ...) (ODE.h:205)
  cb.relSlot = m.pars.eps_abs;
  cb.adt = std::fabs(dt);
  ck(cudaMemsetAsync(m.dErr, 0, sizeof(unsigned long long), st), "cudaMemsetAsync");
  comboKernel<<<gridFor(total, m.nSM), 256, 0, st>>>(m.rho, m.xout, cb, total, m.dErr);
  ck(cudaGetLastError(), "master: solution");
  unsigned long long bits = 0;
  ck(cudaMemcpyAsync(&bits, m.dErr, sizeof(bits), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  ck(cudaStreamSynchronize(st), "master: step");
  double err;
  std::memcpy(&err, &bits, sizeof(err));
  return err;
}

// ode_engine::Base::step (ODE.h:234-262) then the Master::step epilogue (Master.h:185-206)
void step(cqg_master& m, double deltaT) {
  const double timeBefore = m.t;
  const double nextDtTry = std::fabs(deltaT) < std::fabs(m.dtTry / 10.) ? m.dtTry : 0.;
  if (std::fabs(m.dtTry) > std::fabs(deltaT)) m.dtTry = deltaT;
  for (int attempt = 0;; ++attempt) {
    if (attempt >= std::max(1, m.pars.max_attempts)) throw std::runtime_error("master: ODE attempt limit exceeded");
    ++m.nAttempts;
    const double dt = m.dtTry;
    double err = tryStep(m, dt);
    if (!std::isfinite(err)) throw std::runtime_error("master: non-finite error norm");
    if (err > 1.) {
      m.dtTry = dt * std::max(0.9 * std::pow(err, -1. / 3.), 0.2);
      ++m.nFailed;
      continue;
    }
    m.t += dt;
    if (err < 0.5) {
      err = std::max(std::pow(5., -5.), err);
      m.dtTry = dt * 0.9 * std::pow(err, -1. / 5.);
    }
    std::swap(m.rho, m.xout);
    break;
  }
  m.dtDid = m.t - timeBefore;
  if (nextDtTry) m.dtTry = nextDtTry;
  ++m.nSteps;

  const long long D = m.D, total = D * D;
  cudaStream_t st = m.stream;
  const dev::SysDev& sd = m.sys->sd;
  if (sd.lambda) {
    exactFactorsKernel<<<unsigned((D + 255) / 256), 256, 0, st>>>(sd.lambda, m.t - m.t0, int(D), m.u);
    exactKernel<<<gridFor(total, m.nSM), 256, 0, st>>>(m.rho, m.u, int(D));
    ck(cudaGetLastError(), "master: exact part");
  }
  m.t0 = m.t;
  const dim3 tiles(unsigned((D + kTile - 1) / kTile), unsigned((D + kTile - 1) / kTile)), tb(kTile, 8);
  tileKernel<<<tiles, tb, 0, st>>>(m.rho, m.xout, int(D), false);
  std::swap(m.rho, m.xout);
  traceKernel<<<1, 256, 0, st>>>(m.rho, int(D), m.dScalar);
  scaleKernel<<<gridFor(total, m.nSM), 256, 0, st>>>(m.rho, total, m.dScalar);
  ck(cudaGetLastError(), "master: renormalisation");
}

void averages(cqg_master& m, double* row) {
  const dev::SysDev& sd = m.sys->sd;
  const int nAvr = m.sys->L.nAvr;
  if (sd.nObs) {
    ck(cudaMemsetAsync(m.dAvr, 0, size_t(std::max(nAvr, 1)) * sizeof(double), m.stream), "cudaMemsetAsync");
    averagesKernel<<<sd.nObs, 256, 0, m.stream>>>(sd, m.rho, m.dAvr);
    ck(cudaGetLastError(), "master: averages");
    ck(cudaMemcpyAsync(row, m.dAvr, size_t(nAvr) * sizeof(double), cudaMemcpyDeviceToHost, m.stream),
       "cudaMemcpyAsync");
  }
  ck(cudaStreamSynchronize(m.stream), "master: averages");
  row[nAvr] = m.dtDid;
}

}  // namespace

extern "C" {

int cqg_master_create(const cqg_system* sys, const cqg_complex* psi0, const cqg_mcwf_pars* pars, cqg_master** out) {
  return guardedCuda([&] {
    if (!sys || !psi0 || !pars || !out) return fail(CQG_E_INVALID, "cqg_master_create: null argument");
    if (!(pars->eps_rel > 0) || !(pars->eps_abs >= 0)) return fail(CQG_E_INVALID, "cqg_master_create: eps_rel > 0 required");
    auto m = std::make_unique<cqg_master>();
    m->sys = sys;
    m->D = sys->L.D;
    m->pars = *pars;
    if (m->pars.max_attempts <= 0) m->pars.max_attempts = 100000;
    m->device = sys->device;
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    ck(cudaDeviceGetAttribute(&m->nSM, cudaDevAttrMultiProcessorCount, m->device), "attribute");
    ck(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    const size_t n = size_t(m->D) * size_t(m->D), mat = ((n * sizeof(double2)) + 255) & ~size_t(255);
    const size_t avrBytes = (size_t(sys->L.nAvr + 1) * sizeof(double) + 255) & ~size_t(255);
    const size_t total = 11 * mat + 1024 + avrBytes + size_t(m->D) * sizeof(double2);
    ck(cudaMalloc(&m->dmem, total), "cudaMalloc(master)");
    char* b = static_cast<char*>(m->dmem);
    double2** bufs[11] = {&m->rho, &m->K[0], &m->K[1], &m->K[2], &m->K[3], &m->K[4], &m->K[5],
                          &m->y, &m->xout, &m->t1, &m->t2};
    for (int k = 0; k < 11; ++k) *bufs[k] = reinterpret_cast<double2*>(b + k * mat);
    m->dErr = reinterpret_cast<unsigned long long*>(b + 11 * mat);
    m->dScalar = reinterpret_cast<double*>(b + 11 * mat + 256);
    m->dAvr = reinterpret_cast<double*>(b + 11 * mat + 1024);
    m->u = reinterpret_cast<double2*>(b + 11 * mat + 1024 + avrBytes);
    // rho = |psi0><psi0|, column-major
    std::vector<double2> rho(n);
    const int64_t D = m->D;
    for (int64_t j = 0; j < D; ++j)
      for (int64_t i = 0; i < D; ++i) {
        const cqg_complex a = psi0[i], c = psi0[j];
        rho[size_t(j) * D + i] = make_double2(a.re * c.re + a.im * c.im, a.im * c.re - a.re * c.im);
      }
    ck(cudaMemcpy(m->rho, rho.data(), n * sizeof(double2), cudaMemcpyHostToDevice), "cudaMemcpy(rho)");
    m->dtTry = pars->dt_init > 0 ? pars->dt_init : 1. / (10. * sys->L.highestFrequency);
    *out = m.release();
    return CQG_OK;
  });
}

int cqg_master_run(cqg_master* m, double Dt, int32_t n_intervals, double* avr_out) {
  return guardedCuda([&] {
    if (!m || !(Dt > 0) || n_intervals < 1) return fail(CQG_E_INVALID, "cqg_master_run: Dt > 0 and n_intervals >= 1");
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    const int cols = m->sys->L.nAvr + 1;
    std::vector<double> row(cols);
    try {
      for (int k = 0; k < n_intervals; ++k) {
        const double endTime = m->t + Dt;
        double dt;
        while ((dt = endTime - m->t) != 0.) step(*m, dt);
        if (avr_out) {
          averages(*m, row.data());
          std::copy(row.begin(), row.end(), avr_out + size_t(k) * cols);
        }
      }
    } catch (const CudaError&) {
      throw;
    } catch (const std::runtime_error& e) {
      return fail(CQG_E_STALLED, e.what());
    }
    return CQG_OK;
  });
}

int cqg_master_steps(cqg_master* m, int32_t n_steps, double T, double* avr_out) {
  return guardedCuda([&] {
    if (!m || n_steps < 0) return fail(CQG_E_INVALID, "cqg_master_steps: n_steps >= 0 required");
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    try {
      for (int k = 0; k < n_steps && m->t < T; ++k) step(*m, T - m->t);
    } catch (const CudaError&) {
      throw;
    } catch (const std::runtime_error& e) {
      return fail(CQG_E_STALLED, e.what());
    }
    if (avr_out) averages(*m, avr_out);
    return CQG_OK;
  });
}

int cqg_master_averages(cqg_master* m, double* avr_out) {
  return guardedCuda([&] {
    if (!m || !avr_out) return fail(CQG_E_INVALID, "cqg_master_averages: null argument");
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    averages(*m, avr_out);
    return CQG_OK;
  });
}

int cqg_master_get_rho(const cqg_master* m, cqg_complex* rho) {
  return guardedCuda([&] {
    if (!m || !rho) return fail(CQG_E_INVALID, "cqg_master_get_rho: null argument");
    const int64_t D = m->D;
    std::vector<double2> r(size_t(D) * D);
    ck(cudaMemcpy(r.data(), m->rho, r.size() * sizeof(double2), cudaMemcpyDeviceToHost), "cudaMemcpy(rho)");
    for (int64_t i = 0; i < D; ++i)
      for (int64_t j = 0; j < D; ++j) rho[size_t(i) * D + j] = {r[size_t(j) * D + i].x, r[size_t(j) * D + i].y};
    return CQG_OK;
  });
}

int cqg_master_get_times(const cqg_master* m, double* t, double* dt_did, double* dt_try) {
  if (!m) return fail(CQG_E_INVALID, "cqg_master_get_times: null master");
  if (t) *t = m->t;
  if (dt_did) *dt_did = m->dtDid;
  if (dt_try) *dt_try = m->dtTry;
  return CQG_OK;
}

int cqg_master_destroy(cqg_master* m) {
  delete m;
  return CQG_OK;
}

}  // extern "C"
