#include "lowering.hpp"

#include <cmath>
#include <stdexcept>
#include <string>

namespace cqg {

namespace {

using dcomp = std::complex<double>;

struct Entry {
  int64_t in;
  dcomp val, freq;
};

struct Shape {
  int rank;
  int64_t dims[CQG_MAX_RANK];
  int64_t strides[CQG_MAX_RANK];
  int64_t D;
};

Shape shapeOf(const cqg_system_desc& d) {
  Shape s{};
  if (d.rank < 1 || d.rank > CQG_MAX_RANK) throw std::invalid_argument("system rank must be in 1..8");
  s.rank = d.rank;
  s.D = 1;
  for (int a = d.rank - 1; a >= 0; --a) {
    if (d.dims[a] < 1) throw std::invalid_argument("system dimension must be positive");
    s.dims[a] = d.dims[a];
    s.strides[a] = s.D;
    s.D *= d.dims[a];
    if (s.D > (int64_t(1) << 31)) throw std::invalid_argument("total dimension too large");
  }
  return s;
}

// Enumerates every (out, in, coefficient, freq) of a placed tridiagonal in the
// reference's application order: slices, then diagonal index, then box C-order.
template <typename F>
void enumerate(const Shape& s, const cqg_tridiagonal& t, const char* what, F&& f) {
  if (t.rank < 1 || t.rank > s.rank) throw std::invalid_argument(std::string(what) + ": tridiagonal rank out of range");
  if (!t.diagonals) throw std::invalid_argument(std::string(what) + ": diagonals pointer is NULL");
  bool retained[CQG_MAX_RANK] = {};
  for (int a = 0; a < t.rank; ++a) {
    if (t.axes[a] < 0 || t.axes[a] >= s.rank || retained[t.axes[a]])
      throw std::invalid_argument(std::string(what) + ": bad or repeated axis");
    retained[t.axes[a]] = true;
    if (t.differences[a] < 0 || t.differences[a] > s.dims[t.axes[a]])
      throw std::invalid_argument(std::string(what) + ": difference K out of range");
  }
  size_t L = 1;
  for (int a = 0; a < t.rank; ++a) L *= 3;
  // dummy-axis odometer
  int64_t idx[CQG_MAX_RANK] = {};
  while (true) {
    int64_t base = 0;
    for (int a = 0; a < s.rank; ++a) base += idx[a] * s.strides[a];
    for (size_t j = 0; j < L; ++j) {
      const cqg_complex* dj = t.diagonals[j];
      if (!dj) continue;
      int dig[CQG_MAX_RANK];
      size_t rem = j;
      for (int a = t.rank - 1; a >= 0; --a) {
        dig[a] = int(rem % 3);
        rem /= 3;
      }
      int64_t ext[CQG_MAX_RANK], outOff = 0, inOff = 0, boxSize = 1;
      for (int a = 0; a < t.rank; ++a) {
        const int64_t N = s.dims[t.axes[a]], K = t.differences[a];
        if (dig[a] != 0 && K == 0) throw std::invalid_argument(std::string(what) + ": off-diagonal with K = 0");
        ext[a] = dig[a] == 0 ? N : N - K;
        boxSize *= ext[a];
        if (dig[a] == 1) outOff += K * s.strides[t.axes[a]];
        if (dig[a] == 2) inOff += K * s.strides[t.axes[a]];
      }
      const cqg_complex* fj = t.freqs ? t.freqs[j] : nullptr;
      int64_t m[CQG_MAX_RANK] = {};
      for (int64_t c = 0; c < boxSize; ++c) {
        int64_t off = 0;
        for (int a = 0; a < t.rank; ++a) off += m[a] * s.strides[t.axes[a]];
        const dcomp v(dj[c].re, dj[c].im);
        const dcomp fr = fj ? dcomp(fj[c].re, fj[c].im) : dcomp(0, 0);
        if (!std::isfinite(v.real()) || !std::isfinite(v.imag()) || !std::isfinite(fr.real()) ||
            !std::isfinite(fr.imag()))
          throw std::invalid_argument(std::string(what) + ": non-finite coefficient");
        f(base + off + outOff, base + off + inOff, v, fr, j == 0);
        for (int a = t.rank - 1; a >= 0; --a) {
          if (++m[a] < ext[a]) break;
          m[a] = 0;
        }
      }
    }
    int a = s.rank - 1;
    for (; a >= 0; --a) {
      if (retained[a]) continue;
      if (++idx[a] < s.dims[a]) break;
      idx[a] = 0;
    }
    if (a < 0) break;
  }
}

EllOperator toEll(int64_t D, std::vector<std::vector<Entry>>& rows, std::vector<dcomp>* diag, bool anyFreq) {
  EllOperator e;
  e.D = D;
  size_t S = 0;
  for (auto& r : rows) S = std::max(S, r.size());
  e.S = int(S);
  if (diag) e.diag = *diag;
  e.col.assign(S * D, 0);
  e.val.assign(S * D, dcomp(0, 0));
  if (anyFreq) e.freq.assign(S * D, dcomp(0, 0));
  for (int64_t r = 0; r < D; ++r)
    for (size_t s = 0; s < S; ++s) {
      if (s < rows[r].size()) {
        e.col[s * D + r] = int32_t(rows[r][s].in);
        e.val[s * D + r] = rows[r][s].val;
        if (anyFreq) e.freq[s * D + r] = rows[r][s].freq;
      } else {
        e.col[s * D + r] = int32_t(r);  // padding: own row, zero coefficient
      }
    }
  return e;
}

EllOperator lowerGeneric(const Shape& s, const cqg_tridiagonal* terms, int n, const char* what) {
  std::vector<std::vector<Entry>> rows(s.D);
  bool anyFreq = false;
  for (int i = 0; i < n; ++i)
    enumerate(s, terms[i], what, [&](int64_t out, int64_t in, dcomp v, dcomp fr, bool) {
      rows[out].push_back({in, v, fr});
      anyFreq |= fr != dcomp(0, 0);
    });
  return toEll(s.D, rows, nullptr, anyFreq);
}

}  // namespace

LoweredSystem lowerSystem(const cqg_system_desc& d) {
  const Shape s = shapeOf(d);
  LoweredSystem L;
  L.rank = s.rank;
  for (int a = 0; a < s.rank; ++a) L.dims[a] = s.dims[a];
  L.D = s.D;
  L.hasH = d.has_hamiltonian != 0;
  L.highestFrequency = d.highest_frequency;
  if (d.n_ham < 0 || (d.n_ham && !d.ham)) throw std::invalid_argument("ham: bad term list");

  // Hamiltonian: fused diagonal + off-diagonal slots
  {
    std::vector<std::vector<Entry>> rows(s.D);
    std::vector<dcomp> diag(s.D, dcomp(0, 0));
    bool anyFreq = false;
    for (int i = 0; i < d.n_ham; ++i)
      enumerate(s, d.ham[i], "ham", [&](int64_t out, int64_t in, dcomp v, dcomp fr, bool isMain) {
        if (isMain && out == in)
          diag[out] += v;
        else {
          rows[out].push_back({in, v, fr});
          anyFreq |= fr != dcomp(0, 0);
        }
      });
    L.ham = toEll(s.D, rows, &diag, anyFreq);
  }

  // Exact part: lambda[row] = sum_a lambda_a[n_a]
  for (int a = 0; a < s.rank; ++a)
    if (d.exact[a]) L.hasEx = true;
  if (L.hasEx) {
    L.lambda.assign(s.D, dcomp(0, 0));
    for (int64_t r = 0; r < s.D; ++r)
      for (int a = 0; a < s.rank; ++a)
        if (d.exact[a]) {
          const int64_t n = (r / s.strides[a]) % s.dims[a];
          L.lambda[r] += dcomp(d.exact[a][n].re, d.exact[a][n].im);
        }
  }

  if (d.n_jumps < 0 || (d.n_jumps && !d.jumps)) throw std::invalid_argument("jumps: bad list");
  L.hasLi = d.n_jumps > 0;
  for (int m = 0; m < d.n_jumps; ++m) {
    L.jumps.push_back(lowerGeneric(s, &d.jumps[m].op, 1, "jump"));
    std::vector<double> w;
    if (d.jumps[m].rate_weights) {
      const int a = d.jumps[m].rate_axis;
      if (a < 0 || a >= s.rank) throw std::invalid_argument("jump: rate_axis out of range");
      w.resize(s.D);
      for (int64_t r = 0; r < s.D; ++r) {
        w[r] = d.jumps[m].rate_weights[(r / s.strides[a]) % s.dims[a]];
        if (!std::isfinite(w[r])) throw std::invalid_argument("jump: non-finite rate weight");
      }
    }
    L.weights.push_back(std::move(w));
  }

  if (d.n_obs < 0 || (d.n_obs && !d.obs)) throw std::invalid_argument("obs: bad list");
  if (d.n_avr < 0) throw std::invalid_argument("n_avr negative");
  L.nAvr = d.n_avr;
  for (int k = 0; k < d.n_obs; ++k) {
    const auto& o = d.obs[k];
    if (o.col_re >= d.n_avr || o.col_im >= d.n_avr) throw std::invalid_argument("obs: column out of range");
    if (o.dense) {
      const int a = o.dense_axis;
      if (a < 0 || a >= s.rank) throw std::invalid_argument("obs: dense_axis out of range");
      const int64_t N = s.dims[a];
      std::vector<std::vector<Entry>> rows(s.D);
      for (int64_t r = 0; r < s.D; ++r) {
        const int64_t i = (r / s.strides[a]) % s.dims[a];
        const int64_t base = r - i * s.strides[a];
        for (int64_t j = 0; j < N; ++j) {
          const dcomp v(o.dense[i * N + j].re, o.dense[i * N + j].im);
          if (v != dcomp(0, 0)) rows[r].push_back({base + j * s.strides[a], v, 0});
        }
      }
      L.obs.push_back(toEll(s.D, rows, nullptr, false));
    } else {
      L.obs.push_back(lowerGeneric(s, &o.op, 1, "obs"));
    }
    L.obsColRe.push_back(o.col_re);
    L.obsColIm.push_back(o.col_im);
  }
  // fast-transform candidates
  int fAxis = -1;
  bool fOk = true;
  for (int k = 0; k < d.n_obs; ++k) {
    const auto& o = d.obs[k];
    if (!o.fourier) continue;
    if (!o.dense || !o.fourier_weights || o.col_im >= 0 || (fAxis >= 0 && o.dense_axis != fAxis)) {
      fOk = false;
      continue;
    }
    fAxis = o.dense_axis;
    L.fourierObs.push_back(k);
  }
  if (fAxis >= 0) {
    const int64_t N = s.dims[fAxis];
    if (!fOk || N < 2 || N > 2048 || (N & (N - 1)) || L.fourierObs.size() > 4) {
      L.fourierObs.clear();
    } else {
      L.fourierN = N;
      L.fourierStride = s.strides[fAxis];
      for (int k : L.fourierObs)
        for (int64_t m = 0; m < N; ++m) {
          const double w = d.obs[k].fourier_weights[m];
          if (!std::isfinite(w)) throw std::invalid_argument("obs: non-finite fourier weight");
          L.fourierW.push_back(w);
        }
    }
  }
  return L;
}

}  // namespace cqg
