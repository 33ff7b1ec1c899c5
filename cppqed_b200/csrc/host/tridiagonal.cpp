#include "tridiagonal.hpp"

#include <algorithm>

namespace cqg {

namespace {

size_t pow3(int r) {
  size_t res = 1;
  for (int i = 0; i < r; ++i) res *= 3;
  return res;
}

bool compatible(const CVec& a, size_t diffA, const CVec& b, size_t diffB = 0) {
  if (a.empty() || b.empty() || a.size() - diffA == b.size() - diffB) return true;
  return false;
}

}  // namespace

bool Tridiagonal::empty() const {
  for (auto& d : diagonals_)
    if (!d.empty()) return false;
  return true;
}

bool Tridiagonal::hasFreqs() const {
  for (auto& f : freqs_)
    if (!f.empty()) return true;
  return false;
}

int Tridiagonal::digit(size_t index, int a) const {
  const int r = rank();
  size_t p = pow3(r - 1 - a);
  return int((index / p) % 3);
}

size_t Tridiagonal::boxExtent(size_t index, int a) const {
  return digit(index, a) == 0 ? dims_[a] : dims_[a] - k_[a];
}

size_t Tridiagonal::boxSize(size_t index) const {
  size_t s = 1;
  for (int a = 0; a < rank(); ++a) s *= boxExtent(index, a);
  return s;
}

Tridiagonal Tridiagonal::unary(const CVec& zero, size_t k, const CVec& minus, const CVec& plus, bool toFreqs) {
  Tridiagonal res;
  size_t dim = std::max(std::max(zero.size(), minus.size() + k), plus.size() + k);
  res.dims_ = {dim};
  res.k_ = {k};
  res.diagonals_ = {toFreqs ? CVec{} : zero, minus, plus};
  res.freqs_ = {CVec{}, CVec{}, CVec{}};
  if (toFreqs) {
    CVec negZero(zero.size());
    for (size_t i = 0; i < zero.size(); ++i) negZero[i] = -zero[i];
    res.furnishWithFreqs(negZero);
  }
  if (!compatible(zero, k, minus) || !compatible(zero, k, plus) || !compatible(minus, 0, plus, 0) ||
      ((minus.size() || plus.size()) && !k))
    throw std::invalid_argument("Tridiagonal consistency error");
  return res;
}

Tridiagonal Tridiagonal::identity(size_t dim) { return unary(CVec(dim, dcomp(1., 0.))); }

Tridiagonal& Tridiagonal::furnishWithFreqs(const CVec& mainDiagonal) {
  if (rank() != 1) throw std::invalid_argument("furnishWithFreqs works in the unary case only");
  const size_t k = k_[0];
  const long diagonalSize = long(dims_[0]) - long(k);
  if (diagonalSize > 0) {
    freqs_[1].assign(size_t(diagonalSize), dcomp());
    for (long n = 0; n < diagonalSize; ++n) freqs_[1][n] = mainDiagonal[n + k] - mainDiagonal[n];
    freqs_[2].resize(size_t(diagonalSize));
    for (long n = 0; n < diagonalSize; ++n) freqs_[2][n] = -freqs_[1][n];
  }
  return *this;
}

Tridiagonal Tridiagonal::dagger() const {
  Tridiagonal res;
  res.dims_ = dims_;
  res.k_ = k_;
  res.freqs_ = freqs_;
  res.diagonals_.assign(diagonals_.size(), CVec{});
  const int r = rank();
  for (size_t ind = 0; ind < diagonals_.size(); ++ind) {
    size_t t = 0;
    for (int a = 0; a < r; ++a) t = t * 3 + size_t((3 - digit(ind, a)) % 3);
    // the transposed diagonal keeps the same box (minus <-> plus have equal extents); the
    // multi-index inside the box is unchanged, as Blitz references the same array layout
    CVec c(diagonals_[ind].size());
    for (size_t i = 0; i < c.size(); ++i) c[i] = std::conj(diagonals_[ind][i]);
    res.diagonals_[t] = std::move(c);
  }
  return res;
}

Tridiagonal& Tridiagonal::operator+=(const Tridiagonal& other) {
  if (dims_.empty()) {  // default-constructed: adopt the structure of `other`
    *this = other;
    return *this;
  }
  if (other.dims_.empty()) return *this;
  if (other.rank() != rank()) throw std::invalid_argument("Tridiagonal rank mismatch");
  for (int a = 0; a < rank(); ++a) {
    if (other.dims_[a] != dims_[a]) throw std::invalid_argument("Tridiagonal dimension mismatch");
    if (!k_[a])
      k_[a] = other.k_[a];
    else if (other.k_[a] && k_[a] != other.k_[a])
      throw std::invalid_argument("Tridiagonal structure mismatch is binOp1");
  }
  for (size_t i = 0; i < diagonals_.size(); ++i) {
    const CVec& from = other.diagonals_[i];
    CVec& to = diagonals_[i];
    if (!from.empty()) {
      if (to.empty())
        to = from;
      else {
        if (to.size() != from.size()) throw std::invalid_argument("Tridiagonal diagonal shape mismatch");
        for (size_t n = 0; n < to.size(); ++n) to[n] += from[n];
      }
    }
  }
  for (size_t i = 0; i < freqs_.size(); ++i) {
    const CVec& from = other.freqs_[i];
    CVec& to = freqs_[i];
    if (!from.empty()) {
      if (!to.empty()) {
        bool allDiffer = to.size() == from.size();
        for (size_t n = 0; allDiffer && n < to.size(); ++n) allDiffer = to[n] != from[n];
        if (allDiffer) throw std::runtime_error("Tridiagonal structure mismatch is operator+=");
      }
      to = from;
    }
  }
  return *this;
}

Tridiagonal Tridiagonal::operator-() const {
  Tridiagonal res(*this);
  for (auto& d : res.diagonals_)
    for (auto& v : d) v = -v;
  return res;
}

Tridiagonal& Tridiagonal::operator*=(dcomp c) {
  for (auto& d : diagonals_)
    for (auto& v : d) v *= c;
  return *this;
}

Tridiagonal Tridiagonal::direct(const Tridiagonal& t1, const Tridiagonal& t2) {
  Tridiagonal res;
  res.dims_ = t1.dims_;
  res.dims_.insert(res.dims_.end(), t2.dims_.begin(), t2.dims_.end());
  res.k_ = t1.k_;
  res.k_.insert(res.k_.end(), t2.k_.begin(), t2.k_.end());
  const size_t L1 = t1.diagonals_.size(), L2 = t2.diagonals_.size();
  res.diagonals_.assign(L1 * L2, CVec{});
  res.freqs_.assign(L1 * L2, CVec{});
  for (size_t i = 0; i < L1; ++i)
    for (size_t j = 0; j < L2; ++j) {
      const CVec &d1 = t1.diagonals_[i], &d2 = t2.diagonals_[j];
      if (!d1.empty() && !d2.empty()) {
        CVec d(d1.size() * d2.size());
        for (size_t a = 0; a < d1.size(); ++a)
          for (size_t b = 0; b < d2.size(); ++b) d[a * d2.size() + b] = d1[a] * d2[b];
        res.diagonals_[i * L2 + j] = std::move(d);
      }
      const CVec &f1 = t1.freqs_[i], &f2 = t2.freqs_[j];
      if (!f1.empty() && !f2.empty()) {
        CVec f(f1.size() * f2.size());
        for (size_t a = 0; a < f1.size(); ++a)
          for (size_t b = 0; b < f2.size(); ++b) f[a * f2.size() + b] = f1[a] + f2[b];
        res.freqs_[i * L2 + j] = std::move(f);
      }
    }
  return res;
}

}  // namespace cqg
