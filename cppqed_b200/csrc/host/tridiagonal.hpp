// Runtime-rank banded operator with the semantics of quantumoperator::Tridiagonal<RANK>
// (quantumoperator/Tridiagonal.h:71-287, Tridiagonal.tcc, Tridiagonal.cc).
//
// The reference fixes RANK at compile time and stores 3^RANK Blitz arrays; here the
// rank is a runtime value because the operator is only a host-side description that
// is lowered once to device tables.  The algebra (direct product, Hermitian
// conjugate, sum, furnishing with interaction-picture frequencies) follows the
// reference rule for rule, because the coefficient values it produces are what the
// device kernels consume.
#pragma once

#include <complex>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <vector>

namespace cqg {

using dcomp = std::complex<double>;
using CVec = std::vector<dcomp>;
using DVec = std::vector<double>;

class Tridiagonal {
 public:
  Tridiagonal() = default;

  // Unary constructor (Tridiagonal.cc:42-62): zero = main diagonal, k = K,
  // minus = alpha^(-) on |n+K><n|, plus = alpha^(+) on |n><n+K|.  With toFreqs the
  // main diagonal is turned into frequencies (furnishWithFreqs(-zero)).
  static Tridiagonal unary(const CVec& zero, size_t k = 0, const CVec& minus = {}, const CVec& plus = {},
                           bool toFreqs = false);

  // quantumoperator::identity (Tridiagonal.cc:66-71)
  static Tridiagonal identity(size_t dim);

  int rank() const { return int(dims_.size()); }
  const std::vector<size_t>& dims() const { return dims_; }
  const std::vector<size_t>& differences() const { return k_; }
  const std::vector<CVec>& diagonals() const { return diagonals_; }
  const std::vector<CVec>& freqs() const { return freqs_; }
  std::vector<CVec>& diagonalsMutable() { return diagonals_; }
  size_t length() const { return diagonals_.size(); }
  bool empty() const;
  bool hasFreqs() const;

  // extent of the box of diagonal `index` along axis `a`
  size_t boxExtent(size_t index, int a) const;
  size_t boxSize(size_t index) const;
  int digit(size_t index, int a) const;

  // Tridiagonal<1>::furnishWithFreqs (Tridiagonal.cc:24-36): freqs(1)(n) = main(n+k) - main(n),
  // freqs(2) = -freqs(1).  Unary only, as in the reference.
  Tridiagonal& furnishWithFreqs(const CVec& mainDiagonal);

  // hermitianConjugate (Tridiagonal.tcc:84-115): digit d -> (3-d)%3, values conjugated,
  // frequencies left in place.
  Tridiagonal dagger() const;

  Tridiagonal& operator+=(const Tridiagonal& other);  // Tridiagonal.tcc:118-148
  Tridiagonal& operator-=(const Tridiagonal& other) { return *this += -other; }
  Tridiagonal operator-() const;                      // negated diagonals, freqs untouched
  Tridiagonal& operator*=(dcomp c);                   // Tridiagonal.tcc:73-79
  Tridiagonal& operator/=(dcomp c) { return *this *= (1. / c); }

  // Direct product t1 (x) t2 (Tridiagonal.tcc:28-70): diagonals multiply, frequencies add.
  static Tridiagonal direct(const Tridiagonal& t1, const Tridiagonal& t2);

 private:
  std::vector<size_t> dims_, k_;
  std::vector<CVec> diagonals_, freqs_;  // 3^rank entries each, empty vector = empty diagonal
};

inline Tridiagonal operator+(Tridiagonal a, const Tridiagonal& b) { return a += b; }
inline Tridiagonal operator-(Tridiagonal a, const Tridiagonal& b) { return a -= b; }
inline Tridiagonal operator*(Tridiagonal a, dcomp c) { return a *= c; }
inline Tridiagonal operator*(dcomp c, Tridiagonal a) { return a *= c; }
inline Tridiagonal operator*(Tridiagonal a, double c) { return a *= dcomp(c, 0.); }
inline Tridiagonal operator*(double c, Tridiagonal a) { return a *= dcomp(c, 0.); }
inline Tridiagonal operator/(Tridiagonal a, dcomp c) { return a /= c; }
inline Tridiagonal operator/(Tridiagonal a, double c) { return a /= dcomp(c, 0.); }
// operator* between two tridiagonals is the direct product, as in the reference (Tridiagonal.h:319-324)
inline Tridiagonal operator*(const Tridiagonal& a, const Tridiagonal& b) { return Tridiagonal::direct(a, b); }

inline Tridiagonal tridiagMinusHC(const Tridiagonal& t) { return t - t.dagger(); }  // Tridiagonal.h:333
inline Tridiagonal tridiagPlusHC(const Tridiagonal& t) { return t + t.dagger(); }   // Tridiagonal.h:340

}  // namespace cqg
