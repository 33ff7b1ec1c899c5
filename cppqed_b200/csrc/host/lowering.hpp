// Lowering of a cqg_system_desc to row-gather (ELL) tables for the device.
//
// The reference applies each Tridiagonal term slice by slice
// (Tridiagonal.tcc:220-263, BinarySystem.cc:194-207, Composite.tcc:178-197): for every
// retained-axis diagonal, dpsi(out range) += d(box) * psi(in range).  On the device
// every thread owns output rows, so the same operator is stored per output row:
// a fused main diagonal (all time-independent main-diagonal contributions summed in
// term order) plus `S` off-diagonal slots (input row, coefficient, interaction-picture
// frequency) in the reference's term / diagonal order.  Padding slots point at the row
// itself with a zero coefficient, so the kernels never branch on them.
#pragma once

#include <complex>
#include <cstdint>
#include <vector>

#include "cqg.h"

namespace cqg {

struct EllOperator {
  int64_t D = 0;
  int S = 0;                           // slots per row
  std::vector<std::complex<double>> diag;  // [D] (only for Hamiltonians; empty otherwise)
  std::vector<int32_t> col;            // [S][D]
  std::vector<std::complex<double>> val;   // [S][D]
  std::vector<std::complex<double>> freq;  // [S][D] or empty when time-independent
};

// The Hamiltonian's off-diagonal terms in the per-axis form of the reference's Tridiagonal
// (Tridiagonal.tcc:220-263): every non-empty off-diagonal diagonal of a term of rank 1 or 2
// is a direct product of one vector per retained axis (how the reference builds every
// Tridiagonal of rank > 1, Tridiagonal.tcc:56-64), so a row's coefficient is the product of
// one entry per axis and its frequency the sum.  Built only when every such diagonal
// factorises to rounding (1e-14 relative), the system has at most 3 axes and the slot count
// is small; the main diagonals stay fused into `ham.diag`.
struct FactoredSlot {
  int nAx = 0;         // retained axes: 1 or 2
  int axis[2] = {};    // system axes
  int digit[2] = {};   // 0 main, 1 "minus" (out n+K <- in n), 2 "plus" (out n <- in n+K)
  int64_t K[2] = {};
  int off[2] = {};     // offsets of the per-axis factors in `factors`
  int64_t inShift = 0; // input row minus output row
};
struct FactoredOperator {
  bool ok = false;
  std::vector<FactoredSlot> slots;          // in the reference's term / diagonal order
  std::vector<std::complex<double>> factors;
  std::vector<std::complex<double>> freqs;  // per factor entry, summed over the axes (IP)
  bool anyFreq = false;
};

struct LoweredSystem {
  int rank = 0;
  int64_t dims[CQG_MAX_RANK] = {};
  int64_t D = 0;
  bool hasH = false, hasEx = false, hasLi = false;
  EllOperator ham;                     // H/i with fused diagonal
  FactoredOperator fac;                // the same off-diagonal terms per axis, where they factorise
  std::vector<std::complex<double>> lambda;  // [D] Exact exponent per row (empty: none)
  std::vector<EllOperator> jumps;      // J_m, slots include diagonal entries
  std::vector<std::vector<double>> weights;  // [m][D] closed-form rate weights (empty: ||J psi||^2)
  std::vector<EllOperator> obs;        // observables, slots include diagonal entries
  std::vector<int> obsColRe, obsColIm;
  // Observables that may be evaluated by a fast k -> x transform along one axis (all on the
  // same axis, N = 2^n <= 2048 points, real-valued): their indices, the axis' length and
  // stride, and their weights [nFourier][N].  Empty when none or when the conditions fail.
  std::vector<int> fourierObs;
  int64_t fourierN = 0, fourierStride = 0;
  std::vector<double> fourierW;
  int nAvr = 0;
  double highestFrequency = 0;
};

// Validates the descriptor (ranks, axes, sizes, differences) and builds the tables.
// Throws std::invalid_argument with a message naming the offending field.
LoweredSystem lowerSystem(const cqg_system_desc& d);

}  // namespace cqg
