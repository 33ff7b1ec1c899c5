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

struct LoweredSystem {
  int rank = 0;
  int64_t dims[CQG_MAX_RANK] = {};
  int64_t D = 0;
  bool hasH = false, hasEx = false, hasLi = false;
  EllOperator ham;                     // H/i with fused diagonal
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
