// Per-trajectory random streams on the device.
//
// PCG64 (O'Neill, "PCG: A Family of Simple Fast Space-Efficient Statistically Good
// Algorithms for Random Number Generation", 2014): 128-bit LCG with multiplier
// 0x2360ED051FC65DA44385DF649FCCF645, increment (stream << 1) | 1, state seeded as
// (seed + inc) * mult + inc, XSL-RR output of the advanced state.  This is the
// reference's pcg64{seed, stream} (Random.h:116-126, MCWF_Trajectory.h:208), so with
// it a device trajectory draws the same numbers as the reference trajectory.
//
// The uniform double is libstdc++'s generate_canonical<double,53> for a 64-bit
// engine: double(x) / 2^64 rounded to nearest, mapped below 1 when it rounds up
// (std::uniform_real_distribution<double>, MCWF_Trajectory.h:161,191).
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11): counter-based; key = seed, counter = (draw index, trajectory).
#pragma once

#include <cstdint>

namespace cqg {
namespace dev {

struct U128 {
  uint64_t hi, lo;
};

__host__ __device__ inline U128 add128(U128 a, U128 b) {
  U128 r;
  r.lo = a.lo + b.lo;
  r.hi = a.hi + b.hi + (r.lo < a.lo ? 1u : 0u);
  return r;
}

__host__ __device__ inline U128 mul128(U128 a, U128 b) {
  U128 r;
#ifdef __CUDA_ARCH__
  r.lo = a.lo * b.lo;
  r.hi = __umul64hi(a.lo, b.lo) + a.hi * b.lo + a.lo * b.hi;
#else
  unsigned __int128 p = (unsigned __int128)a.lo * b.lo;
  r.lo = (uint64_t)p;
  r.hi = (uint64_t)(p >> 64) + a.hi * b.lo + a.lo * b.hi;
#endif
  return r;
}

constexpr uint64_t PCG_MULT_HI = 0x2360ED051FC65DA4ull;
constexpr uint64_t PCG_MULT_LO = 0x4385DF649FCCF645ull;

struct Pcg64 {
  U128 state, inc;

  __host__ __device__ static Pcg64 seeded(uint64_t seed, uint64_t stream) {
    Pcg64 g;
    g.inc.lo = (stream << 1) | 1u;
    g.inc.hi = stream >> 63;
    U128 s = add128(U128{0, seed}, g.inc);
    g.state = add128(mul128(s, U128{PCG_MULT_HI, PCG_MULT_LO}), g.inc);
    return g;
  }

  __host__ __device__ uint64_t next() {
    state = add128(mul128(state, U128{PCG_MULT_HI, PCG_MULT_LO}), inc);
    const unsigned rot = unsigned(state.hi >> 58);
    const uint64_t x = state.hi ^ state.lo;
    return rot ? (x >> rot) | (x << (64 - rot)) : x;
  }
};

__device__ inline double canonicalFromU64(uint64_t x) {
  double u = __ull2double_rn(x) * 0x1p-64;
  if (u >= 1.0) u = 0x1.fffffffffffffp-1;  // nextafter(1, 0)
  return u;
}

// Philox4x32-10
__device__ inline void philox4x32_10(uint32_t ctr[4], uint32_t key[2]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, ctr[0]), lo0 = M0 * ctr[0];
    const uint32_t hi1 = __umulhi(M1, ctr[2]), lo1 = M1 * ctr[2];
    const uint32_t c0 = hi1 ^ ctr[1] ^ key[0];
    const uint32_t c1 = lo1;
    const uint32_t c2 = hi0 ^ ctr[3] ^ key[1];
    const uint32_t c3 = lo0;
    ctr[0] = c0;
    ctr[1] = c1;
    ctr[2] = c2;
    ctr[3] = c3;
    key[0] += W0;
    key[1] += W1;
  }
}

__device__ inline double philoxUniform(uint64_t seed, uint64_t traj, uint64_t draw) {
  uint32_t ctr[4] = {uint32_t(draw), uint32_t(draw >> 32), uint32_t(traj), uint32_t(traj >> 32)};
  uint32_t key[2] = {uint32_t(seed), uint32_t(seed >> 32)};
  philox4x32_10(ctr, key);
  const uint64_t bits = (uint64_t(ctr[0]) << 32) | ctr[1];
  return double(bits >> 11) * 0x1p-53;  // [0, 1)
}

}  // namespace dev
}  // namespace cqg
