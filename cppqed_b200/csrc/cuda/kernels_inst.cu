// Explicit instantiation of the fused MCWF warp kernel for one (precision, rows per lane,
// picture) triple; the build compiles this file once per triple (-DCQG_REAL, -DCQG_E,
// -DCQG_IP) so the instances compile in parallel.  Exposes
// pick_<real>_e<E>_ip<IP>(SMAX, high occupancy).
#include "mcwf_kernel.cuh"

#ifndef CQG_REAL
#error "CQG_REAL must be defined"
#endif
#ifndef CQG_E
#error "CQG_E must be defined"
#endif
#ifndef CQG_IP
#error "CQG_IP must be defined"
#endif

#define CQG_CAT2(a, b, c, d) a##b##_e##c##_ip##d
#define CQG_CAT(a, b, c, d) CQG_CAT2(a, b, c, d)

namespace cqg {
namespace dev {

using KernelFn = void (*)(TrajDev, RunArgs);

// The instance reads exactly SMAX slots of the padded tables (a system with fewer slots
// reads zero coefficients in the rest): 2 (a driven mode), 3 (Jaynes-Cummings), 4, 8.
// highOccupancy selects the instance compiled for more resident CTAs where there is one.
template <int SMAX, bool IP>
KernelFn pickOccupancy(bool highOccupancy) {
  if constexpr (warpHighOccupancyVariant(CQG_E, SMAX, IP)) {
    if (highOccupancy) return &mcwfWarpKernel<CQG_REAL, CQG_E, SMAX, IP, WarpMinBlocksHigh<CQG_E>::value>;
  }
  return &mcwfWarpKernel<CQG_REAL, CQG_E, SMAX, IP, WarpMinBlocks<CQG_E, IP>::value>;
}

KernelFn CQG_CAT(pick_, CQG_REAL, CQG_E, CQG_IP)(int smax, bool highOccupancy) {
  constexpr bool IP = CQG_IP != 0;
  if (smax <= 2) return pickOccupancy<2, IP>(highOccupancy);
  if (smax <= 3) return pickOccupancy<3, IP>(highOccupancy);
  if (smax <= 4) return pickOccupancy<4, IP>(highOccupancy);
  return pickOccupancy<8, IP>(highOccupancy);
}

}  // namespace dev
}  // namespace cqg
