// Explicit instantiation of the fused MCWF warp kernel for one (precision, rows per
// lane) pair; the build compiles this file once per pair (-DCQG_REAL, -DCQG_E) so the
// instances compile in parallel.  Exposes pick_<real>_e<E>(SMAX, interaction picture).
#include "mcwf_kernel.cuh"

#ifndef CQG_REAL
#error "CQG_REAL must be defined"
#endif
#ifndef CQG_E
#error "CQG_E must be defined"
#endif

#define CQG_CAT2(a, b, c) a##b##_e##c
#define CQG_CAT(a, b, c) CQG_CAT2(a, b, c)

namespace cqg {
namespace dev {

using KernelFn = void (*)(TrajDev, RunArgs);

// The instance reads exactly SMAX slots of the padded tables (a system with fewer slots
// reads zero coefficients in the rest): 2 (a driven mode), 3 (Jaynes-Cummings), 4, 8.
KernelFn CQG_CAT(pick_, CQG_REAL, CQG_E)(int smax, bool ip) {
  if (ip) {
    if (smax <= 2) return &mcwfWarpKernel<CQG_REAL, CQG_E, 2, true>;
    if (smax <= 3) return &mcwfWarpKernel<CQG_REAL, CQG_E, 3, true>;
    if (smax <= 4) return &mcwfWarpKernel<CQG_REAL, CQG_E, 4, true>;
    return &mcwfWarpKernel<CQG_REAL, CQG_E, 8, true>;
  }
  if (smax <= 2) return &mcwfWarpKernel<CQG_REAL, CQG_E, 2, false>;
  if (smax <= 3) return &mcwfWarpKernel<CQG_REAL, CQG_E, 3, false>;
  if (smax <= 4) return &mcwfWarpKernel<CQG_REAL, CQG_E, 4, false>;
  return &mcwfWarpKernel<CQG_REAL, CQG_E, 8, false>;
}

}  // namespace dev
}  // namespace cqg
