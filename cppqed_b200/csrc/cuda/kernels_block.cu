// Instantiation of the block-per-trajectory MCWF kernel (mcwf_block.cuh) for both precisions.
#include "mcwf_block.cuh"

namespace cqg {
namespace dev {

using BlockKernelFn = void (*)(TrajDev, RunArgs, BlockScratch, int);

BlockKernelFn pick_block(bool fp64, bool ip) {
  if (ip) return fp64 ? &mcwfBlockKernel<double, true> : &mcwfBlockKernel<float, true>;
  return fp64 ? &mcwfBlockKernel<double, false> : &mcwfBlockKernel<float, false>;
}

}  // namespace dev
}  // namespace cqg
