// Instantiation of the block-per-trajectory MCWF kernel (mcwf_block.cuh) for both precisions.
#include "mcwf_block.cuh"

namespace cqg {
namespace dev {

using BlockKernelFn = void (*)(TrajDev, RunArgs, BlockScratch, int);

BlockKernelFn pick_block(bool fp64) {
  return fp64 ? &mcwfBlockKernel<double> : &mcwfBlockKernel<float>;
}

}  // namespace dev
}  // namespace cqg
