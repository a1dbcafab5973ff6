// dmf_kernel_t32.cu -- instantiations of the solve kernel for tile width 32.
#include "dmf_kernel.cuh"

namespace dmfk {

KernelFn solve_kernel_t32(int minb) {
  return minb == 1 ? k_solve<32, kBlock, 1> : k_solve<32, kBlock, 2>;
}

}  // namespace dmfk
