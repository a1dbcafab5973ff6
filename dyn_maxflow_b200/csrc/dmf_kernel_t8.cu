// dmf_kernel_t8.cu -- instantiations of the solve kernel for tile width 8.
#include "dmf_kernel.cuh"

namespace dmfk {

KernelFn solve_kernel_t8(int minb) {
  return minb == 1 ? k_solve<8, kBlock, 1> : k_solve<8, kBlock, 2>;
}

}  // namespace dmfk
