// dmf_kernel_t4.cu -- instantiations of the solve kernel for tile width 4.
#include "dmf_kernel.cuh"

namespace dmfk {

KernelFn solve_kernel_t4(int minb) {
  return minb == 1 ? k_solve<4, kBlock, 1> : k_solve<4, kBlock, 2>;
}

}  // namespace dmfk
