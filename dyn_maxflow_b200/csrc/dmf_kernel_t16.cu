// dmf_kernel_t16.cu -- instantiations of the solve kernel for tile width 16.
#include "dmf_kernel.cuh"

namespace dmfk {

KernelFn solve_kernel_t16(int minb) {
  return minb == 1 ? k_solve<16, kBlock, 1> : k_solve<16, kBlock, 2>;
}

}  // namespace dmfk
