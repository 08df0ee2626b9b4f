// ensemble_part_mid.cu -- instantiations of the persistent ensemble kernel (ensemble_kernel.cuh).
#include "ensemble_kernel.cuh"

namespace obl {
template struct EnsKernel<float, 1, 4, 4>;
template struct EnsKernel<double, 1, 4, 4>;
} // namespace obl
