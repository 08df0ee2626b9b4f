// ensemble_part_rows.cu -- instantiations of the persistent ensemble kernel (ensemble_kernel.cuh).
#include "ensemble_kernel.cuh"

namespace obl {
template struct EnsKernel<float, 0, 1, 2>;
template struct EnsKernel<double, 0, 1, 2>;
template struct EnsKernel<float, 4, 6, 2>;
template struct EnsKernel<double, 4, 6, 2>;
} // namespace obl
