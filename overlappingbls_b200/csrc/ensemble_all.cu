// ensemble_all.cu -- instantiations of the persistent ensemble kernel (ensemble_kernel.cuh).
#include "ensemble_kernel.cuh"

namespace obl {
template struct EnsKernel<float, 0, 6, 2>;
template struct EnsKernel<double, 0, 6, 2>;
} // namespace obl
