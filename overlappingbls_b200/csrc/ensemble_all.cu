// ensemble_all.cu -- instantiations of the persistent ensemble kernel (ensemble_kernel.cuh).
#include "ensemble_kernel.cuh"

namespace obl {
template struct EnsKernel<float, 0, 6, OBL_ENS_MINB>;
template struct EnsKernel<double, 0, 6, OBL_ENS_MINB>;
template struct EnsFlowKernel<float, OBL_ENS_MINB>;
template struct EnsFlowKernel<double, OBL_ENS_MINB>;
} // namespace obl
