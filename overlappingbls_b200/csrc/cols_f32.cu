// Column (y-direction) kernel instantiations for float.
#include "lines_dispatch.cuh"
namespace obl {
template cudaError_t launch_cols<float>(int, bool, int, const ColArgs<float> &, cudaStream_t);
}
