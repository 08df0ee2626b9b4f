// Column (y-direction) kernel instantiations for double.
#include "lines_dispatch.cuh"
namespace obl {
template cudaError_t launch_cols<double>(int, bool, int, const ColArgs<double> &, cudaStream_t);
}
