// Row (x-direction) kernel instantiations for float.
#include "lines_dispatch.cuh"
namespace obl {
template cudaError_t launch_rows<float>(int, int, const RowArgs<float> &, cudaStream_t);
}
