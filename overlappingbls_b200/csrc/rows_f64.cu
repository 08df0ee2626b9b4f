// Row (x-direction) kernel instantiations for double.
#include "lines_dispatch.cuh"
namespace obl {
template cudaError_t launch_rows<double>(int, int, const RowArgs<double> &, cudaStream_t);
}
