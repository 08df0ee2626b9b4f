// Row (x-direction) kernel instantiations for float.
#include "lines_dispatch.cuh"
namespace obl {
template cudaError_t launch_rows<float>(int, int, const RowArgs<float> &, cudaStream_t);
std::vector<double> plan_table(int n, int role)
{
    switch (n) {
#define OBL_CASE(N) case N: return plan_table_n<N>(role);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return {};
}
bool line_length_supported(int n)
{
    switch (n) {
#define OBL_CASE(N) case N: return true;
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return false;
}
}
