// Instantiations of ragged_kernel.
#include "dispatch.h"
#include "ragged.cuh"

namespace sigk {
RaggedFn get_ragged_kernel(bool f64cells, bool in64)
{
    if (f64cells) return in64 ? ragged_kernel<double, double> : ragged_kernel<double, float>;
    return in64 ? ragged_kernel<float, double> : ragged_kernel<float, float>;
}
RaggedDeltaFn get_ragged_delta_kernel(bool f64cells, bool in64)
{
    if (f64cells) return in64 ? ragged_delta_kernel<double, double> : ragged_delta_kernel<double, float>;
    return in64 ? ragged_delta_kernel<float, double> : ragged_delta_kernel<float, float>;
}
} // namespace sigk
