// Instantiations of ragged_kernel.
#include "dispatch.h"
#include "ragged.cuh"

namespace sigk {
RaggedFn get_ragged_kernel(bool f64cells, bool in64, bool mat, bool mat64)
{
    if (mat && mat64) return in64 ? ragged_kernel<double, double, true, double> : ragged_kernel<double, float, true, double>;
    if (mat) {
        if (f64cells) return in64 ? ragged_kernel<double, double, true> : ragged_kernel<double, float, true>;
        return in64 ? ragged_kernel<float, double, true> : ragged_kernel<float, float, true>;
    }
    if (f64cells) return in64 ? ragged_kernel<double, double, false> : ragged_kernel<double, float, false>;
    return in64 ? ragged_kernel<float, double, false> : ragged_kernel<float, float, false>;
}
RaggedDeltaFn get_ragged_delta_kernel(bool f64cells, bool in64)
{
    if (f64cells) return in64 ? ragged_delta_kernel<double, double> : ragged_delta_kernel<double, float>;
    return in64 ? ragged_delta_kernel<float, double> : ragged_delta_kernel<float, float>;
}
} // namespace sigk
