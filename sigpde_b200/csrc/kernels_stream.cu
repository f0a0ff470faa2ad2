// Instantiations of stream_kernel and delta_kernel.
#include "dispatch.h"
#include "stream.cuh"

namespace sigk {
namespace {
template <typename T, typename TIN, int R>
StreamFn by_o(int O)
{
    switch (O) {
    case 0: return stream_kernel<T, TIN, R, 0>;
    case 1: return stream_kernel<T, TIN, R, 1>;
    case 2: return stream_kernel<T, TIN, R, 2>;
    case 3: return stream_kernel<T, TIN, R, 3>;
    default: return stream_kernel<T, TIN, R, 4>;
    }
}
template <typename T, typename TIN>
StreamFn by_r(int R, int O)
{
    switch (R) {
    case 2: return by_o<T, TIN, 2>(O);
    case 4: return by_o<T, TIN, 4>(O);
    case 8: return by_o<T, TIN, 8>(O);
    default: return by_o<T, TIN, 16>(O);
    }
}
} // namespace

StreamFn get_stream_kernel(bool f64cells, bool in64, int R, int O)
{
    if (f64cells) return in64 ? by_r<double, double>(R, O) : by_r<double, float>(R, O);
    return in64 ? by_r<float, double>(R, O) : by_r<float, float>(R, O);
}

DeltaFn get_delta_kernel(bool f64cells, bool in64)
{
    if (f64cells) return in64 ? delta_kernel<double, double> : delta_kernel<double, float>;
    return in64 ? delta_kernel<float, double> : delta_kernel<float, float>;
}
} // namespace sigk
