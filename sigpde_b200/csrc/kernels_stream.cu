// Instantiations of stream_smem_kernel and delta_kernel.
#include "dispatch.h"
#include "stream.cuh"

namespace sigk {
namespace {
template <typename T, int R>
StreamFn by_o(int O)
{
    switch (O) {
    case 0: return stream_smem_kernel<T, R, 0>;
    case 1: return stream_smem_kernel<T, R, 1>;
    case 2: return stream_smem_kernel<T, R, 2>;
    case 3: return stream_smem_kernel<T, R, 3>;
    default: return stream_smem_kernel<T, R, 4>;
    }
}
template <typename T>
StreamFn by_r(int R, int O)
{
    switch (R) {
    case 2: return by_o<T, 2>(O);
    case 4: return by_o<T, 4>(O);
    case 8: return by_o<T, 8>(O);
    default: return by_o<T, 16>(O);
    }
}
} // namespace

StreamFn get_stream_smem_kernel(bool f64cells, int R, int O)
{
    return f64cells ? by_r<double>(R, O) : by_r<float>(R, O);
}

StreamFn get_stream_reg_kernel(bool f64cells, int R, int O, int D)
{
    return f64cells ? get_stream_reg_kernel_f64(R, O, D) : get_stream_reg_kernel_f32(R, O, D);
}

DeltaFn get_delta_kernel(bool f64cells, bool in64)
{
    if (f64cells) return in64 ? delta_kernel<double, double> : delta_kernel<double, float>;
    return in64 ? delta_kernel<float, double> : delta_kernel<float, float>;
}
} // namespace sigk
