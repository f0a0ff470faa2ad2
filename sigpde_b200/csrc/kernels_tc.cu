// Instantiations of the tensor-core increment kernels (tc.cuh).
#include "dispatch.h"
#include "tc.cuh"

namespace sigk {
namespace {
template <typename T, int R>
StreamIncFn inc_by_o(int O)
{
    switch (O) {
    case 0: return stream_inc_kernel<T, R, 0>;
    case 1: return stream_inc_kernel<T, R, 1>;
    case 2: return stream_inc_kernel<T, R, 2>;
    case 3: return stream_inc_kernel<T, R, 3>;
    default: return stream_inc_kernel<T, R, 4>;
    }
}
template <typename T>
StreamIncFn inc_by_r(int R, int O)
{
    switch (R) {
    case 2: return inc_by_o<T, 2>(O);
    case 4: return inc_by_o<T, 4>(O);
    case 8: return inc_by_o<T, 8>(O);
    default: return inc_by_o<T, 16>(O);
    }
}
} // namespace

StreamIncFn get_stream_inc_kernel(bool f64cells, int R, int O)
{
    return f64cells ? inc_by_r<double>(R, O) : inc_by_r<float>(R, O);
}

TcImageFn get_tc_image_kernel(bool in64) { return in64 ? tc_image_kernel<double> : tc_image_kernel<float>; }

TcGemmFn get_tc_gemm_kernel() { return tc_gemm_kernel<kTcBN>; }

TcRaggedImageFn get_tc_ragged_image_kernel(bool in64)
{
    return in64 ? tc_ragged_image_kernel<double> : tc_ragged_image_kernel<float>;
}

} // namespace sigk
