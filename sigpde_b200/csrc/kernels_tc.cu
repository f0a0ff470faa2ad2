// Instantiations of the tensor-core increment kernels (tc.cuh).
#include "dispatch.h"
#include "dgemm_inc.cuh"
#include "static_inc.cuh"
#include "tc.cuh"

namespace sigk {
namespace {
template <typename T, int R, typename TM, int W>
StreamIncFn inc_by_o(int O)
{
    switch (O) {
    case 0: return stream_inc_kernel<T, R, 0, TM, W>;
    case 1: return stream_inc_kernel<T, R, 1, TM, W>;
    case 2: return stream_inc_kernel<T, R, 2, TM, W>;
    case 3: return stream_inc_kernel<T, R, 3, TM, W>;
    default: return stream_inc_kernel<T, R, 4, TM, W>;
    }
}
template <typename T, typename TM>
StreamIncFn inc_by_r(int R, int O, int W)
{
    if (W == 16) { // half-warp pipelines: pairs of at most 16 R rows, R <= 8
        switch (R) {
        case 2: return inc_by_o<T, 2, TM, 16>(O);
        case 4: return inc_by_o<T, 4, TM, 16>(O);
        default: return inc_by_o<T, 8, TM, 16>(O);
        }
    }
    switch (R) {
    case 2: return inc_by_o<T, 2, TM, 32>(O);
    case 4: return inc_by_o<T, 4, TM, 32>(O);
    case 8: return inc_by_o<T, 8, TM, 32>(O);
    default: return inc_by_o<T, 16, TM, 32>(O);
    }
}
} // namespace

StreamIncFn get_stream_inc_kernel(bool f64cells, int R, int O, bool mat64, int W)
{
    if (mat64) return inc_by_r<double, double>(R, O, W);
    return f64cells ? inc_by_r<double, float>(R, O, W) : inc_by_r<float, float>(R, O, W);
}

TcImageFn get_tc_image_kernel(bool in64) { return in64 ? tc_image_kernel<double> : tc_image_kernel<float>; }

TcGemmFn get_tc_gemm_kernel(int bn) { return bn == 128 ? tc_gemm_kernel<128> : tc_gemm_kernel<kTcBN>; }

DgemmIncFn get_dgemm_inc_kernel() { return dgemm_inc_kernel<kDgTile>; }

DgemmIncFn get_dgemm_inc_pipe_kernel(int64_t d)
{
    if (d <= 16) return dgemm_inc_pipe_kernel<16>;
    if (d <= 32) return dgemm_inc_pipe_kernel<32>;
    return nullptr;
}

size_t dgemm_inc_pipe_smem(int64_t d) { return dgemm_pipe_smem_bytes(d <= 16 ? 16 : 32); }

RaggedImage64Fn get_ragged_image64_kernel(bool in64)
{
    return in64 ? ragged_image64_kernel<double> : ragged_image64_kernel<float>;
}

RaggedDgemmFn get_ragged_dgemm_kernel() { return ragged_dgemm_kernel<kDgTile>; }

RaggedDgemmFn get_ragged_dgemm_pipe_kernel(int64_t d)
{
    if (d <= 16) return ragged_dgemm_pipe_kernel<16>;
    if (d <= 32) return ragged_dgemm_pipe_kernel<32>;
    return nullptr;
}

namespace {
template <int KIND, typename TO>
StaticIncFn static_by_dim(int64_t d)
{
    if (d <= 2) return static_inc_kernel<KIND, 2, TO>;
    if (d <= 4) return static_inc_kernel<KIND, 4, TO>;
    if (d <= 8) return static_inc_kernel<KIND, 8, TO>;
    if (d <= 16) return static_inc_kernel<KIND, 16, TO>;
    if (d <= 32) return static_inc_kernel<KIND, 32, TO>;
    return nullptr;
}
} // namespace

StaticIncFn get_static_inc_kernel(int kind, int64_t dim, bool out64)
{
    if (kind == kStaticRbf)
        return out64 ? static_by_dim<kStaticRbf, double>(dim) : static_by_dim<kStaticRbf, float>(dim);
    if (kind == kStaticL1Rbf)
        return out64 ? static_by_dim<kStaticL1Rbf, double>(dim) : static_by_dim<kStaticL1Rbf, float>(dim);
    return nullptr;
}

TcRaggedImageFn get_tc_ragged_image_kernel(bool in64)
{
    return in64 ? tc_ragged_image_kernel<double> : tc_ragged_image_kernel<float>;
}

} // namespace sigk
