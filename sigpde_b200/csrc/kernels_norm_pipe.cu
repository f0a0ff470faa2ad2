// Instantiations of normalize_pipe_kernel (one CTA per path, bands as a warp pipeline).
#include "dispatch.h"
#include "norm_pipe.cuh"

namespace sigk {
namespace {
template <typename TIN, int R, int M>
NormFn pipe_by_o(int O)
{
    switch (O) {
    case 0: return normalize_pipe_kernel<TIN, R, 0, M>;
    case 1: return normalize_pipe_kernel<TIN, R, 1, M>;
    case 2: return normalize_pipe_kernel<TIN, R, 2, M>;
    case 3: return normalize_pipe_kernel<TIN, R, 3, M>;
    default: return normalize_pipe_kernel<TIN, R, 4, M>;
    }
}
template <typename TIN, int M>
NormFn pipe_by_r(int R, int O)
{
    switch (R) {
    case 2: return pipe_by_o<TIN, 2, M>(O);
    case 4: return pipe_by_o<TIN, 4, M>(O);
    case 8: return pipe_by_o<TIN, 8, M>(O);
    default: return pipe_by_o<TIN, 16, M>(O);
    }
}
template <typename TIN>
NormFn pipe_by_mode(int mode, int R, int O)
{
    switch (mode) {
    case kNormGiven: return pipe_by_r<TIN, kNormGiven>(R, O);
    case kNormTile: return pipe_by_r<TIN, kNormTile>(R, O);
    default: return pipe_by_r<TIN, kNormDelta>(R, O);
    }
}
} // namespace

NormFn get_norm_pipe_kernel(bool in64, int mode, int R, int O)
{
    return in64 ? pipe_by_mode<double>(mode, R, O) : pipe_by_mode<float>(mode, R, O);
}
} // namespace sigk
