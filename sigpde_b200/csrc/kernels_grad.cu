// Instantiations of the backward-pass kernels (grad.cuh).
#include "dispatch.h"
#include "grad.cuh"

namespace sigk {
namespace {
template <int R>
GradFns grad_by_o(int O)
{
    GradFns f{};
    switch (O) {
    case 0: f = {grad_fwd_kernel<R, 0>, grad_bwd_kernel<R, 0>}; break;
    case 1: if constexpr (R >= 2) f = {grad_fwd_kernel<R, 1>, grad_bwd_kernel<R, 1>}; break;
    case 2: if constexpr (R >= 4) f = {grad_fwd_kernel<R, 2>, grad_bwd_kernel<R, 2>}; break;
    case 3: if constexpr (R >= 8) f = {grad_fwd_kernel<R, 3>, grad_bwd_kernel<R, 3>}; break;
    case 4: if constexpr (R >= 16) f = {grad_fwd_kernel<R, 4>, grad_bwd_kernel<R, 4>}; break;
    default: break;
    }
    return f;
}
} // namespace

GradFns get_grad_kernels(int R, int O)
{
    switch (R) {
    case 1: return grad_by_o<1>(O);
    case 2: return grad_by_o<2>(O);
    case 4: return grad_by_o<4>(O);
    case 8: return grad_by_o<8>(O);
    case 16: return grad_by_o<16>(O);
    default: return GradFns{};
    }
}

GradAuxFns get_grad_aux_kernels()
{
    return {grad_pair_inc_kernel<>, grad_gx_kernel<>, grad_gy_kernel<>, grad_reduce_kernel<>, grad_points_kernel<>,
            grad_rows_kernel<>, grad_gy_gram_kernel<>, grad_inc_blocks_kernel<>};
}

} // namespace sigk
