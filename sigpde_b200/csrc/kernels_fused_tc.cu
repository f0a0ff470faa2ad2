// Instantiations of the fused tensor-core Gram kernel (fused_tc.cuh): rows per
// lane R and dyadic order O with R >= 2^O and at most 4 coarse rows a lane, and
// a boundary every 16 or 8 steps.
#include "dispatch.h"
#include "fused_tc.cuh"

namespace sigk {
namespace {
template <int RING>
FusedTcFn by_shape(int R, int O)
{
    switch (O) {
    case 0:
        if (R == 2) return fused_tc_kernel<2, 0, RING>;
        if (R == 4) return fused_tc_kernel<4, 0, RING>;
        return nullptr;
    case 1:
        if (R == 2) return fused_tc_kernel<2, 1, RING>;
        if (R == 4) return fused_tc_kernel<4, 1, RING>;
        if (R == 8) return fused_tc_kernel<8, 1, RING>;
        return nullptr;
    case 2:
        if (R == 4) return fused_tc_kernel<4, 2, RING>;
        if (R == 8) return fused_tc_kernel<8, 2, RING>;
        if (R == 16) return fused_tc_kernel<16, 2, RING>;
        return nullptr;
    case 3:
        if (R == 8) return fused_tc_kernel<8, 3, RING>;
        if (R == 16) return fused_tc_kernel<16, 3, RING>;
        return nullptr;
    default:
        return nullptr;
    }
}
} // namespace

FusedTcFn get_fused_tc_kernel(int R, int O, int ring)
{
    if (ring == 16) return by_shape<16>(R, O);
    if (ring == 8) return by_shape<8>(R, O);
    return nullptr;
}

} // namespace sigk
