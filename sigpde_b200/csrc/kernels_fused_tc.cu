// Instantiations of the fused tensor-core Gram kernel (fused_tc.cuh): rows per
// lane R and dyadic order O with R >= 2^O and at most 4 coarse rows a lane.
#include "dispatch.h"
#include "fused_tc.cuh"

namespace sigk {

FusedTcFn get_fused_tc_kernel(int R, int O)
{
    switch (O) {
    case 0:
        if (R == 2) return fused_tc_kernel<2, 0>;
        if (R == 4) return fused_tc_kernel<4, 0>;
        return nullptr;
    case 1:
        if (R == 2) return fused_tc_kernel<2, 1>;
        if (R == 4) return fused_tc_kernel<4, 1>;
        if (R == 8) return fused_tc_kernel<8, 1>;
        return nullptr;
    case 2:
        if (R == 4) return fused_tc_kernel<4, 2>;
        if (R == 8) return fused_tc_kernel<8, 2>;
        if (R == 16) return fused_tc_kernel<16, 2>;
        return nullptr;
    case 3:
        if (R == 8) return fused_tc_kernel<8, 3>;
        if (R == 16) return fused_tc_kernel<16, 3>;
        return nullptr;
    default:
        return nullptr;
    }
}

} // namespace sigk
