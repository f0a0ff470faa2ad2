// Instantiations of normalize_kernel (float64 cells and bracket arithmetic).
#include "dispatch.h"
#include "sigk_kernels.cuh"

namespace sigk {
namespace {
template <typename TIN, int R, bool FI>
NormFn by_o(int O)
{
    switch (O) {
    case 0: return normalize_kernel<TIN, R, 0, FI>;
    case 1: return normalize_kernel<TIN, R, 1, FI>;
    case 2: return normalize_kernel<TIN, R, 2, FI>;
    case 3: return normalize_kernel<TIN, R, 3, FI>;
    default: return normalize_kernel<TIN, R, 4, FI>;
    }
}
template <typename TIN, bool FI>
NormFn by_r(int R, int O)
{
    switch (R) {
    case 2: return by_o<TIN, 2, FI>(O);
    case 4: return by_o<TIN, 4, FI>(O);
    case 8: return by_o<TIN, 8, FI>(O);
    default: return by_o<TIN, 16, FI>(O);
    }
}
} // namespace

NormFn get_norm_kernel(bool in64, bool from_inc, int R, int O)
{
    if (in64) return from_inc ? by_r<double, true>(R, O) : by_r<double, false>(R, O);
    return from_inc ? by_r<float, true>(R, O) : by_r<float, false>(R, O);
}
} // namespace sigk
