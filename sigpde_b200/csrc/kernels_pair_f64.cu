// Instantiations of pair_kernel with float64 cells (SIGK_PREC_FP64).
#include "dispatch.h"
#include "sigk_kernels.cuh"

namespace sigk {
namespace {
template <typename TIN, int R, bool FI>
PairFn by_o(int O)
{
    switch (O) {
    case 0: return pair_kernel<double, TIN, R, 0, FI>;
    case 1: return pair_kernel<double, TIN, R, 1, FI>;
    case 2: return pair_kernel<double, TIN, R, 2, FI>;
    case 3: return pair_kernel<double, TIN, R, 3, FI>;
    default: return pair_kernel<double, TIN, R, 4, FI>;
    }
}
template <typename TIN, bool FI>
PairFn by_r(int R, int O)
{
    switch (R) {
    case 2: return by_o<TIN, 2, FI>(O);
    case 4: return by_o<TIN, 4, FI>(O);
    case 8: return by_o<TIN, 8, FI>(O);
    default: return by_o<TIN, 16, FI>(O);
    }
}
} // namespace

PairFn get_pair_kernel_f64(bool in64, bool from_inc, int R, int O)
{
    if (in64) return from_inc ? by_r<double, true>(R, O) : by_r<double, false>(R, O);
    return from_inc ? by_r<float, true>(R, O) : by_r<float, false>(R, O);
}
} // namespace sigk
