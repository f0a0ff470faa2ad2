// Instantiations of pair_kernel with float64 cells (SIGK_PREC_FP64).
#include "dispatch.h"
#include "sigk_kernels.cuh"

namespace sigk {
namespace {
template <typename TIN, int R, int FI>
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
template <typename TIN, int FI>
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

PairFn get_pair_kernel_f64(bool in64, int mode, int R, int O)
{
    if (in64) {
        if (mode == kPairMat64) return by_r<double, kPairMat64>(R, O);
        if (mode == kPairMat) return by_r<double, kPairMat>(R, O);
        return mode == kPairGiven ? by_r<double, kPairGiven>(R, O) : by_r<double, kPairDelta>(R, O);
    }
    if (mode == kPairMat64) return by_r<float, kPairMat64>(R, O);
    if (mode == kPairMat) return by_r<float, kPairMat>(R, O);
    return mode == kPairGiven ? by_r<float, kPairGiven>(R, O) : by_r<float, kPairDelta>(R, O);
}
} // namespace sigk
