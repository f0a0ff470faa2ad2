// Float64 increment matrix of a non-linear static kernel, straight from the
// path points (fp64 Grams with RBFKernel / L1RBFKernel).
//
// The reference materialises the static Gram k(x_p, y_q) of every point pair
// in the input dtype (sigpde/torch/static_kernels.py:13-53), takes the 4-term
// second difference and divides by 4^order (sigpde/torch/kernel.py:18-21),
// then scales by scale_x[i] * scale_y[j] inside the solver
// (sigpde/cuda_gram_kernels.py:43-60).  Here one kernel evaluates k in
// float64 and writes the scaled coarse increments
//   inc(ci, cj) = ((k(x_ci+1, y_cj+1) + k(x_ci, y_cj)) - k(x_ci+1, y_cj) - k(x_ci, y_cj+1))
//                 * 4^-order * scale_x * scale_y
// into the layout of the float64 increment matrix (dgemm_inc.cuh), which the
// wavefront then reads (stream_inc_kernel / pair_kernel, float64 elements).
//
//   RBF     k = exp(-(|x|^2 + |y|^2 - 2 <x, y>) / sigma)   (static_kernels.py:13-36)
//   L1-RBF  k = exp(-sum_k |x_k - y_k| / sigma)            (static_kernels.py:38-53)
//
// Work split: lane l of a warp holds one x point in registers (dimensions
// padded to DM with zeros, which add nothing to either distance); a warp
// covers 32 consecutive points of the chunk's point sequence (path-major) and
// outputs the 31 rows whose lower point is on lanes 0..30, reading the upper
// point's kernel values from lane l+1 by a shuffle, so each k is evaluated
// about once per stored increment.  The CTA walks a tile of 64 columns (y
// cells) whose points are staged in shared memory: k(x, y_cj) of one column
// is k(x, y_cj+1) of the previous one within a y path.
#pragma once

#include "dgemm_inc.cuh"

namespace sigk {

enum : int { kStaticLinear = 0, kStaticRbf = 1, kStaticL1Rbf = 2 }; // values of sigk_static_kind

constexpr int kStTileN = 64;        // columns (y cells) per tile
constexpr int kStWarps = 8;         // warps per CTA
constexpr int kStRowsPerWarp = 31;  // points 0..31 of a warp give rows 0..30
constexpr int kStSlots = 2 * kStTileN + 1; // y points of a tile: its cells' lower points plus each path's last

struct StaticIncParams {
    const void *x, *y;    // points (npaths, len, d), float32 or float64; x chunk-relative
    int in64;
    int64_t npaths_x, lx, rows_x;
    int64_t npaths_y, ly;
    int64_t d;
    double inv_param;     // 1 / sigma
    double f;             // 4^-order
    const void *sx, *sy;  // per-path scales in the input dtype (x chunk-relative) or null
    int mode;             // kTcAll / kTcLower
    int64_t x0;           // kTcLower: global index of the first x path
    void *out;            // TO (double for float64 cells, float for float32 cells)
    int64_t ld;           // = npaths_x * rows_x
};

__device__ __forceinline__ double load_elem(const void *base, int64_t i, int in64)
{
    return in64 ? reinterpret_cast<const double *>(base)[i] : (double)reinterpret_cast<const float *>(base)[i];
}

// e^a for a <= 0 (arguments up to a few ulps above 0 are fine); measured
// about 25% faster in this kernel than the library exp, whose out-of-line
// slow path costs registers and spills here.  Cody-Waite
// range reduction and a Taylor polynomial: a = k ln2 + r with k = rint(a /
// ln2), |r| <= ln2 / 2, r = (a - k ln2_hi) - k ln2_lo where ln2_hi holds the
// 32 leading bits of ln 2 (k ln2_hi is exact for |k| < 2^21) and ln2_lo =
// ln 2 - ln2_hi; e^r = sum_{n <= 13} r^n / n! (truncation below 5e-18
// relative), as even and odd parts in r^2; then 2^k is added to the exponent field.  Results below
// 2^-1021 (a < -707.7) flush to zero, where every increment they feed is
// below 1e-300.
__device__ __forceinline__ double exp_nonpos(double a)
{
    constexpr double kLog2e = 1.4426950408889634;
    constexpr double kLn2Hi = 0.6931471806019545;     // 0x3fe62e42ff000000
    constexpr double kLn2Lo = -4.2009150726810846e-11; // ln 2 - kLn2Hi
    const double kd = rint(a * kLog2e);
    const double r = fma(-kd, kLn2Lo, fma(-kd, kLn2Hi, a));
    // even and odd halves as two independent Horner chains in r^2 (half the dependent latency)
    const double r2 = r * r;
    double e = 2.08767569878681e-09;                   // 1/12!
    double o = 1.6059043836821613e-10;                 // 1/13!
    e = fma(e, r2, 2.755731922398589e-07);             // 1/10!
    o = fma(o, r2, 2.505210838544172e-08);             // 1/11!
    e = fma(e, r2, 2.48015873015873e-05);              // 1/8!
    o = fma(o, r2, 2.7557319223985893e-06);            // 1/9!
    e = fma(e, r2, 0.001388888888888889);              // 1/6!
    o = fma(o, r2, 0.0001984126984126984);             // 1/7!
    e = fma(e, r2, 0.041666666666666664);              // 1/4!
    o = fma(o, r2, 0.008333333333333333);              // 1/5!
    e = fma(e, r2, 0.5);                               // 1/2!
    o = fma(o, r2, 0.16666666666666666);               // 1/3!
    e = fma(e, r2, 1.0);                               // 1/0!
    o = fma(o, r2, 1.0);                               // 1/1!
    const double q = fma(o, r, e);
    const int k = (int)kd;
    return k < -1021 ? 0.0 : __longlong_as_double(__double_as_longlong(q) + ((long long)k << 52));
}

// k for one y point from the lane's x point.  The y points in shared memory
// are pre-scaled: RBF y * (2 / sigma) with |y|^2 / sigma beside them and the
// lane's |x|^2 / sigma in xn, so the exponent is <x, y'> - xn - yn; L1-RBF x
// and y both / sigma.
template <int KIND, int DM>
__device__ __forceinline__ double static_k(const double (&xp)[DM], double xn, const double *yp, double yn)
{
    double a;
    if constexpr (KIND == kStaticRbf) {
        double d0 = 0.0, d1 = 0.0; // even / odd dimensions: two independent chains
#pragma unroll
        for (int k = 0; k < DM; k += 2) {
            const double2 v = *reinterpret_cast<const double2 *>(yp + k);
            d0 = fma(xp[k], v.x, d0);
            d1 = fma(xp[k + 1], v.y, d1);
        }
        a = ((d0 + d1) - xn) - yn;
    } else {
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int k = 0; k < DM; k += 2) {
            const double2 v = *reinterpret_cast<const double2 *>(yp + k);
            s0 += fabs(xp[k] - v.x);
            s1 += fabs(xp[k + 1] - v.y);
        }
        a = -(s0 + s1);
    }
    return exp_nonpos(a);
}

// TO: the matrix element type.  Every increment is formed in float64; float32
// cells read it rounded once to float32 (the tensor-core modes' matrix type).
template <int KIND, int DM, typename TO>
__global__ void __launch_bounds__(kStWarps * 32) static_inc_kernel(StaticIncParams p)
{
    TO *const out = reinterpret_cast<TO *>(p.out);
    static_assert(DM % 2 == 0, "points are read as double2");
    __shared__ __align__(16) double ys[kStSlots][DM];
    __shared__ double yns[kStSlots];
    __shared__ double ysc[kStTileN];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t lx = p.lx, ncx = lx - 1, ncy = p.ly - 1;
    const int64_t npts = p.npaths_x * lx;
    const int64_t gbase = (int64_t)blockIdx.x * kStWarps * kStRowsPerWarp;
    const int64_t g = gbase + (int64_t)warp * kStRowsPerWarp + lane;
    const bool gin = g < npts;
    const int64_t px = gin ? g / lx : 0, ci = gin ? g - px * lx : 0;
    const double xs = KIND == kStaticRbf ? 1.0 : p.inv_param;   // L1-RBF: x / sigma
    const double ysf = KIND == kStaticRbf ? 2.0 * p.inv_param : p.inv_param;
    double xp[DM];
    double xn = 0.0;
#pragma unroll
    for (int k = 0; k < DM; ++k) {
        const double v = (gin && k < p.d) ? load_elem(p.x, g * p.d + k, p.in64) : 0.0;
        xn = fma(v, v, xn);
        xp[k] = v * xs;
    }
    xn *= p.inv_param;
    // lanes 0..30 own the point; a point below the path's last gives a row, the last writes the padding rows
    const bool row = gin && lane < kStRowsPerWarp && ci < ncx;
    const bool pad = gin && lane < kStRowsPerWarp && ci == ncx;
    const double sxf = (p.sx ? load_elem(p.sx, px, p.in64) : 1.0) * p.f;
    const int64_t m = px * p.rows_x + ci;
    int64_t g_hi = gbase + kStWarps * kStRowsPerWarp; // last point this CTA reads
    if (g_hi > npts - 1) g_hi = npts - 1;
    const int64_t px_hi = g_hi / lx;

    const int64_t ncols = p.npaths_y * ncy;
    for (int64_t n0 = (int64_t)blockIdx.y * kStTileN; n0 < ncols; n0 += (int64_t)gridDim.y * kStTileN) {
        const int64_t q0 = n0 / ncy;
        if (p.mode == kTcLower && q0 > px_hi + p.x0) break; // this and later tiles are above the diagonal
        const int nt = (int)((ncols - n0) < kStTileN ? (ncols - n0) : kStTileN);
        __syncthreads(); // the previous tile's readers are done
        // column c's lower point goes to slot c + (its path - first path); its upper point is the next
        // slot, written by column c + 1 within a path, else here
        for (int c = threadIdx.x; c < nt; c += blockDim.x) {
            const int64_t n = n0 + c, qy = n / ncy, cj = n - qy * ncy;
            const int s = (int)(c + (qy - q0));
            const bool last = cj == ncy - 1 || c == nt - 1;
            for (int h = 0; h <= (last ? 1 : 0); ++h) {
                const int64_t pt = qy * p.ly + cj + h;
                double yn = 0.0;
#pragma unroll
                for (int k = 0; k < DM; ++k) {
                    const double v = k < p.d ? load_elem(p.y, pt * p.d + k, p.in64) : 0.0;
                    ys[s + h][k] = v * ysf;
                    yn = fma(v, v, yn);
                }
                yns[s + h] = yn * p.inv_param;
            }
            ysc[c] = p.sy ? load_elem(p.sy, qy, p.in64) : 1.0;
        }
        __syncthreads();
        if (pad) { // zero rows ncx .. rows_x - 1 of this path, every column of the tile
            for (int c = 0; c < nt; ++c)
                for (int64_t r = 0; r < p.rows_x - ncx; ++r) out[(n0 + c) * p.ld + m + r] = TO(0);
        }
        // the tile's columns in runs within one y path: k(x, y_cj) of a column is k(x, y_cj+1) of the last
        int c = 0, s = 0;
        int cj = (int)(n0 - q0 * ncy);
        TO *o = out + n0 * p.ld + m;
        while (c < nt) {
            const int run = (int)((nt - c) < (ncy - cj) ? (nt - c) : (ncy - cj));
            const double scl = sxf * ysc[c];
            double k_lo = static_k<KIND, DM>(xp, xn, ys[s], yns[s]);
            double k_lo_up = __shfl_down_sync(0xffffffffu, k_lo, 1); // k(x_ci+1, y_cj) from the next lane
#pragma unroll 2
            for (int i = 1; i <= run; ++i) {
                const double k_hi = static_k<KIND, DM>(xp, xn, ys[s + i], yns[s + i]);
                const double k_hi_up = __shfl_down_sync(0xffffffffu, k_hi, 1);
                if (row) *o = TO((((k_hi_up + k_lo) - k_lo_up) - k_hi) * scl);
                o += p.ld;
                k_lo = k_hi;
                k_lo_up = k_hi_up;
            }
            c += run;
            s += run + 1; // skip this path's last point
            cj = 0;
        }
    }
}

} // namespace sigk
