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
    double *out;
    int64_t ld;           // = npaths_x * rows_x
};

__device__ __forceinline__ double load_elem(const void *base, int64_t i, int in64)
{
    return in64 ? reinterpret_cast<const double *>(base)[i] : (double)reinterpret_cast<const float *>(base)[i];
}

template <int KIND, int DM>
__device__ __forceinline__ double static_k(const double (&xp)[DM], double xn, const double *yp, double yn, double inv)
{
    if constexpr (KIND == kStaticRbf) {
        double dot = 0.0;
#pragma unroll
        for (int k = 0; k < DM; k += 2) {
            const double2 v = *reinterpret_cast<const double2 *>(yp + k);
            dot = fma(xp[k], v.x, dot);
            dot = fma(xp[k + 1], v.y, dot);
        }
        return exp(-((xn + yn) - 2.0 * dot) * inv);
    } else {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < DM; k += 2) {
            const double2 v = *reinterpret_cast<const double2 *>(yp + k);
            s += fabs(xp[k] - v.x);
            s += fabs(xp[k + 1] - v.y);
        }
        return exp(-s * inv);
    }
}

template <int KIND, int DM>
__global__ void __launch_bounds__(kStWarps * 32) static_inc_kernel(StaticIncParams p)
{
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
    double xp[DM];
    double xn = 0.0;
#pragma unroll
    for (int k = 0; k < DM; ++k) {
        xp[k] = (gin && k < p.d) ? load_elem(p.x, g * p.d + k, p.in64) : 0.0;
        xn = fma(xp[k], xp[k], xn);
    }
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
                    ys[s + h][k] = v;
                    yn = fma(v, v, yn);
                }
                yns[s + h] = yn;
            }
            ysc[c] = p.sy ? load_elem(p.sy, qy, p.in64) : 1.0;
        }
        __syncthreads();
        int64_t cj = n0 - q0 * ncy;
        int s = 0;
        double k_lo = 0.0, k_lo_up = 0.0; // k(x_ci, y_cj) of this lane and of the next (x_ci+1)
        double *o = p.out + n0 * p.ld + m;
        for (int c = 0; c < nt; ++c) {
            if (c == 0 || cj == 0) { // uniform: first column of the tile or of a y path
                k_lo = static_k<KIND, DM>(xp, xn, ys[s], yns[s], p.inv_param);
                k_lo_up = __shfl_down_sync(0xffffffffu, k_lo, 1);
            }
            const double k_hi = static_k<KIND, DM>(xp, xn, ys[s + 1], yns[s + 1], p.inv_param);
            const double k_hi_up = __shfl_down_sync(0xffffffffu, k_hi, 1);
            if (row) {
                *o = (((k_hi_up + k_lo) - k_lo_up) - k_hi) * (sxf * ysc[c]);
            } else if (pad) {
                for (int64_t r = 0; r < p.rows_x - ncx; ++r) o[r] = 0.0;
            }
            k_lo = k_hi;
            k_lo_up = k_hi_up;
            o += p.ld;
            ++s;
            if (++cj == ncy) { // the next column starts a new path: skip this path's last point
                cj = 0;
                ++s;
            }
        }
    }
}

} // namespace sigk
