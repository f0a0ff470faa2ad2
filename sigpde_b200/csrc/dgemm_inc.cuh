// Float64 increment matrix on the CUDA cores, for wide paths in fp64 mode.
//
// The fused kernels form each coarse increment <dx_ci, dy_cj> inside the
// wavefront: d FMAs per coarse cell, re-done by every pair, on the critical
// path of each step.  For d >= 16 that dominates, so the Gram ops first write
// the increments of all pairs with one register-blocked FP64 GEMM over the
// scaled, dimension-major differences (delta_kernel) and the wavefront then
// reads them (stream_inc_kernel / pair_kernel in matrix mode, float64
// elements).  Each entry is summed as fma(dx_k, dy_k, acc) for k = 0 .. d-1
// in order, from zero: the order of the fused kernels, so the results are
// bitwise those of the fused path.
//
// Layout as for the tensor-core matrix (tc.cuh): out[n * ld + m], m = x path *
// rows_x + ci (rows ci >= ncx are zero), n = y path * ncy + cj.
#pragma once

#include "tc.cuh"

namespace sigk {

constexpr int kDgTile = 64; // rows and columns of a CTA tile
constexpr int kDgK = 16;    // K chunk staged in shared memory

struct DgemmIncParams {
    const double *dx;     // (npaths_x, d, ncx), chunk-relative
    const double *dy;     // (npaths_y, d, ncy)
    int64_t npaths_x, ncx, rows_x;
    int64_t npaths_y, ncy;
    int64_t d;
    int mode;             // kTcAll / kTcLower
    int64_t x0;           // kTcLower: global index of the first x path
    double *out;
    int64_t ld;           // = npaths_x * rows_x
};

template <int TILE = kDgTile>
__global__ void __launch_bounds__(256, 3) dgemm_inc_kernel(DgemmIncParams p)
{
    static_assert(TILE == 64, "4x4 outputs per thread of a 16x16 block");
    __shared__ double As[kDgK][TILE + 1];
    __shared__ double Bs[kDgK][TILE + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t m0 = (int64_t)blockIdx.x * TILE;
    const int64_t n_rows = p.npaths_y * p.ncy;
    for (int64_t n0 = (int64_t)blockIdx.y * TILE; n0 < n_rows; n0 += (int64_t)gridDim.y * TILE) {
        if (p.mode == kTcLower) { // tiles entirely above the diagonal of path pairs are not needed
            int64_t i_hi = (m0 + TILE - 1) / p.rows_x;
            if (i_hi >= p.npaths_x) i_hi = p.npaths_x - 1;
            if (n0 / p.ncy > i_hi + p.x0) continue; // uniform across the CTA
        }
        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
        // this thread stages row mm = threadIdx.x % 64 of the A and B tiles (K rows threadIdx.x / 64 + 4r):
        // its path and cell are fixed for the tile, so the divisions happen once
        const int mm = threadIdx.x & (TILE - 1), kq = threadIdx.x / TILE;
        const int64_t m = m0 + mm, n = n0 + mm;
        const int64_t px = m / p.rows_x, cx = m - px * p.rows_x;
        const int64_t qy = n / p.ncy, cy = n - qy * p.ncy;
        const bool a_ok = px < p.npaths_x && cx < p.ncx, b_ok = qy < p.npaths_y;
        const double *a_src = p.dx + (a_ok ? px * p.d * p.ncx + cx : 0);
        const double *b_src = p.dy + (b_ok ? qy * p.d * p.ncy + cy : 0);
        for (int64_t k0 = 0; k0 < p.d; k0 += kDgK) {
            // stage A[m][k] and B[n][k] for k in [k0, k0 + 16): threads run over m (n), which are
            // contiguous within a path in the dimension-major differences
#pragma unroll
            for (int r = 0; r < kDgK * TILE / 256; ++r) {
                const int kk = kq + r * (256 / TILE);
                const int64_t k = k0 + kk;
                As[kk][mm] = (a_ok && k < p.d) ? a_src[k * p.ncx] : 0.0;
                Bs[kk][mm] = (b_ok && k < p.d) ? b_src[k * p.ncy] : 0.0;
            }
            __syncthreads();
            const int kn = (int)((p.d - k0) < kDgK ? (p.d - k0) : kDgK);
            for (int kk = 0; kk < kn; ++kk) {
                double a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
                for (int j = 0; j < 4; ++j) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
            }
            __syncthreads();
        }
        // out[n * ld + m]: for each (i, j) the 16 threads of a half-warp write 16 consecutive m
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t n = n0 + ty + 16 * j;
            if (n >= n_rows) continue;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t m = m0 + tx + 16 * i;
                if (m < p.ld) p.out[n * p.ld + m] = acc[i][j];
            }
        }
    }
}

} // namespace sigk
