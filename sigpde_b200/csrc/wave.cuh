// wave.cuh -- warp-synchronous anti-diagonal Goursat wavefront for sm_100a.
//
// One warp solves one (x, y) pair.  The refined grid has n = (len_x-1)*2^order
// rows and m = (len_y-1)*2^order columns; K = 1 on row 0 and column 0 and
//   K[i][j] = (K[i][j-1] + K[i-1][j]) * A - K[i-1][j-1] * B,
//   A = 1 + c/2 + c^2/12,  B = 1 - c^2/12,
// with c the coarse increment of cell (i,j) (sigpde/cuda_device_functions.py:3-5
// restated with the coefficients hoisted per coarse cell).
//
// Layout of the work in registers (no global scratch, no __syncthreads):
//   * rows are cut into bands of 32*R; lane l of the warp owns R consecutive
//     rows of the band and keeps their current column in registers;
//   * every step the lane advances its rows by C = 2^order columns (C = 8 for
//     order >= 4): an R x C block whose cells share one coarse column, so each
//     step needs R/2^order increments and R/2^order (A, B) pairs;
//   * lane l runs one step behind lane l-1 and receives lane l-1's bottom row
//     of the same column block through __shfl_up_sync (C values per step);
//   * a band that is not the last writes its bottom row to a per-warp
//     boundary buffer that the next band's lane 0 reads.
// The R x C block is straight-line code, so the compiler overlaps its cells
// along anti-diagonals (critical path R + C - 1 cells, 3 FP ops per cell).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sigk {

constexpr unsigned kFullMask = 0xffffffffu;

template <typename T>
__device__ __forceinline__ T ld_in(const T *p)
{
    return __ldg(p);
}

// Stencil coefficients of one coarse cell and the cell update
//   K11 = (K10 + K01) * A - K00 * B,   A = 1 + a,  B = 1 - b,
//   a = c/2 + c^2/12,  b = c^2/12.
// float64 cells hold (A, B) and update in 3 operations.  float32 cells hold
// (a, b): rounding A = 1 + c/2 to float32 keeps only ~2^-24 / c of the
// increment's relative precision (c shrinks like 4^-order), which made float32
// results ~50x less accurate than the reference's float64-arithmetic /
// float32-storage cells.  The float32 update is
//   K11 = K10 + ((K01 - K00) + K00 * b + s * a),  s = K10 + K01,
// where K01 - K00 is exact (neighbouring cells are within a factor 2 of each
// other, Sterbenz) and everything inside the parentheses is of the size of the
// increment term, so the only rounding at the magnitude of K is the final
// addition -- one rounding per cell, as in the reference's float32 storage.
// It costs 5 float32 operations per cell.
template <typename T>
__device__ __forceinline__ void stencil_coefs(T c, T &A, T &B)
{
    const T c2 = c * c;
    A = fma(c2, T(1.0 / 12.0), fma(c, T(0.5), T(1)));
    B = fma(c2, T(-1.0 / 12.0), T(1));
}

template <>
__device__ __forceinline__ void stencil_coefs<float>(float c, float &a, float &b)
{
    const float c2 = c * c;
    b = c2 * (1.0f / 12.0f);
    a = fmaf(c, 0.5f, b);
}

template <typename T>
__device__ __forceinline__ T stencil_cell(T k00, T k01, T k10, T A, T B)
{
    return fma(k10 + k01, A, -(k00 * B));
}

template <>
__device__ __forceinline__ float stencil_cell<float>(float k00, float k01, float k10, float a, float b)
{
    const float s = k10 + k01;
    return k10 + fmaf(s, a, fmaf(k00, b, k01 - k00));
}

// Compile-time shape of one lane's block.
template <int R, int O>
struct BlockShape {
    static constexpr int C = (O <= 3) ? (1 << O) : 8;                       // fine columns per step
    static constexpr int RC = (O <= 3) ? ((R >> O) > 0 ? (R >> O) : 1) : 1; // coarse rows per lane
    static constexpr int ROWS_PER_COARSE = (O <= 3) ? (1 << O) : 1 << 30;
    __host__ __device__ static constexpr int rc_of(int r) { return (RC == 1) ? 0 : r / ROWS_PER_COARSE; }
};

// Geometry of one solve.
struct SolveGeom {
    int64_t ncx, ncy; // coarse cells per side (len - 1)
    int order;
    int64_t n, m;     // refined rows / columns
    int nbands;
    int64_t nsteps;   // column blocks per band
};

template <int R, int O>
__device__ __forceinline__ SolveGeom make_geom(int64_t ncx, int64_t ncy, int order)
{
    SolveGeom g;
    g.ncx = ncx;
    g.ncy = ncy;
    g.order = order;
    g.n = ncx << order;
    g.m = ncy << order;
    g.nbands = (int)((g.n + 32 * R - 1) / (32 * R));
    g.nsteps = g.m / BlockShape<R, O>::C;
    return g;
}

// Increments read from a precomputed float matrix: c[rc] = m[cj * ld + ci0 + rc].
// Each read also asks the L2 for the lane's rows kIncPrefetch columns ahead,
// so the wavefront's loads find them there instead of waiting on HBM.
constexpr int kIncPrefetch = 8;

__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// RC consecutive values row[ci0 .. ci0+RC) of a float or double matrix as T,
// with 16-byte vector loads (the caller keeps rows and ci0 aligned); chunks
// starting at or beyond ncx read as 0.
template <typename T, typename TM, int RC>
__device__ __forceinline__ void load_mat_vals(const TM *row, int ci0, int ncx, T (&c)[RC])
{
    if constexpr (RC == 1) {
        c[0] = ci0 < ncx ? T(row[ci0]) : T(0);
    } else if constexpr (sizeof(TM) == 8) {
#pragma unroll
        for (int q = 0; q < RC / 2; ++q) {
            const double2 v = (ci0 + 2 * q < ncx) ? *reinterpret_cast<const double2 *>(row + ci0 + 2 * q)
                                                  : make_double2(0.0, 0.0);
            c[2 * q + 0] = T(v.x);
            c[2 * q + 1] = T(v.y);
        }
    } else if constexpr (RC == 2) {
        const float2 v = ci0 < ncx ? *reinterpret_cast<const float2 *>(row + ci0) : make_float2(0.f, 0.f);
        c[0] = T(v.x);
        c[1] = T(v.y);
    } else {
#pragma unroll
        for (int q = 0; q < RC / 4; ++q) {
            const float4 v = (ci0 + 4 * q < ncx) ? *reinterpret_cast<const float4 *>(row + ci0 + 4 * q)
                                                 : make_float4(0.f, 0.f, 0.f, 0.f);
            c[4 * q + 0] = T(v.x);
            c[4 * q + 1] = T(v.y);
            c[4 * q + 2] = T(v.z);
            c[4 * q + 3] = T(v.w);
        }
    }
}

// The same values as load_mat_vals, left in the matrix's type so that the
// registers can be read a step later: no conversion (which would wait for the
// load) happens here, and the zero fill is a predicated load, not a select.
template <typename TM, int RC>
__device__ __forceinline__ void load_mat_raw(const TM *row, int ci0, int ncx, TM (&v)[RC])
{
    if constexpr (RC == 1) {
        v[0] = TM(0);
        if (ci0 < ncx) v[0] = row[ci0];
    } else if constexpr (sizeof(TM) == 8) {
#pragma unroll
        for (int q = 0; q < RC / 2; ++q) {
            double2 t = make_double2(0.0, 0.0);
            if (ci0 + 2 * q < ncx) t = *reinterpret_cast<const double2 *>(row + ci0 + 2 * q);
            v[2 * q + 0] = t.x;
            v[2 * q + 1] = t.y;
        }
    } else if constexpr (RC == 2) {
        float2 t = make_float2(0.f, 0.f);
        if (ci0 < ncx) t = *reinterpret_cast<const float2 *>(row + ci0);
        v[0] = t.x;
        v[1] = t.y;
    } else {
#pragma unroll
        for (int q = 0; q < RC / 4; ++q) {
            float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
            if (ci0 + 4 * q < ncx) t = *reinterpret_cast<const float4 *>(row + ci0 + 4 * q);
            v[4 * q + 0] = t.x;
            v[4 * q + 1] = t.y;
            v[4 * q + 2] = t.z;
            v[4 * q + 3] = t.w;
        }
    }
}

template <typename T, int RC, typename TM = float>
struct MatIncs {
    const TM *base;
    int64_t ld, ncy;
    int ci0 = 0, ncx = 0;
    __device__ __forceinline__ void stage(int64_t ci0_, int64_t ncx_, int, bool)
    {
        ci0 = (int)ci0_;
        ncx = (int)ncx_;
    }
    __device__ __forceinline__ void column(int64_t cj, int, T (&c)[RC]) const
    {
        const TM *row = base + cj * ld;
        if (cj + kIncPrefetch < ncy && ci0 < ncx) prefetch_l2(row + kIncPrefetch * ld + ci0);
        load_mat_vals<T, TM, RC>(row, ci0, ncx, c);
    }
};

// Source of increments from precomputed, already scaled path differences in
// T, stored dimension-major per path (dX[k * ncx + ci], dY[k * ncy + cj]): the
// lanes of a warp read neighbouring columns cj of one dimension k together
// (lane l is one column behind lane l-1), so the loads coalesce.
// c(ci, cj) = <dX[ci], dY[cj]> (times fscale): taking the differences first
// (exact in float64 for float32 paths) avoids the cancellation of the
// reference's 4-term difference of the static Gram (sigpde/torch/kernel.py:
// 13-21); both are equal in exact arithmetic.  The lane's dx rows live in
// shared memory as [rc][k][lane] (conflict-free) when a staging area is
// given, else they are re-read from global memory.
template <typename T, int RC>
struct DeltaIncs {
    const T *dX;
    const T *dY;
    int64_t d;
    T *dxs;      // this warp's staging area: RC * d * 32 values, or null
    int64_t ci0 = 0, ncx = 0, ncy = 0;
    bool rc_per_row = false;
    T fscale = T(1); // extra factor on every increment (the robust kernel's t^2)

    __device__ __forceinline__ void stage(int64_t ci0_, int64_t ncx_, int lane, bool rc_per_row_)
    {
        ci0 = ci0_;
        ncx = ncx_;
        rc_per_row = rc_per_row_;
        if (!dxs) return;
        __syncwarp();
        for (int rc = 0; rc < RC; ++rc) {
            const int64_t ci = ci0 + (rc_per_row ? rc : 0);
            const bool ok = ci < ncx;
            for (int64_t k = 0; k < d; ++k) dxs[(rc * d + k) * 32 + lane] = ok ? dX[k * ncx + ci] : T(0);
        }
        __syncwarp();
    }

    __device__ __forceinline__ void column(int64_t cj, int lane, T (&c)[RC]) const
    {
#pragma unroll
        for (int rc = 0; rc < RC; ++rc) c[rc] = T(0);
        const T *dy = dY + cj;
        if (dxs) {
            // no unroll here: unrolling by 4 made the uneven batch 30% slower (11.2 vs 8.6 ms) and the
            // fused d = 32 Grams 25% slower
            for (int64_t k = 0; k < d; ++k) {
                const T v = dy[k * ncy];
#pragma unroll
                for (int rc = 0; rc < RC; ++rc) c[rc] = fma(dxs[(rc * d + k) * 32 + lane], v, c[rc]);
            }
        } else {
            for (int64_t k = 0; k < d; ++k) {
                const T v = dy[k * ncy];
#pragma unroll
                for (int rc = 0; rc < RC; ++rc) {
                    const int64_t ci = ci0 + (rc_per_row ? rc : 0);
                    if (ci < ncx) c[rc] = fma(dX[k * ncx + ci], v, c[rc]);
                }
            }
        }
#pragma unroll
        for (int rc = 0; rc < RC; ++rc) c[rc] *= fscale;
    }
};

// Source of increments from a coarse increment tile held in shared memory,
// tile[cj * pitch + ci], times fscale.  Used when the same pair is solved many
// times (the robust root-find re-solves a path's self-kernel every iteration
// with a new scale): the tile is built once per path.
template <typename T, int RC>
struct TileIncs {
    const T *tile;
    int64_t pitch;
    T fscale;
    int64_t ci0 = 0, ncx = 0;
    bool rc_per_row = false;

    __device__ __forceinline__ void stage(int64_t ci0_, int64_t ncx_, int, bool rc_per_row_)
    {
        ci0 = ci0_;
        ncx = ncx_;
        rc_per_row = rc_per_row_;
    }

    __device__ __forceinline__ void column(int64_t cj, int, T (&c)[RC]) const
    {
        const T *col = tile + cj * pitch;
#pragma unroll
        for (int rc = 0; rc < RC; ++rc) {
            const int64_t ci = ci0 + (rc_per_row ? rc : 0);
            c[rc] = (ci < ncx) ? col[ci] * fscale : T(0);
        }
    }
};

// Source of precomputed coarse increments (generic static kernels): strided
// reads of inc[ci][cj] in TIN, times fscale.
template <typename T, typename TIN, int RC>
struct GivenIncs {
    const TIN *inc;
    int64_t si, sj;
    T fscale;
    int64_t ci0;
    bool rc_per_row;
    int64_t ncx;

    __device__ __forceinline__ void stage(int64_t ci0_, int64_t ncx_, int, bool rc_per_row_)
    {
        ci0 = ci0_;
        ncx = ncx_;
        rc_per_row = rc_per_row_;
    }

    __device__ __forceinline__ void column(int64_t cj, int, T (&c)[RC]) const
    {
#pragma unroll
        for (int rc = 0; rc < RC; ++rc) {
            const int64_t ci = ci0 + (rc_per_row ? rc : 0);
            c[rc] = (ci < ncx) ? T(ld_in(inc + ci * si + cj * sj)) * fscale : T(0);
        }
    }
};

// Solve one pair with the warp.  Returns K[n][m] in every lane.
// bnd: per-warp boundary row buffer of m + 1 values (only touched when the
// pair has more than one band).
template <typename T, int R, int O, class Src>
__device__ T warp_solve(const SolveGeom &g, Src &src, T *bnd)
{
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    const int lane = threadIdx.x & 31;
    const bool rc_per_row = (RC > 1);
    T result = T(1);

    for (int b = 0; b < g.nbands; ++b) {
        const int64_t row0 = (int64_t)b * 32 * R + (int64_t)lane * R; // first refined row (0-based)
        src.stage(row0 >> g.order, g.ncx, lane, rc_per_row);

        T left[R];
#pragma unroll
        for (int r = 0; r < R; ++r) left[r] = T(1);
        T bot[C];
#pragma unroll
        for (int c = 0; c < C; ++c) bot[c] = T(1);
        T corner_next = T(1);
        const bool first_band = (b == 0);
        const bool write_bnd = (lane == 31) && (b + 1 < g.nbands);

        const int64_t total = g.nsteps + 31;
        for (int64_t s = 0; s < total; ++s) {
            const int64_t q = s - lane;
            T top[C];
#pragma unroll
            for (int c = 0; c < C; ++c) top[c] = __shfl_up_sync(kFullMask, bot[c], 1);
            const bool active = (q >= 0) && (q < g.nsteps);
            if (lane == 0) {
                if (first_band) {
#pragma unroll
                    for (int c = 0; c < C; ++c) top[c] = T(1);
                } else if (active) {
#pragma unroll
                    for (int c = 0; c < C; ++c) top[c] = bnd[q * C + 1 + c];
                }
            }
            if (active) {
                const T corner = (q == 0) ? T(1) : corner_next;
                corner_next = top[C - 1];
                T cc[RC];
                src.column((q * C) >> g.order, lane, cc);
                T A[RC], B[RC];
#pragma unroll
                for (int rc = 0; rc < RC; ++rc) stencil_coefs(cc[rc], A[rc], B[rc]);
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    T up = top[c];
                    T dg = (c == 0) ? corner : top[c - 1];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const T l = left[r];
                        const T v = stencil_cell(dg, up, l, A[BS::rc_of(r)], B[BS::rc_of(r)]);
                        dg = l;
                        up = v;
                        left[r] = v;
                    }
                    bot[c] = up;
                }
                if (write_bnd) {
#pragma unroll
                    for (int c = 0; c < C; ++c) bnd[q * C + 1 + c] = bot[c];
                }
            }
        }
        __syncwarp(); // orders lane 31's boundary stores before the next band's loads

        if (b == g.nbands - 1) {
            const int64_t last = g.n - 1 - (int64_t)b * 32 * R; // row index within the band
            const int lstar = (int)(last / R);
            const int rstar = (int)(last % R);
            T v = left[0];
#pragma unroll
            for (int r = 1; r < R; ++r)
                if (r == rstar) v = left[r];
            result = __shfl_sync(kFullMask, v, lstar);
        }
    }
    return result;
}

} // namespace sigk
