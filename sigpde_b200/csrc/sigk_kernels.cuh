// sigk_kernels.cuh -- persistent-warp kernels built on warp_solve (wave.cuh).
//
//   pair_kernel       pairwise / Gram / symmetric-Gram signature kernels
//   normalize_kernel  robust normalisation: per-path Chandrupatla root-find
//                     whose every iteration re-solves the PDE on-chip
//
// Each kernel is a grid of 4-warp blocks sized to the resident capacity of
// the device; warp w handles work items w, w + W, w + 2W, ... (W = warps in
// the grid).  Gram items are numbered row-major, so neighbouring warps share
// x_i and read neighbouring y_j (L1/L2 reuse).
#pragma once

#include <type_traits>

#include "wave.cuh"

namespace sigk {

enum : int { kOpPairwise = 0, kOpGram = 1, kOpGramSym = 2 };

constexpr int kWarpsPerBlock = 4;

struct PairParams {
    int op;
    const void *x;
    const void *y;
    int64_t nx, ny;     // path counts (pairwise: batch in both)
    int64_t ncx, ncy;   // coarse cells per side (len - 1)
    int64_t d;
    int order;
    double fscale;      // static_scale * 4^-order (path mode) or 1 (increment mode)
    const void *sx;
    const void *sy;
    const void *dx;     // path mode: scaled differences (nx, d, ncx) in T, dimension-major (delta_kernel)
    const void *dy;     // (ny, d, ncy)
    const void *inc;    // increment mode only
    int64_t is0, is1, is2, is3;
    // matrix mode (tensor-core increments, tc.cuh): pair (xi, yj)'s increments start at
    // mat + yj * ncy * mat_ld + (xi - x0) * mat_rows_x (Gram ops; pairwise: mat + (item - item0) * ncy *
    // mat_rows_x), mat_ld (pairwise: mat_rows_x) floats per coarse column
    const void *mat;         // float (tensor-core increments) or double (dgemm_inc_kernel) elements
    const unsigned *mat_err; // non-zero: the GEMM gave up a wait, the matrix is incomplete (results NaN)
    int64_t mat_ld, mat_rows_x, x0;
    int64_t item0;      // first item of this launch (matrix mode works in chunks of x paths)
    void *out;
    int64_t out_ld;
    int64_t nitems;
    void *bnd;          // per-warp boundary rows (multi-band pairs only)
    int64_t bnd_stride; // elements per warp
    int stage_smem;     // 1: dx rows staged in shared memory
};

// Lower-triangle index w -> (i, j), i >= j, w = i*(i+1)/2 + j.
__device__ __forceinline__ void tri_decode(int64_t w, int64_t &i, int64_t &j)
{
    int64_t r = (int64_t)((sqrt(8.0 * (double)w + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > w) --r;
    while ((r + 1) * (r + 2) / 2 <= w) ++r;
    i = r;
    j = w - r * (r + 1) / 2;
}

template <typename TIN>
__device__ __forceinline__ double scale_at(const void *s, int64_t i)
{
    return s ? (double)reinterpret_cast<const TIN *>(s)[i] : 1.0;
}

enum : int { kPairDelta = 0, kPairGiven = 1, kPairMat = 2, kPairMat64 = 3 };

template <typename T, typename TIN, int R, int O, int MODE>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) pair_kernel(PairParams p)
{
    using BS = BlockShape<R, O>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const SolveGeom g = make_geom<R, O>(p.ncx, p.ncy, p.order);
    T *bnd = p.bnd ? reinterpret_cast<T *>(p.bnd) + gwarp * p.bnd_stride : nullptr;
    TIN *out = reinterpret_cast<TIN *>(p.out);

    for (int64_t item0 = gwarp; item0 < p.nitems; item0 += nwarps) {
        const int64_t item = p.item0 + item0;
        int64_t xi, yj;
        if (p.op == kOpPairwise) {
            xi = item;
            yj = item;
        } else if (p.op == kOpGram) {
            xi = item / p.ny;
            yj = item - xi * p.ny;
        } else {
            tri_decode(item, xi, yj);
        }
        double s = p.fscale;
        if (p.sx) s *= scale_at<TIN>(p.sx, xi);
        if (p.sy) s *= scale_at<TIN>(p.sy, yj);

        T val;
        if constexpr (MODE == kPairMat || MODE == kPairMat64) {
            using TM = typename std::conditional<MODE == kPairMat64, double, float>::type;
            MatIncs<T, BS::RC, TM> src;
            const TM *mat = reinterpret_cast<const TM *>(p.mat);
            if (p.op == kOpPairwise) {
                src.base = mat + (item - p.item0) * p.ncy * p.mat_rows_x;
                src.ld = p.mat_rows_x;
            } else {
                src.base = mat + yj * p.ncy * p.mat_ld + (xi - p.x0) * p.mat_rows_x;
                src.ld = p.mat_ld;
            }
            src.ncy = p.ncy;
            val = (p.mat_err == nullptr || *p.mat_err == 0) ? warp_solve<T, R, O>(g, src, bnd) : T(NAN);
        } else if constexpr (MODE == kPairGiven) {
            GivenIncs<T, TIN, BS::RC> src;
            const TIN *base = reinterpret_cast<const TIN *>(p.inc);
            if (p.op == kOpPairwise) {
                src.inc = base + item * p.is0;
                src.si = p.is1;
                src.sj = p.is2;
            } else {
                src.inc = base + xi * p.is0 + yj * p.is1;
                src.si = p.is2;
                src.sj = p.is3;
            }
            src.fscale = T(s);
            val = warp_solve<T, R, O>(g, src, bnd);
        } else {
            DeltaIncs<T, BS::RC> src;
            src.dX = reinterpret_cast<const T *>(p.dx) + xi * p.d * p.ncx;
            src.dY = reinterpret_cast<const T *>(p.dy) + yj * p.d * p.ncy;
            src.d = p.d;
            src.ncy = p.ncy;
            src.dxs = p.stage_smem ? reinterpret_cast<T *>(smem_raw) + (int64_t)wib * BS::RC * p.d * 32 : nullptr;
            val = warp_solve<T, R, O>(g, src, bnd);
        }
        if (lane == 0) {
            if (p.op == kOpPairwise) {
                out[item] = TIN(val);
            } else {
                out[xi * p.out_ld + yj] = TIN(val);
                if (p.op == kOpGramSym && xi != yj) out[yj * p.out_ld + xi] = TIN(val);
            }
        }
    }
}

enum : int { kNormDelta = 0, kNormGiven = 1, kNormTile = 2 };

struct NormParams {
    const void *x;
    const double *dx;   // delta / tile modes: path differences (n, d, nc), dimension-major, unscaled
    int64_t tile_pitch; // tile mode: row pitch (elements) of the shared-memory increment tile
    int64_t n;
    int64_t nc;
    int64_t d;
    int order;
    double fscale;      // static_scale * 4^-order (path mode) or 1
    const void *inc;    // increment mode only
    int64_t is0, is1, is2;
    double *knorm;      // builtin: output (may be null); external: input
    const double *fnorm; // null: builtin f(s) = 2 - 1/(1 + log s)
    double tol;
    int maxit;
    void *lam;
    int *iters;
    void *bnd;
    int64_t bnd_stride;
    int stage_smem;
    // pipelined kernel (norm_pipe.cuh): per-CTA band progress counters (16 ints per CTA,
    // zeroed before the launch) and the flag a band wait that ran out sets
    int *prog;
    int *err;
};

// k(x,x), f(k) and the Chandrupatla iteration for one path, given solve(s) =
// k at increments scaled by s: sigpde/cuda_pairwise_kernels.py:88-165 with
// the argument order of sigpde/torch/kernel.py:186-193: g(l) = k(l x) - f(k),
// g(0) = 1 - f(k), g(1) = k - f(k).  All bracket state is float64 and uniform
// across the threads that call it (solve returns the same value to all of
// them); `writer` stores k(x,x).
template <class Solve>
__device__ __forceinline__ void normalize_path(const NormParams &p, int64_t b, bool writer, Solve &&solve,
                                               double &out, int &it)
{
    double k, fk;
    if (p.fnorm == nullptr) {
        k = solve(1.0);
        if (isnan(k)) k = __longlong_as_double(0x7ff0000000000000LL); // NaN -> +inf (kernel.py:183)
        fk = 2.0 - 1.0 / (1.0 + log(k));                              // kernel.py:23-24
        if (p.knorm && writer) p.knorm[b] = k;
    } else {
        k = p.knorm[b];
        fk = p.fnorm[b];
    }
    out = 0.0;
    it = 0;
    if (k >= 1.0) { // lambda is forced to 0 for k < 1 (kernel.py:195), so the loop is skipped
        double a = 0.0, c = 0.0, bb = 1.0;
        double fa = 1.0 - fk;
        double fb = k - fk;
        double fc = fa;
        double t = 0.5;
        for (it = 0; it < p.maxit;) {
            const double xt = a + t * (bb - a);
            const double sol = solve(xt * xt);
            const double ft = isnan(sol) ? __longlong_as_double(0x7ff0000000000000LL) : sol - fk;
            ++it;
            if (ft * fa >= 0) {
                c = a;
                fc = fa;
            } else {
                c = bb;
                bb = a;
                fc = fb;
                fb = fa;
            }
            a = xt;
            fa = ft;
            if (fabs(fa) < fabs(fb)) {
                out = a;
                if (fabs(fa) < p.tol) break;
            } else {
                out = bb;
                if (fabs(fb) < p.tol) break;
            }
            const double xi = (a - bb) / (c - bb);
            const double phi = (fa - fb) / (fc - fb);
            if (phi * phi < xi && (1 - phi) * (1 - phi) < 1 - xi)
                t = fa / (fb - fa) * fc / (fb - fc) + (c - a) / (bb - a) * fa / (fc - fa) * fb / (fc - fb);
            else
                t = 0.5;
            if (!(0 < t && t < 1)) t = 0.5;
        }
    }
}

// One path per warp: every bracket iteration re-solves the path's PDE on chip.
template <typename TIN, int R, int O, int MODE>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) normalize_kernel(NormParams p)
{
    using T = double;
    using BS = BlockShape<R, O>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const SolveGeom g = make_geom<R, O>(p.nc, p.nc, p.order);
    T *bnd = p.bnd ? reinterpret_cast<T *>(p.bnd) + gwarp * p.bnd_stride : nullptr;
    TIN *lam_out = reinterpret_cast<TIN *>(p.lam);

    for (int64_t b = gwarp; b < p.n; b += nwarps) {
        DeltaIncs<T, BS::RC> dsrc;
        GivenIncs<T, TIN, BS::RC> gsrc;
        TileIncs<T, BS::RC> tsrc;
        if constexpr (MODE == kNormGiven) {
            gsrc.inc = reinterpret_cast<const TIN *>(p.inc) + b * p.is0;
            gsrc.si = p.is1;
            gsrc.sj = p.is2;
        } else if constexpr (MODE == kNormDelta) {
            dsrc.dX = p.dx + b * p.d * p.nc;
            dsrc.dY = dsrc.dX;
            dsrc.d = p.d;
            dsrc.ncy = p.nc;
            dsrc.dxs = p.stage_smem ? reinterpret_cast<T *>(smem_raw) + (int64_t)wib * BS::RC * p.d * 32 : nullptr;
        } else {
            // build this path's coarse increment tile once: tile[cj][ci] = <dx_ci, dx_cj>
            T *tile = reinterpret_cast<T *>(smem_raw) + (int64_t)wib * p.nc * p.tile_pitch;
            const double *dxb = p.dx + b * p.d * p.nc;
            __syncwarp(); // the previous path's solves are done with the tile
            for (int64_t e = lane; e < p.nc * p.nc; e += 32) {
                const int64_t cj = e / p.nc;
                const int64_t ci = e - cj * p.nc;
                T acc = T(0);
                for (int64_t k = 0; k < p.d; ++k) acc = fma(dxb[k * p.nc + ci], dxb[k * p.nc + cj], acc);
                tile[cj * p.tile_pitch + ci] = acc;
            }
            __syncwarp();
            tsrc.tile = tile;
            tsrc.pitch = p.tile_pitch;
        }
        auto solve = [&](double scale) -> double {
            if constexpr (MODE == kNormGiven) {
                gsrc.fscale = p.fscale * scale;
                return warp_solve<T, R, O>(g, gsrc, bnd);
            } else if constexpr (MODE == kNormDelta) {
                dsrc.fscale = p.fscale * scale;
                return warp_solve<T, R, O>(g, dsrc, bnd);
            } else {
                tsrc.fscale = p.fscale * scale;
                return warp_solve<T, R, O>(g, tsrc, bnd);
            }
        };

        double out = 0.0;
        int it = 0;
        normalize_path(p, b, lane == 0, solve, out, it);
        if (lane == 0) {
            if (lam_out) lam_out[b] = TIN(out);
            if (p.iters) p.iters[b] = it;
        }
    }
}

} // namespace sigk
