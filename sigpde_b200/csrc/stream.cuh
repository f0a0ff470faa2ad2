// stream.cuh -- streaming wavefront: one warp walks a contiguous run of pairs.
//
// The per-pair warp solve of wave.cuh spends 31 of its nsteps + 31 steps
// filling and draining the lane pipeline (lane l runs l steps behind lane 0).
// Here the pipeline never drains between pairs: lane l starts pair k+1 the
// step after it finished pair k, exactly one step behind lane l-1, so a warp
// that owns E pairs runs E * nsteps + 31 steps instead of E * (nsteps + 31).
//
// Preconditions (checked on the host): one band (refined rows <= 32 R) and
// nsteps >= 32 column blocks per pair.
//
// Increments come from path differences precomputed in T by delta_kernel
// (float64 differences of float32 points are exact) with all scale factors
// folded in, so the inner loop does no conversions and no scaling:
// c(ci, cj) = <dX[ci], dY[cj]>.
//
// Two variants:
//   stream_reg_kernel  -- the lane's dx rows (RC coarse rows x D dims, D the
//                         dimension padded to a power of two) live in
//                         registers and are reloaded only when the lane's x
//                         path changes (rarely, for a row-major Gram);
//   stream_smem_kernel -- for RC * D > 32: dx rows double-buffered in shared
//                         memory.  The buffer for pair k is written (by the
//                         whole warp, when lane 0 starts pair k) at least one
//                         step after lane 31 finished pair k - 2, its last
//                         reader, because nsteps >= 32.
#pragma once

#include "sigk_kernels.cuh"

namespace sigk {

// dx[p][k][c] = T(x[p][c+1][k]) - T(x[p][c][k]) for all paths p, stored
// dimension-major: the lanes of a warp read neighbouring coarse columns c of
// one dimension k in the same instruction (lane l is one column behind lane
// l-1), so a load touches 2 cache lines instead of 16.  Dimensions d <= k < dp
// are written as zeros (dp = padded dimension of the register variant), so the
// inner loop needs no bound checks.
// Every row is multiplied by f * s[p] (s may be null): folding the static
// scale, 4^-order and the per-path scales into the differences leaves the
// stream kernels nothing to scale, since <f s_i dx_i, s_j dy_j> is the scaled
// increment f * s_i * s_j * <dx_i, dy_j> of sigpde/cuda_gram_kernels.py:52,60.
template <typename T, typename TIN>
__global__ void delta_kernel(const void *x_, int64_t npaths, int64_t len, int64_t d, int64_t dp, double f,
                             const void *s_, void *dx_)
{
    const TIN *__restrict__ x = reinterpret_cast<const TIN *>(x_);
    const TIN *__restrict__ sc = reinterpret_cast<const TIN *>(s_);
    T *__restrict__ dx = reinterpret_cast<T *>(dx_);
    const int64_t nc = len - 1;
    const int64_t per_path = nc * dp;
    const int64_t total = npaths * per_path;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = e / per_path;
        const int64_t r = e - p * per_path; // k * nc + c
        const int64_t k = r / nc;
        const int64_t c = r - k * nc;
        if (k < d) {
            const TIN *xp = x + p * len * d + c * d + k;
            const T g = sc ? T(f * (double)sc[p]) : T(f);
            dx[e] = (T(xp[d]) - T(xp[0])) * g;
        } else {
            dx[e] = T(0);
        }
    }
}

struct StreamParams {
    int op;             // kOpPairwise / kOpGram / kOpGramSym
    int in64;           // 1: scales and output are float64, 0: float32
    const void *dx;     // (nx, dp, ncx) in T, scaled (see delta_kernel)
    const void *dy;     // (ny, dp, ncy) in T, scaled
    int64_t nx, ny;
    int64_t ncx, ncy, d;
    int64_t dp;         // padded dimension of dx / dy (d for the shared-memory variant)
    int order;
    void *out;
    int64_t out_ld;
    int64_t nitems;
    int64_t per_warp;   // items per warp (contiguous run)
};

__device__ __forceinline__ void stream_decode(const StreamParams &p, int64_t item, int64_t &xi, int64_t &yj)
{
    if (p.op == kOpPairwise) {
        xi = item;
        yj = item;
    } else if (p.op == kOpGram) {
        xi = item / p.ny;
        yj = item - xi * p.ny;
    } else {
        tri_decode(item, xi, yj);
    }
}

template <typename T>
__device__ __forceinline__ void stream_store(const StreamParams &p, int64_t item, int64_t xi, int64_t yj, T v)
{
    int64_t i0, i1 = -1;
    if (p.op == kOpPairwise) {
        i0 = item;
    } else {
        i0 = xi * p.out_ld + yj;
        if (p.op == kOpGramSym && xi != yj) i1 = yj * p.out_ld + xi;
    }
    if (p.in64) {
        double *o = reinterpret_cast<double *>(p.out);
        o[i0] = double(v);
        if (i1 >= 0) o[i1] = double(v);
    } else {
        float *o = reinterpret_cast<float *>(p.out);
        o[i0] = float(v);
        if (i1 >= 0) o[i1] = float(v);
    }
}

// One R x C block of cells: left[] holds the lane's column on entry and the
// new column on exit; top[] is the row above (from lane l-1), corner the cell
// above-left; bot[] receives the block's bottom row.
template <typename T, int R, int O>
__device__ __forceinline__ void stream_block(T (&left)[R], const T (&top)[BlockShape<R, O>::C], T corner,
                                             const T (&A)[BlockShape<R, O>::RC], const T (&B)[BlockShape<R, O>::RC],
                                             T (&bot)[BlockShape<R, O>::C])
{
    using BS = BlockShape<R, O>;
#pragma unroll
    for (int c = 0; c < BS::C; ++c) {
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
}

template <typename T, int R>
__device__ __forceinline__ T pick_row(const T (&left)[R], int rstar)
{
    T v = left[0];
#pragma unroll
    for (int r = 1; r < R; ++r)
        if (r == rstar) v = left[r];
    return v;
}

// Paired float32 cells.  A float32 lane of stream_reg_kernel is issue-bound
// (5 float32 instructions per cell plus the per-step shuffles and loads), so
// here each lane advances two pairs at once and every cell operation is one
// sm_100 paired instruction (add / mul / fma .f32x2) on a (pair a, pair b)
// register pair.  The arithmetic of each half is exactly the float32
// stencil_coefs / stencil_cell above (k01 - k00 is formed as
// fma(k00, -1, k01), which rounds identically), so every value is
// bit-identical to stream_reg_kernel<float>.
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }

template <>
__device__ __forceinline__ void stencil_coefs<float2>(float2 c, float2 &a, float2 &b)
{
    const float2 c2 = __fmul2_rn(c, c);
    b = __fmul2_rn(c2, splat2(1.0f / 12.0f));
    a = __ffma2_rn(c, splat2(0.5f), b);
}

template <>
__device__ __forceinline__ float2 stencil_cell<float2>(float2 k00, float2 k01, float2 k10, float2 a, float2 b)
{
    const float2 s = __fadd2_rn(k10, k01);
    const float2 t = __ffma2_rn(k00, splat2(-1.0f), k01);
    return __fadd2_rn(k10, __ffma2_rn(s, a, __ffma2_rn(k00, b, t)));
}

// stream_reg_kernel with paired float32 cells: the warp's run of items is
// walked two at a time (items first + 2k and first + 2k + 1 share every
// pipeline step; an odd run leaves the last step's second half unused).
// dx holds (x_a, x_b) for each coarse row and dimension; it is reloaded only
// when either x path changes.
template <int R, int O, int D>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) stream_reg_paired_kernel(StreamParams p)
{
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    const int64_t first = gwarp * p.per_warp;
    if (first >= p.nitems) return; // warp-uniform
    const int cnt = (int)((p.nitems - first) < p.per_warp ? (p.nitems - first) : p.per_warp);
    const int cnt2 = (cnt + 1) >> 1;
    const float *dX = reinterpret_cast<const float *>(p.dx);
    const float *dY = reinterpret_cast<const float *>(p.dy);
    const int ncx = (int)p.ncx, ncy = (int)p.ncy;
    const int n = ncx << p.order;
    const int nsteps = (ncy << p.order) / C;
    const int ci0 = (lane * R) >> p.order;
    const int lstar = (n - 1) / R, rstar = (n - 1) % R;
    const float2 one = splat2(1.0f);

    float2 dx[RC][D];
    int64_t cur_xa = -1, cur_xb = -1;
    float2 left[R];
#pragma unroll
    for (int r = 0; r < R; ++r) left[r] = one;
    float2 bot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) bot[c] = one;
    float2 corner_next = one;
    int q = 0, k = 0;
    int64_t ia = first, xa = 0, ya = 0, xb = 0, yb = 0;
    bool hasb = false;
    const float *dypa = dY, *dypb = dY;

    const int total = cnt2 * nsteps + 31;
    for (int s = 0; s < total; ++s) {
        float2 top[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            top[c].x = __shfl_up_sync(kFullMask, bot[c].x, 1);
            top[c].y = __shfl_up_sync(kFullMask, bot[c].y, 1);
        }
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < C; ++c) top[c] = one;
        }
        if (s >= lane && k < cnt2) {
            if (q == 0) { // this lane starts items first + 2k, first + 2k + 1
                ia = first + 2 * k;
                hasb = 2 * k + 1 < cnt;
                stream_decode(p, ia, xa, ya);
                if (hasb) {
                    stream_decode(p, ia + 1, xb, yb);
                } else {
                    xb = xa;
                    yb = ya;
                }
                dypa = dY + ya * (int64_t)D * ncy;
                dypb = dY + yb * (int64_t)D * ncy;
                if (xa != cur_xa || xb != cur_xb) {
                    cur_xa = xa;
                    cur_xb = xb;
                    const float *srca = dX + xa * (int64_t)D * ncx;
                    const float *srcb = dX + xb * (int64_t)D * ncx;
#pragma unroll
                    for (int rc = 0; rc < RC; ++rc) {
                        const int ci = ci0 + (RC > 1 ? rc : 0);
                        const bool ok = ci < ncx;
#pragma unroll
                        for (int kk = 0; kk < D; ++kk)
                            dx[rc][kk] = ok ? make_float2(srca[kk * ncx + ci], srcb[kk * ncx + ci]) : splat2(0.0f);
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r) left[r] = one;
            }
            const float2 corner = (q == 0) ? one : corner_next;
            corner_next = top[C - 1];
            const int cj = (O <= 3) ? q : ((q * C) >> p.order);
            float2 cc[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) cc[rc] = splat2(0.0f);
            const float *dyra = dypa + cj;
            const float *dyrb = dypb + cj;
#pragma unroll
            for (int kk = 0; kk < D; ++kk) {
                const float2 dy = make_float2(dyra[kk * ncy], dyrb[kk * ncy]);
#pragma unroll
                for (int rc = 0; rc < RC; ++rc) cc[rc] = __ffma2_rn(dx[rc][kk], dy, cc[rc]);
            }
            float2 A[RC], B[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) stencil_coefs(cc[rc], A[rc], B[rc]);
            stream_block<float2, R, O>(left, top, corner, A, B, bot);
            if (q == nsteps - 1 && lane == lstar) {
                const float2 v = pick_row(left, rstar);
                stream_store(p, ia, xa, ya, v.x);
                if (hasb) stream_store(p, ia + 1, xb, yb, v.y);
            }
            if (++q == nsteps) {
                q = 0;
                ++k;
            }
        }
    }
}

// Two Gram entries per lane with float64 cells: the lane advances entries
// (xi, ya) and (xi, ya + 1) of one x path together, so each cell operation
// comes as two independent float64 instructions (twice the instruction-level
// parallelism of stream_reg_kernel, with dx held once).  Each half is exactly
// stream_reg_kernel<double>'s arithmetic.  kOpGram only; items are entry pairs
// t: xi = t / hy, ya = 2 (t % hy), hy = ceil(ny / 2) (the second entry is
// absent when ya + 1 == ny).
struct Dbl2 {
    double x, y;
};

template <>
__device__ __forceinline__ void stencil_coefs<Dbl2>(Dbl2 c, Dbl2 &A, Dbl2 &B)
{
    stencil_coefs<double>(c.x, A.x, B.x);
    stencil_coefs<double>(c.y, A.y, B.y);
}

template <>
__device__ __forceinline__ Dbl2 stencil_cell<Dbl2>(Dbl2 k00, Dbl2 k01, Dbl2 k10, Dbl2 A, Dbl2 B)
{
    return Dbl2{stencil_cell<double>(k00.x, k01.x, k10.x, A.x, B.x), stencil_cell<double>(k00.y, k01.y, k10.y, A.y, B.y)};
}

// Increments one step ahead (stream_reg_kernel, stream_reg_dual_kernel).  A
// step's increments take D loads of dy and RC x D dependent fma chains; formed
// at the start of the step, they put a load latency and D fmas on the critical
// path ahead of the first cell.  So a lane forms the increments of its NEXT
// step (the same fma chains, bitwise) in the same basic block as the current
// step's cells, where the loads and dot products, which do not depend on the
// cells, fill the cells' latency gaps (Gram 256 x 256, L = 128, d = 8, order
// 2: 5.13 ms against 5.31 ms with the increments formed in-step).  The next
// entry of the run is decoded one entry ahead, when the current one starts;
// when it has another x path, the dot products formed with the old dx are
// discarded and redone after the dx reload (rare: a run moves to a new x path
// at most a few times).
template <typename T, int D, int RC>
__device__ __forceinline__ void stream_dot(const T (&dx)[RC][D], const T *dyr, int64_t ncy, T (&cc)[RC])
{
#pragma unroll
    for (int rc = 0; rc < RC; ++rc) cc[rc] = T(0);
#pragma unroll
    for (int kk = 0; kk < D; ++kk) {
        const T dy = dyr[kk * ncy];
#pragma unroll
        for (int rc = 0; rc < RC; ++rc) cc[rc] = fma(dx[rc][kk], dy, cc[rc]);
    }
}

template <typename T, int D, int RC>
__device__ __forceinline__ void stream_load_dx(const T *dX, int64_t xi, int ncx, int ci0, T (&dx)[RC][D])
{
    const T *src = dX + xi * (int64_t)D * ncx;
#pragma unroll
    for (int rc = 0; rc < RC; ++rc) {
        const int ci = ci0 + (RC > 1 ? rc : 0);
#pragma unroll
        for (int kk = 0; kk < D; ++kk) dx[rc][kk] = (ci < ncx) ? src[kk * ncx + ci] : T(0);
    }
}

// Three CTAs (12 warps) per SM, except for blocks of 8 or more coarse rows a lane,
// whose coefficient arrays need more than 168 registers.
template <typename T, int R, int O, int D>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, (BlockShape<R, O>::RC >= 8 ? 2 : 3))
    stream_reg_kernel(StreamParams p)
{
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    const int64_t first = gwarp * p.per_warp;
    if (first >= p.nitems) return; // warp-uniform
    const int cnt = (int)((p.nitems - first) < p.per_warp ? (p.nitems - first) : p.per_warp);
    const T *dX = reinterpret_cast<const T *>(p.dx);
    const T *dY = reinterpret_cast<const T *>(p.dy);
    const int ncx = (int)p.ncx, ncy = (int)p.ncy;
    const int n = ncx << p.order;
    const int nsteps = (ncy << p.order) / C;
    const int ci0 = (lane * R) >> p.order;
    const int lstar = (n - 1) / R, rstar = (n - 1) % R;
    const int64_t ystride = (int64_t)D * ncy;

    // the entry being solved and the next one of the run (decoded when the current one starts)
    int64_t item = first, xi = 0, yj = 0;
    int64_t nxi, nyj;
    stream_decode(p, first, nxi, nyj);
    const T *dyp = dY + nyj * ystride, *ndyp = dyp;
    T dx[RC][D];
    int64_t cur_x = nxi;
    stream_load_dx<T, D, RC>(dX, nxi, ncx, ci0, dx);
    T cc[RC]; // increments of this lane's next step
    stream_dot<T, D, RC>(dx, dyp, ncy, cc);

    T left[R];
#pragma unroll
    for (int r = 0; r < R; ++r) left[r] = T(1);
    T bot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) bot[c] = T(1);
    T corner_next = T(1);
    int q = 0, k = 0;

    const int total = cnt * nsteps + 31;
    for (int s = 0; s < total; ++s) {
        T top[C];
#pragma unroll
        for (int c = 0; c < C; ++c) top[c] = __shfl_up_sync(kFullMask, bot[c], 1);
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < C; ++c) top[c] = T(1);
        }
        if (s >= lane && k < cnt) {
            if (q == 0) { // this lane starts entry `first + k`, decoded at the previous start
                item = first + k;
                xi = nxi;
                yj = nyj;
                dyp = ndyp;
                if (xi != cur_x) { // the ahead increments used the previous x path's dx
                    cur_x = xi;
                    stream_load_dx<T, D, RC>(dX, xi, ncx, ci0, dx);
                    stream_dot<T, D, RC>(dx, dyp, ncy, cc);
                }
                if (k + 1 < cnt) {
                    stream_decode(p, item + 1, nxi, nyj);
                    ndyp = dY + nyj * ystride;
                }
#pragma unroll
                for (int r = 0; r < R; ++r) left[r] = T(1);
            }
            const T corner = (q == 0) ? T(1) : corner_next;
            corner_next = top[C - 1];
            T A[RC], B[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) stencil_coefs(cc[rc], A[rc], B[rc]);
            // the next step: q + 1 of this entry, or step 0 of the next one
            const int qn = (q + 1 == nsteps) ? 0 : q + 1;
            const int cjn = (O <= 3) ? qn : ((qn * C) >> p.order);
            stream_dot<T, D, RC>(dx, ((qn == 0) ? ndyp : dyp) + cjn, ncy, cc);
            stream_block<T, R, O>(left, top, corner, A, B, bot);
            if (q == nsteps - 1 && lane == lstar) stream_store(p, item, xi, yj, pick_row(left, rstar));
            if (++q == nsteps) {
                q = 0;
                ++k;
            }
        }
    }
}

// Two entries of one x path per lane, increments one step ahead as in
// stream_reg_kernel.
template <int R, int O, int D>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 2) stream_reg_dual_kernel(StreamParams p)
{
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    const int64_t first = gwarp * p.per_warp;
    if (first >= p.nitems) return; // warp-uniform
    const int cnt = (int)((p.nitems - first) < p.per_warp ? (p.nitems - first) : p.per_warp);
    const double *dX = reinterpret_cast<const double *>(p.dx);
    const double *dY = reinterpret_cast<const double *>(p.dy);
    const int ncx = (int)p.ncx, ncy = (int)p.ncy;
    const int n = ncx << p.order;
    const int nsteps = (ncy << p.order) / C;
    const int ci0 = (lane * R) >> p.order;
    const int lstar = (n - 1) / R, rstar = (n - 1) % R;
    const int64_t hy = (p.ny + 1) >> 1;
    const int64_t ystride = (int64_t)D * ncy;
    const Dbl2 one{1.0, 1.0};

    // entry pair t -> x path t / hy, y paths ya = 2 (t % hy) and ya + 1 (absent when ya + 1 == ny)
    auto decode = [&](int64_t t, int64_t &x, int64_t &ya, bool &hasb, const double *&pa, const double *&pb) {
        x = t / hy;
        ya = 2 * (t - x * hy);
        hasb = ya + 1 < p.ny;
        pa = dY + ya * ystride;
        pb = hasb ? pa + ystride : pa;
    };
    int64_t xi = 0, ya = 0, nxi, nya;
    bool hasb = false, nhasb;
    const double *dypa, *dypb, *ndypa, *ndypb;
    decode(first, nxi, nya, nhasb, ndypa, ndypb);
    dypa = ndypa;
    dypb = ndypb;
    double dx[RC][D];
    int64_t cur_x = nxi;
    stream_load_dx<double, D, RC>(dX, nxi, ncx, ci0, dx);
    double cca[RC], ccb[RC]; // increments of this lane's next step, entries a and b
    stream_dot<double, D, RC>(dx, dypa, ncy, cca);
    stream_dot<double, D, RC>(dx, dypb, ncy, ccb);

    Dbl2 left[R];
#pragma unroll
    for (int r = 0; r < R; ++r) left[r] = one;
    Dbl2 bot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) bot[c] = one;
    Dbl2 corner_next = one;
    int q = 0, k = 0;

    const int total = cnt * nsteps + 31;
    for (int s = 0; s < total; ++s) {
        Dbl2 top[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            top[c].x = __shfl_up_sync(kFullMask, bot[c].x, 1);
            top[c].y = __shfl_up_sync(kFullMask, bot[c].y, 1);
        }
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < C; ++c) top[c] = one;
        }
        if (s >= lane && k < cnt) {
            if (q == 0) { // this lane starts entry pair `first + k`, decoded at the previous start
                xi = nxi;
                ya = nya;
                hasb = nhasb;
                dypa = ndypa;
                dypb = ndypb;
                if (xi != cur_x) { // the ahead increments used the previous x path's dx
                    cur_x = xi;
                    stream_load_dx<double, D, RC>(dX, xi, ncx, ci0, dx);
                    stream_dot<double, D, RC>(dx, dypa, ncy, cca);
                    stream_dot<double, D, RC>(dx, dypb, ncy, ccb);
                }
                if (k + 1 < cnt) decode(first + k + 1, nxi, nya, nhasb, ndypa, ndypb);
#pragma unroll
                for (int r = 0; r < R; ++r) left[r] = one;
            }
            const Dbl2 corner = (q == 0) ? one : corner_next;
            corner_next = top[C - 1];
            Dbl2 A[RC], B[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) stencil_coefs(Dbl2{cca[rc], ccb[rc]}, A[rc], B[rc]);
            const int qn = (q + 1 == nsteps) ? 0 : q + 1;
            const int cjn = (O <= 3) ? qn : ((qn * C) >> p.order);
            stream_dot<double, D, RC>(dx, ((qn == 0) ? ndypa : dypa) + cjn, ncy, cca);
            stream_dot<double, D, RC>(dx, ((qn == 0) ? ndypb : dypb) + cjn, ncy, ccb);
            stream_block<Dbl2, R, O>(left, top, corner, A, B, bot);
            if (q == nsteps - 1 && lane == lstar) {
                const Dbl2 v = pick_row(left, rstar);
                stream_store(p, 0, xi, ya, v.x);
                if (hasb) stream_store(p, 0, xi, ya + 1, v.y);
            }
            if (++q == nsteps) {
                q = 0;
                ++k;
            }
        }
    }
}

template <typename T, int R, int O>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) stream_smem_kernel(StreamParams p)
{
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    const int64_t first = gwarp * p.per_warp;
    if (first >= p.nitems) return; // warp-uniform
    const int cnt = (int)((p.nitems - first) < p.per_warp ? (p.nitems - first) : p.per_warp);

    const int ncx = (int)p.ncx, ncy = (int)p.ncy, d = (int)p.d;
    const int stage_elems = RC * d * 32;
    T *buf0 = reinterpret_cast<T *>(smem_raw) + (int64_t)wib * 2 * stage_elems;
    T *buf1 = buf0 + stage_elems;
    const T *dX = reinterpret_cast<const T *>(p.dx);
    const T *dY = reinterpret_cast<const T *>(p.dy);

    const int n = ncx << p.order;
    const int nsteps = (ncy << p.order) / C;
    const int ci0 = (lane * R) >> p.order;
    const int lstar = (n - 1) / R, rstar = (n - 1) % R;

    T left[R];
#pragma unroll
    for (int r = 0; r < R; ++r) left[r] = T(1);
    T bot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) bot[c] = T(1);
    T corner_next = T(1);
    int q = 0, k = 0;
    int64_t item = first, xi = 0, yj = 0;
    const T *dyp = dY;
    const T *dxs = buf0;
    int staged = 0;     // pairs staged so far (warp-uniform)
    int next_stage = 0; // step at which lane 0 starts pair `staged`

    const int total = cnt * nsteps + 31;
    for (int s = 0; s < total; ++s) {
        if (staged < cnt && s == next_stage) { // warp-uniform: lane 0 starts a new pair now
            int64_t sxi, syj;
            stream_decode(p, first + staged, sxi, syj);
            T *dst = (staged & 1) ? buf1 : buf0;
            const T *src = dX + sxi * (int64_t)d * ncx;
            __syncwarp();
            for (int rc = 0; rc < RC; ++rc) {
                const int ci = ci0 + (RC > 1 ? rc : 0);
                const bool ok = ci < ncx;
                for (int kk = 0; kk < d; ++kk) dst[(rc * d + kk) * 32 + lane] = ok ? src[kk * ncx + ci] : T(0);
            }
            __syncwarp();
            ++staged;
            next_stage += nsteps;
        }
        T top[C];
#pragma unroll
        for (int c = 0; c < C; ++c) top[c] = __shfl_up_sync(kFullMask, bot[c], 1);
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < C; ++c) top[c] = T(1);
        }
        if (s >= lane && k < cnt) {
            if (q == 0) {
                item = first + k;
                stream_decode(p, item, xi, yj);
                dyp = dY + yj * (int64_t)d * ncy;
                dxs = (k & 1) ? buf1 : buf0;
#pragma unroll
                for (int r = 0; r < R; ++r) left[r] = T(1);
            }
            const T corner = (q == 0) ? T(1) : corner_next;
            corner_next = top[C - 1];
            const int cj = (q * C) >> p.order;
            T cc[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) cc[rc] = T(0);
            const T *dyr = dyp + cj;
            for (int kk = 0; kk < d; ++kk) {
                const T dy = dyr[kk * ncy];
#pragma unroll
                for (int rc = 0; rc < RC; ++rc) cc[rc] = fma(dxs[(rc * d + kk) * 32 + lane], dy, cc[rc]);
            }
            T A[RC], B[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) stencil_coefs(cc[rc], A[rc], B[rc]);
            stream_block<T, R, O>(left, top, corner, A, B, bot);
            if (q == nsteps - 1 && lane == lstar) stream_store(p, item, xi, yj, pick_row(left, rstar));
            if (++q == nsteps) {
                q = 0;
                ++k;
            }
        }
    }
}

} // namespace sigk
