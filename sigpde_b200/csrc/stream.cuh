// stream.cuh -- streaming wavefront: one warp walks a contiguous run of pairs.
//
// The per-pair warp solve of wave.cuh spends 31 of its nsteps + 31 steps
// filling and draining the lane pipeline (lane l runs l steps behind lane 0).
// Here the pipeline never drains between pairs: lane l starts pair k+1 the
// step after it finished pair k, exactly one step behind lane l-1, so a warp
// that owns E pairs runs E * nsteps + 31 steps instead of E * (nsteps + 31).
//
// Preconditions (checked on the host): one band (refined rows <= 32 R) and
// nsteps >= 32 column blocks per pair.  The second condition makes the double
// buffer of staged dx rows safe: the buffer for pair k is written (by the
// whole warp, when lane 0 starts pair k) at least one step after lane 31
// finished pair k - 2, the last reader of that buffer.
//
// Increments come from path differences precomputed in T by delta_kernel
// (float64 differences of float32 points are exact), so the inner loop does
// no conversions: c(ci, cj) = fscale * <dX[ci], dY[cj]>.
#pragma once

#include "sigk_kernels.cuh"

namespace sigk {

// dx[p][c][k] = T(x[p][c+1][k]) - T(x[p][c][k]) for all paths p.
template <typename T, typename TIN>
__global__ void delta_kernel(const void *x_, int64_t npaths, int64_t len, int64_t d, void *dx_)
{
    const TIN *__restrict__ x = reinterpret_cast<const TIN *>(x_);
    T *__restrict__ dx = reinterpret_cast<T *>(dx_);
    const int64_t per_path = (len - 1) * d;
    const int64_t total = npaths * per_path;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = e / per_path;
        const int64_t r = e - p * per_path; // c * d + k
        const TIN *xp = x + p * len * d;
        dx[e] = T(xp[r + d]) - T(xp[r]);
    }
}

struct StreamParams {
    int op;             // kOpPairwise / kOpGram / kOpGramSym
    const void *dx;     // (nx, ncx, d) in T
    const void *dy;     // (ny, ncy, d) in T
    int64_t nx, ny;
    int64_t ncx, ncy, d;
    int order;
    double fscale;
    const void *sx;
    const void *sy;
    void *out;
    int64_t out_ld;
    int64_t nitems;
    int64_t per_warp;   // items per warp (contiguous run)
};

template <typename T, typename TIN, int R, int O>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) stream_kernel(StreamParams p)
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
    const int64_t cnt = (p.nitems - first) < p.per_warp ? (p.nitems - first) : p.per_warp;

    const int64_t d = p.d;
    const int64_t stage_elems = (int64_t)RC * d * 32;
    T *buf0 = reinterpret_cast<T *>(smem_raw) + (int64_t)wib * 2 * stage_elems;
    T *buf1 = buf0 + stage_elems;
    const T *dX = reinterpret_cast<const T *>(p.dx);
    const T *dY = reinterpret_cast<const T *>(p.dy);
    TIN *out = reinterpret_cast<TIN *>(p.out);

    const int64_t n = p.ncx << p.order;
    const int64_t nsteps = (p.ncy << p.order) / C;
    const int64_t ci0 = ((int64_t)lane * R) >> p.order; // first coarse row of this lane
    const int lstar = (int)((n - 1) / R);
    const int rstar = (int)((n - 1) % R);

    auto decode = [&](int64_t item, int64_t &xi, int64_t &yj) {
        if (p.op == kOpPairwise) {
            xi = item;
            yj = item;
        } else if (p.op == kOpGram) {
            xi = item / p.ny;
            yj = item - xi * p.ny;
        } else {
            tri_decode(item, xi, yj);
        }
    };

    T left[R];
#pragma unroll
    for (int r = 0; r < R; ++r) left[r] = T(1);
    T bot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) bot[c] = T(1);
    T corner_next = T(1);
    int64_t q = 0, k = 0;     // this lane's column block and pair offset (valid once s >= lane)
    int64_t item = first, xi = 0, yj = 0;
    const T *dyp = dY;
    T fs = T(0);
    const T *dxs = buf0;
    int64_t staged = 0;       // pairs staged so far (warp-uniform)
    int64_t next_stage = 0;   // step at which lane 0 starts pair `staged`

    const int64_t total = cnt * nsteps + 31;
    for (int64_t s = 0; s < total; ++s) {
        if (staged < cnt && s == next_stage) { // warp-uniform: lane 0 starts a new pair now
            int64_t sxi, syj;
            decode(first + staged, sxi, syj);
            T *dst = (staged & 1) ? buf1 : buf0;
            const T *src = dX + sxi * p.ncx * d;
            __syncwarp();
            for (int rc = 0; rc < RC; ++rc) {
                const int64_t ci = ci0 + (RC > 1 ? rc : 0);
                const bool ok = ci < p.ncx;
                for (int64_t kk = 0; kk < d; ++kk) dst[(rc * d + kk) * 32 + lane] = ok ? src[ci * d + kk] : T(0);
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
        const bool active = (s >= lane) && (k < cnt);
        if (active) {
            if (q == 0) { // this lane starts pair `first + k`
                item = first + k;
                decode(item, xi, yj);
                dyp = dY + yj * p.ncy * d;
                double f = p.fscale;
                if (p.sx) f *= scale_at<TIN>(p.sx, xi);
                if (p.sy) f *= scale_at<TIN>(p.sy, yj);
                fs = T(f);
                dxs = (k & 1) ? buf1 : buf0;
#pragma unroll
                for (int r = 0; r < R; ++r) left[r] = T(1);
            }
            const T corner = (q == 0) ? T(1) : corner_next;
            corner_next = top[C - 1];
            // increments of this lane's coarse rows at coarse column cj
            const int64_t cj = (q * C) >> p.order;
            T cc[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) cc[rc] = T(0);
            const T *dyr = dyp + cj * d;
            for (int64_t kk = 0; kk < d; ++kk) {
                const T dy = dyr[kk];
#pragma unroll
                for (int rc = 0; rc < RC; ++rc) cc[rc] = fma(dxs[(rc * d + kk) * 32 + lane], dy, cc[rc]);
            }
            T A[RC], B[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) stencil_coefs(cc[rc] * fs, A[rc], B[rc]);
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
            if (q == nsteps - 1 && lane == lstar) {
                T v = left[0];
#pragma unroll
                for (int r = 1; r < R; ++r)
                    if (r == rstar) v = left[r];
                if (p.op == kOpPairwise) {
                    out[item] = TIN(v);
                } else {
                    out[xi * p.out_ld + yj] = TIN(v);
                    if (p.op == kOpGramSym && xi != yj) out[yj * p.out_ld + xi] = TIN(v);
                }
            }
            if (++q == nsteps) {
                q = 0;
                ++k;
            }
        }
    }
}

} // namespace sigk
