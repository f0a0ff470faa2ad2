// ragged.cuh -- uneven batched pairwise kernel (paths of different lengths and
// a dyadic order per pair), one persistent launch.
//
// Paths are packed: x_pack holds every x path's points back to back, x_off[b]
// is the first point of pair b's x path and x_len[b] its length (same for y).
// A prologue (ragged_delta_kernel) writes every path's differences in the
// cell precision, dimension-major and already scaled (static scale * 4^-order
// * scale_x on the x side, scale_y on the y side), so the wavefront's loads
// coalesce and it does no conversions.
//
// Work items are bands, not pairs.  Pair b is cut into pair_bands[b] bands of
// 32 * pair_rows[b] refined rows (the shorter path on the rows, since
// k(x, y) = k(y, x)); the items of a pair are consecutive, band 0 first, and
// the pairs come longest first.  Warps take items from a global counter, so a
// long pair runs on several warps at once as a pipeline: the warp on band j
// reads band j-1's bottom row from a boundary buffer in global memory as the
// warp on band j-1 publishes it (a progress counter per item, written with
// release semantics every 16 column blocks and at the end, read with acquire
// semantics).  The producer of every band was taken from the counter before
// its consumer, by a warp of this persistent grid, all of whose warps are
// resident, so each wait ends; the waits are nevertheless bounded and, if
// one runs out, the band is poisoned with NaN and an error flag is set.
// Each item picks its variant at run time: dyadic order O and rows per lane R.
#pragma once

#include "sigk_kernels.cuh"

namespace sigk {

// Differences of every path in a packed batch.  Path p (length len[p],
// first point off[p]) writes (len[p] - 1) * d values at (off[p] - p) * d,
// ordered [k][c]; each is multiplied by f * 4^-order[p] * scale[p] (order and
// scale may be null).  Paths shorter than 2 points write nothing.
template <typename T, typename TIN>
__global__ void ragged_delta_kernel(const void *pack_, const int64_t *off, const int64_t *len, const int *order,
                                    double f, const void *scale_, int64_t npaths, int64_t d, void *out_)
{
    const TIN *pack = reinterpret_cast<const TIN *>(pack_);
    const TIN *scale = reinterpret_cast<const TIN *>(scale_);
    T *out = reinterpret_cast<T *>(out_);
    for (int64_t p = blockIdx.y; p < npaths; p += gridDim.y) {
        const int64_t nc = len[p] - 1;
        if (nc < 1) continue;
        double g = f;
        if (order) g *= ldexp(1.0, -2 * order[p]);
        if (scale) g *= (double)scale[p];
        const T gt = T(g);
        const int64_t base = (off[p] - p) * d;
        const TIN *xp = pack + off[p] * d;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nc * d;
             e += (int64_t)gridDim.x * blockDim.x) {
            const int64_t k = e / nc;
            const int64_t c = e - k * nc;
            out[base + e] = (T(xp[(c + 1) * d + k]) - T(xp[c * d + k])) * gt;
        }
    }
}

struct RaggedParams {
    const void *dx_pack;        // scaled differences (see ragged_delta_kernel), T
    const void *dy_pack;
    const int64_t *x_off;
    const int64_t *x_len;
    const int64_t *y_off;
    const int64_t *y_len;
    const int *order;           // per pair
    const int64_t *item_pair;   // per item
    const int *item_band;       // per item
    int64_t nitems;
    const int *pair_rows;       // R per pair (2, 4, 8 or 16)
    const int *pair_bands;      // bands per pair
    const int64_t *pair_bnd_off; // offset of the pair's boundary rows in the pool (elements of T)
    int64_t bnd_elems;          // pool size (elements of T)
    int64_t npairs;
    int64_t d;
    void *out;                  // (npairs,) in TIN
    unsigned long long *counter; // zeroed before the launch
    int *progress;              // per item, zeroed before the launch
    int *error;                 // set to 1 if a wait ran out or an item was invalid
    void *pool;                 // boundary rows
    int stage_elems_per_warp;   // dx staging capacity (elements of T) per warp
    // precomputed increments (tensor-core modes: float; fp64 with a plan: double): pair b's block starts
    // at inc + inc_off[b], column-major over its coarse cells (row path on the rows) with round_up(rows, 4)
    // elements per column
    const void *inc;
    const int64_t *inc_off;
    int64_t inc_elems;
    const unsigned *tc_err;     // non-zero: the GEMM skipped a tile, the matrix is incomplete
    long long poll_limit;       // polls of a band wait before it gives up (kProgressPollLimit by default)
};

constexpr long long kProgressPollLimit = 1ll << 26; // ~4 s with 64 ns sleeps
// Bits of a launch's error word: an item broke the plan rules (or its increments are missing), and a band
// wait ran out.  Either way the affected pair's result is NaN.
constexpr int kErrInvalidItem = 1;
constexpr int kErrWaitTimeout = 2;
constexpr int kProgressStride = 16;                 // column blocks between publications

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Spin (with at most `limit` polls after the first read) until *prog >= need; returns the value seen, or
// -1 on timeout.
__device__ __forceinline__ int wait_progress(const int *prog, int need, long long limit)
{
    int v = ld_acquire(prog);
    for (long long i = 0; v < need; ++i) {
        if (i >= limit) return -1;
        __nanosleep(64);
        v = ld_acquire(prog);
    }
    return v;
}

// One band of one pair.  top_buf / top_prog: the band above (null for band 0);
// bot_buf / bot_prog: this band's bottom row and progress (bot_buf null for the
// last band).  Returns K[n][m] in every lane if `last`, else 1.
// prog_base: progress values of this solve are prog_base + (column blocks
// done), so one set of counters serves consecutive solves (the pipelined
// normalisation re-solves a path several times without resetting them);
// pub_stride: column blocks between publications of the band's progress.
template <typename T, int R, int O, class Src>
__device__ T band_solve(const SolveGeom &g, Src &src, int band, bool last, const T *top_buf, const int *top_prog,
                        T *bot_buf, int *bot_prog, int *error, int prog_base = 0, int pub_stride = kProgressStride,
                        long long poll_limit = kProgressPollLimit)
{
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    const int lane = threadIdx.x & 31;
    const int64_t row0 = (int64_t)band * 32 * R + (int64_t)lane * R;
    src.stage(row0 >> g.order, g.ncx, lane, RC > 1);

    T left[R];
#pragma unroll
    for (int r = 0; r < R; ++r) left[r] = T(1);
    T bot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) bot[c] = T(1);
    T corner_next = T(1);
    const bool writer = (lane == 31) && bot_buf != nullptr;
    int seen = 0;          // lane 0: column blocks of the band above known to be published
    bool poisoned = false; // lane 0: a wait ran out, feed NaN down the band

    const int64_t total = g.nsteps + 31;
    for (int64_t s = 0; s < total; ++s) {
        const int64_t q = s - lane;
        T top[C];
#pragma unroll
        for (int c = 0; c < C; ++c) top[c] = __shfl_up_sync(kFullMask, bot[c], 1);
        const bool active = (q >= 0) && (q < g.nsteps);
        if (lane == 0) {
            if (!top_buf) {
#pragma unroll
                for (int c = 0; c < C; ++c) top[c] = T(1);
            } else if (active) {
                if (!poisoned && seen <= q) {
                    const int v0 = wait_progress(top_prog, prog_base + (int)q + 1, poll_limit);
                    const int v = (v0 < 0 || v0 == 0x7fffffff) ? v0 : v0 - prog_base;
                    if (v < 0 || v == 0x7fffffff) { // ran out, or the band above was refused
                        poisoned = true;
                        if (v < 0) atomicOr(error, kErrWaitTimeout);
                    } else {
                        seen = v;
                    }
                }
#pragma unroll
                for (int c = 0; c < C; ++c)
                    top[c] = poisoned ? T(__longlong_as_double(0x7ff8000000000000LL)) : __ldcg(top_buf + q * C + 1 + c);
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
            if (writer) {
#pragma unroll
                for (int c = 0; c < C; ++c) bot_buf[q * C + 1 + c] = bot[c];
                if ((q + 1) % pub_stride == 0 || q + 1 == g.nsteps) {
                    __threadfence();
                    st_release(bot_prog, prog_base + (int)q + 1);
                }
            }
        }
    }
    T result = T(1);
    if (last) {
        const int64_t lastrow = g.n - 1 - (int64_t)band * 32 * R;
        const int lstar = (int)(lastrow / R);
        const int rstar = (int)(lastrow % R);
        T v = left[0];
#pragma unroll
        for (int r = 1; r < R; ++r)
            if (r == rstar) v = left[r];
        result = __shfl_sync(kFullMask, v, lstar);
    }
    return result;
}

// The increments of one band: from the scaled differences (DeltaIncs, MAT =
// false) or from the pair's precomputed block (MatIncs, MAT = true).
struct BandSource {
    const void *dX, *dY;  // differences (T), !MAT
    int64_t d;
    const void *mat;      // increment block (TM), MAT
    int64_t ld;
};

template <typename T, int R, int O, bool MAT, typename TM>
__device__ T ragged_band(const BandSource &bs, int64_t ncx, int64_t ncy, int order, T *stage, int stage_cap, int band,
                         bool last, const T *top_buf, const int *top_prog, T *bot_buf, int *bot_prog, int *error,
                         long long poll_limit)
{
    using BS = BlockShape<R, O>;
    const SolveGeom g = make_geom<R, O>(ncx, ncy, order);
    if constexpr (MAT) {
        MatIncs<T, BS::RC, TM> src;
        src.base = reinterpret_cast<const TM *>(bs.mat);
        src.ld = bs.ld;
        src.ncy = ncy;
        return band_solve<T, R, O>(g, src, band, last, top_buf, top_prog, bot_buf, bot_prog, error, 0,
                                   kProgressStride, poll_limit);
    } else {
        DeltaIncs<T, BS::RC> src;
        src.dX = reinterpret_cast<const T *>(bs.dX);
        src.dY = reinterpret_cast<const T *>(bs.dY);
        src.d = bs.d;
        src.ncy = ncy;
        src.dxs = ((int64_t)BS::RC * bs.d * 32 <= stage_cap) ? stage : nullptr;
        return band_solve<T, R, O>(g, src, band, last, top_buf, top_prog, bot_buf, bot_prog, error, 0,
                                   kProgressStride, poll_limit);
    }
}

template <typename T, int R, bool MAT, typename TM>
__device__ T ragged_band_by_o(const BandSource &bs, int64_t ncx, int64_t ncy, int order, T *stage, int stage_cap,
                              int band, bool last, const T *tb, const int *tp, T *bb, int *bp, int *error,
                              long long pl)
{
    switch (order) {
    case 0: return ragged_band<T, R, 0, MAT, TM>(bs, ncx, ncy, order, stage, stage_cap, band, last, tb, tp, bb, bp, error, pl);
    case 1: return ragged_band<T, R, 1, MAT, TM>(bs, ncx, ncy, order, stage, stage_cap, band, last, tb, tp, bb, bp, error, pl);
    case 2: return ragged_band<T, R, 2, MAT, TM>(bs, ncx, ncy, order, stage, stage_cap, band, last, tb, tp, bb, bp, error, pl);
    case 3: return ragged_band<T, R, 3, MAT, TM>(bs, ncx, ncy, order, stage, stage_cap, band, last, tb, tp, bb, bp, error, pl);
    default:
        return ragged_band<T, R, 4, MAT, TM>(bs, ncx, ncy, order, stage, stage_cap, band, last, tb, tp, bb, bp, error, pl);
    }
}

template <typename T, typename TIN, bool MAT, typename TM = float>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) ragged_kernel(RaggedParams p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    T *stage = reinterpret_cast<T *>(smem_raw) + (int64_t)wib * p.stage_elems_per_warp;
    const T *dxp = reinterpret_cast<const T *>(p.dx_pack);
    const T *dyp = reinterpret_cast<const T *>(p.dy_pack);
    T *pool = reinterpret_cast<T *>(p.pool);
    TIN *out = reinterpret_cast<TIN *>(p.out);
    const int64_t d = p.d;
    const TIN nan = TIN(__longlong_as_double(0x7ff8000000000000LL));

    while (true) {
        unsigned long long it_ = 0;
        if (lane == 0) it_ = atomicAdd(p.counter, 1ull);
        it_ = __shfl_sync(kFullMask, it_, 0);
        if (it_ >= (unsigned long long)p.nitems) break;
        const int64_t it = (int64_t)it_;
        const int64_t b = p.item_pair[it];
        const int band = p.item_band[it];
        if (b < 0 || b >= p.npairs) { // cannot even name a pair: release any consumer and skip
            if (lane == 0) {
                atomicOr(p.error, kErrInvalidItem);
                st_release(p.progress + it, 0x7fffffff);
            }
            continue;
        }
        const int order = p.order[b];
        const int R = p.pair_rows[b];
        const int nb = p.pair_bands[b];
        int64_t lx = p.x_len[b], ly = p.y_len[b];
        const T *X = MAT ? nullptr : dxp + (p.x_off[b] - b) * d;
        const T *Y = MAT ? nullptr : dyp + (p.y_off[b] - b) * d;
        if (lx > ly) { // shorter path on the rows
            const T *t = X;
            X = Y;
            Y = t;
            const int64_t u = lx;
            lx = ly;
            ly = u;
        }
        const int64_t ncx = lx - 1, ncy = ly - 1;
        // Validate the item before touching memory: order range first (it bounds the shifts),
        // then the shape, the plan (rows, band count, band order) and the boundary pool extent.
        bool ok = order >= 0 && order <= 12 && ncx >= 1 && (R == 2 || R == 4 || R == 8 || R == 16);
        int64_t n = 0, m = 0;
        if (ok) {
            n = ncx << order;
            m = ncy << order;
            ok = nb == (int)((n + 32 * R - 1) / (32 * R)) && band >= 0 && band < nb &&
                 p.pair_bnd_off[b] >= 0 && p.pair_bnd_off[b] + (int64_t)(nb - 1) * (m + 1) <= p.bnd_elems &&
                 m + 1 <= 0x7fffffff;
            if (ok && band > 0) ok = it >= 1 && p.item_pair[it - 1] == b && p.item_band[it - 1] == band - 1;
            if (ok && MAT) { // the pair's increment block lies inside the matrix and is 16-byte aligned
                const int64_t o = p.inc_off[b], ldb = (ncx + 3) & ~3LL;
                ok = o >= 0 && (o & 3) == 0 && o + ncy * ldb <= p.inc_elems && *p.tc_err == 0;
            }
        }
        if (!ok) {
            if (lane == 0) {
                atomicOr(p.error, (MAT && *p.tc_err) ? kErrWaitTimeout : kErrInvalidItem);
                out[b] = nan;
                st_release(p.progress + it, 0x7fffffff); // the band below sees the sentinel and yields NaN
            }
            continue;
        }
        const bool last = band == nb - 1;
        T *base = pool + p.pair_bnd_off[b];
        const T *tb = band > 0 ? base + (int64_t)(band - 1) * (m + 1) : nullptr;
        const int *tp = band > 0 ? p.progress + it - 1 : nullptr;
        T *bb = last ? nullptr : base + (int64_t)band * (m + 1);
        int *bp = p.progress + it;
        BandSource bs;
        bs.dX = X;
        bs.dY = Y;
        bs.d = d;
        bs.mat = MAT ? reinterpret_cast<const TM *>(p.inc) + p.inc_off[b] : nullptr;
        bs.ld = (ncx + 3) & ~3LL;
        const int cap = p.stage_elems_per_warp;
        T v;
        switch (R) {
        case 2: v = ragged_band_by_o<T, 2, MAT, TM>(bs, ncx, ncy, order, stage, cap, band, last, tb, tp, bb, bp, p.error, p.poll_limit); break;
        case 4: v = ragged_band_by_o<T, 4, MAT, TM>(bs, ncx, ncy, order, stage, cap, band, last, tb, tp, bb, bp, p.error, p.poll_limit); break;
        case 8: v = ragged_band_by_o<T, 8, MAT, TM>(bs, ncx, ncy, order, stage, cap, band, last, tb, tp, bb, bp, p.error, p.poll_limit); break;
        default: v = ragged_band_by_o<T, 16, MAT, TM>(bs, ncx, ncy, order, stage, cap, band, last, tb, tp, bb, bp, p.error, p.poll_limit); break;
        }
        if (last && lane == 0) out[b] = TIN(v);
    }
}

} // namespace sigk
