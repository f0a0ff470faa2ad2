// Backward pass: gradients of sum_pairs w * k(x, y) with respect to the path
// points, for the linear static kernel with float64 cells.  The reference has
// no backward pass (its Numba kernels end autograd); this is the adjoint of
// the same scheme (sigpde/cuda_device_functions.py:3-5).
//
// With c the scaled coarse increment of a cell, A(c) = 1 + c/2 + c^2/12 and
// B(c) = 1 - c^2/12, the forward scheme is
//   K(p,q) = (K(p,q-1) + K(p-1,q)) A - K(p-1,q-1) B.
// Its adjoint Lambda = w dk/dK(p,q) satisfies, in reverse order,
//   Lambda(p,q) = P(p,q+1) + P(p+1,q) - Q(p+1,q+1),   Lambda(n,m) = w,
// where each node carries P = A Lambda and Q = B Lambda with the coefficients
// of the cell that produced it (absent nodes carry 0), and
//   dk/dc of a coarse cell = sum over its fine cells of Lambda(p,q) D(p,q),
//   D(p,q) = (K(p,q-1) + K(p-1,q)) A'(c) - K(p-1,q-1) B'(c),
//   A'(c) = 1/2 + c/6,  B'(c) = -c/6.
//
// Kernels
//   grad_fwd_kernel  one warp per pair: the forward wavefront (R rows a lane,
//                    one fine column a step, bands of 32R rows) storing the
//                    top input of every lane step and each lane's rows at the
//                    start of every segment of T = 32/R steps;
//   grad_bwd_kernel  one warp per pair: per segment (last first), each lane
//                    recomputes its rows' K and D over the segment on its own
//                    (no cross-lane dependency: its inputs were stored), then
//                    the adjoint runs the same schedule in reverse for
//                    Lambda, summing Lambda D per coarse cell; each coarse
//                    cell's rows belong to one lane (R >= 2^order), so the
//                    sum is written once, over the cell's increment in the
//                    increment matrix (which then holds dk/dc);
//   grad_gx_kernel / grad_gy_kernel   contractions of dk/dc with the scaled
//                    differences of the other side: the gradients with
//                    respect to the coarse differences;
//   grad_points_kernel   differences of those: gradients at the points.
#pragma once

#include "dgemm_inc.cuh"

namespace sigk {

struct GradParams {
    int op;               // kOpPairwise / kOpGram
    double *mat;          // increments in, dk/dc out; Gram: [n * ld + m], pairwise: per-pair blocks
    int64_t ld;           // Gram: npaths_x(chunk) * rows_x; pairwise: rows_x
    int64_t rows_x;
    int64_t ncx, ncy;
    int order;
    int64_t nitems;       // pairs in this chunk
    int64_t ny;           // Gram: y paths
    const void *w;        // weights (grad_out): pairwise (n,), Gram (n_x, n_y) row-major; input dtype
    int in64;
    int64_t x0;           // first x path of the chunk
    double *dbuf;         // per pair and band grad_band_doubles(m, R): top inputs and segment checkpoints
    double *bnd;          // per pair 2 * (m + 2) doubles: band boundary rows
};

// pair `it` of the chunk: its x path (global), y path, and its increment block
__device__ __forceinline__ void grad_item(const GradParams &p, int64_t it, int64_t &xi, int64_t &yj, double *&base,
                                          int64_t &row_ld)
{
    if (p.op == kOpPairwise) {
        xi = p.x0 + it;
        yj = xi;
        base = p.mat + it * p.ncy * p.rows_x;
        row_ld = p.rows_x;
    } else {
        const int64_t il = it / p.ny;
        xi = p.x0 + il;
        yj = it - il * p.ny;
        base = p.mat + yj * p.ncy * p.ld + il * p.rows_x;
        row_ld = p.ld;
    }
}

// Steps per recompute segment: T * R = 32 doubles of D per lane in shared memory.
template <int R>
constexpr int grad_seg() { return 32 / R; }

// Per pair and band, the forward pass stores what the adjoint needs to
// recompute any segment of T steps lane by lane: the top input K(p0-1, q)
// each lane used at every step ([step][lane]) and each lane's K(rows, q-1)
// at the start of every segment ([segment][row][lane]).
__host__ __device__ __forceinline__ int64_t grad_band_doubles(int m, int R)
{
    const int64_t S = m + 31, T = 32 / R, NS = (S + T - 1) / T;
    return S * 32 + NS * R * 32;
}

// Coefficients of the lane's coarse rows for coarse column cj.
template <int RC>
__device__ __forceinline__ void grad_coefs(const double *base, int64_t row_ld, int ci0, int64_t ncx, int cj,
                                           double (&A)[RC], double (&B)[RC], double (&Ad)[RC], double (&Bd)[RC])
{
#pragma unroll
    for (int rc = 0; rc < RC; ++rc) {
        const int ci = ci0 + rc;
        const double c = ci < ncx ? base[(int64_t)cj * row_ld + ci] : 0.0;
        stencil_coefs(c, A[rc], B[rc]);
        Ad[rc] = fma(c, 1.0 / 6.0, 0.5);
        Bd[rc] = c * (-1.0 / 6.0);
    }
}

// One forward step of the lane's R rows at a column: left holds K(rows, q-1)
// and becomes K(rows, q); D of each row goes to d[r * 32].  Rows beyond n
// (coarse rows >= ncx, c = 0) copy row n and carry Lambda = 0 in the adjoint:
// they need no masking.
template <int R, int O, bool WANT_D>
__device__ __forceinline__ void grad_lane_step(double (&left)[R], double top, double diag, const double *A,
                                               const double *B, const double *Ad, const double *Bd, double *d)
{
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int rc = r >> O;
        const double sum = left[r] + top;
        const double k = sum * A[rc] - diag * B[rc];
        if constexpr (WANT_D) d[r * 32] = sum * Ad[rc] - diag * Bd[rc];
        diag = left[r];
        left[r] = k;
        top = k;
    }
}

template <int R, int O>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) grad_fwd_kernel(GradParams p)
{
    static_assert(R >= (1 << O), "a lane's rows hold whole coarse rows");
    constexpr int RC = R >> O;
    constexpr int T = grad_seg<R>();
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int n = (int)(p.ncx << p.order), m = (int)(p.ncy << p.order);
    const int nb = (n + 32 * R - 1) / (32 * R);
    const int S = m + 31;
    const int64_t band_doubles = grad_band_doubles(m, R);
    for (int64_t it = gwarp; it < p.nitems; it += nwarps) {
        int64_t xi, yj, row_ld;
        double *base;
        grad_item(p, it, xi, yj, base, row_ld);
        double *bnd = p.bnd + it * 2 * (int64_t)(m + 2); // K of the row above the band, columns 0..m
        for (int b = 0; b < nb; ++b) {
            double *tops = p.dbuf + (it * nb + b) * band_doubles + lane;
            double *ck = tops + (int64_t)S * 32;
            const int p0 = b * 32 * R + lane * R + 1; // this lane's first fine row (1-based)
            const int ci0 = (p0 - 1) >> O;            // its first coarse row
            double left[R];
#pragma unroll
            for (int r = 0; r < R; ++r) left[r] = 1.0; // K(p, 0)
            double bot = 1.0, corner = 1.0;            // lane l-1's last row at q-1 (as received), at q-2
            double A[RC], B[RC], Ad[RC], Bd[RC];
            __syncwarp();
            for (int s = 0; s < S; ++s) {
                const double from_above = __shfl_up_sync(0xffffffffu, bot, 1);
                if (s % T == 0) {
#pragma unroll
                    for (int r = 0; r < R; ++r) ck[((int64_t)(s / T) * R + r) * 32] = left[r];
                }
                const int q = s - lane + 1;
                double top = 1.0;
                if (q >= 1 && q <= m) {
                    double diag;
                    if (lane == 0) {
                        top = b == 0 ? 1.0 : bnd[q];
                        diag = b == 0 ? 1.0 : bnd[q - 1];
                    } else {
                        top = from_above;
                        diag = q == 1 ? 1.0 : corner;
                    }
                    if (((q - 1) & ((1 << O) - 1)) == 0) // a new coarse column
                        grad_coefs<RC>(base, row_ld, ci0, p.ncx, (q - 1) >> O, A, B, Ad, Bd);
                    grad_lane_step<R, O, false>(left, top, diag, A, B, Ad, Bd, nullptr);
                    if (lane == 31 && b + 1 < nb) bnd[q] = left[R - 1];
                    corner = from_above;
                    bot = left[R - 1];
                }
                tops[(int64_t)s * 32] = top;
            }
            __syncwarp();
            if (lane == 31 && b + 1 < nb) bnd[0] = 1.0;
            __syncwarp();
        }
    }
}

template <int R, int O>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) grad_bwd_kernel(GradParams p)
{
    static_assert(R >= (1 << O), "a lane's rows hold whole coarse rows");
    constexpr int RC = R >> O;
    constexpr int T = grad_seg<R>();
    __shared__ double dsm[kWarpsPerBlock][T][R][32]; // D of the current segment, per lane
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int n = (int)(p.ncx << p.order), m = (int)(p.ncy << p.order);
    const int nb = (n + 32 * R - 1) / (32 * R);
    const int S = m + 31, NS = (S + T - 1) / T;
    const int64_t band_doubles = grad_band_doubles(m, R);
    double *dl = &dsm[threadIdx.x >> 5][0][0][lane];
    for (int64_t it = gwarp; it < p.nitems; it += nwarps) {
        int64_t xi, yj, row_ld;
        double *base;
        grad_item(p, it, xi, yj, base, row_ld);
        const int64_t widx = p.op == kOpPairwise ? xi : xi * p.ny + yj;
        const double w = p.in64 ? reinterpret_cast<const double *>(p.w)[widx]
                                : (double)reinterpret_cast<const float *>(p.w)[widx];
        double *bP = p.bnd + it * 2 * (int64_t)(m + 2); // P and Q of the row below the band, columns 0..m+1
        double *bQ = bP + (m + 2);
        for (int b = nb - 1; b >= 0; --b) {
            const double *tops = p.dbuf + (it * nb + b) * band_doubles + lane;
            const double *ck = tops + (int64_t)S * 32;
            const int p0 = b * 32 * R + lane * R + 1;
            const int ci0 = (p0 - 1) >> O;
            double Pr[R], Qr[R]; // P, Q of the lane's rows at column q + 1
            // the seed Lambda(n, m) = w enters as the right neighbour of row n at column m
            const int rseed = n - p0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                Pr[r] = r == rseed ? w : 0.0;
                Qr[r] = 0.0;
            }
            double g[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) g[rc] = 0.0;
            double topP = 0.0, topQ = 0.0; // this lane's row 0 P, Q at its last column (published)
            double belowQ_prev = 0.0;      // lane l+1's row 0 Q at column q + 1
            double A[RC], B[RC], Ad[RC], Bd[RC];
            __syncwarp();
            for (int k = NS - 1; k >= 0; --k) {
                const int s0 = k * T;
                // phase A: recompute this segment's steps lane by lane from the checkpoint and the
                // stored top inputs, keeping D in shared memory
                {
                    double left[R], tp[T + 1];
#pragma unroll
                    for (int r = 0; r < R; ++r) left[r] = ck[((int64_t)k * R + r) * 32];
#pragma unroll
                    for (int t = 0; t <= T; ++t) {
                        const int st = s0 - 1 + t;
                        tp[t] = (st >= 0 && st < S) ? tops[(int64_t)st * 32] : 1.0;
                    }
                    bool have = false;
#pragma unroll
                    for (int t = 0; t < T; ++t) {
                        const int q = s0 + t - lane + 1;
                        if (q >= 1 && q <= m) {
                            if (!have || ((q - 1) & ((1 << O) - 1)) == 0)
                                grad_coefs<RC>(base, row_ld, ci0, p.ncx, (q - 1) >> O, A, B, Ad, Bd);
                            have = true;
                            grad_lane_step<R, O, true>(left, tp[t + 1], q == 1 ? 1.0 : tp[t], A, B, Ad, Bd,
                                                       dl + t * R * 32);
                        }
                    }
                }
                // phase B: the adjoint over the same steps in reverse
                bool have = false;
#pragma unroll 1
                for (int t = T - 1; t >= 0; --t) {
                    const int s = s0 + t;
                    if (s >= S) continue; // uniform: the last segment may be short
                    const double belowP = __shfl_down_sync(0xffffffffu, topP, 1);
                    const double belowQ = __shfl_down_sync(0xffffffffu, topQ, 1);
                    const int q = s - lane + 1;
                    if (q >= 1 && q <= m) {
                        double dP, dQ; // P(p+1, q) and Q(p+1, q+1) for the lane's last row
                        if (lane == 31) {
                            const bool last = b + 1 >= nb;
                            dP = last ? 0.0 : bP[q];
                            dQ = last ? 0.0 : bQ[q + 1];
                        } else {
                            dP = belowP;
                            dQ = q == m ? 0.0 : belowQ_prev;
                        }
                        const int cj = (q - 1) >> O;
                        if (!have || q == m || (q & ((1 << O) - 1)) == 0)
                            grad_coefs<RC>(base, row_ld, ci0, p.ncx, cj, A, B, Ad, Bd);
                        have = true;
                        const double *dq = dl + t * R * 32;
#pragma unroll
                        for (int r = R - 1; r >= 0; --r) {
                            const int rc = r >> O;
                            const double lam = Pr[r] + dP - dQ;
                            g[rc] = fma(lam, dq[r * 32], g[rc]);
                            const double P = A[rc] * lam, Q = B[rc] * lam;
                            dQ = Qr[r]; // Q(p, q+1) is the diagonal of the row above
                            dP = P;
                            Pr[r] = P;
                            Qr[r] = Q;
                        }
                        topP = Pr[0];
                        topQ = Qr[0];
                        if (lane == 0 && b > 0) {
                            bP[q] = Pr[0];
                            bQ[q] = Qr[0];
                        }
                        if (((q - 1) & ((1 << O) - 1)) == 0) { // leaving the coarse column: dk/dc is complete
#pragma unroll
                            for (int rc = 0; rc < RC; ++rc) {
                                const int ci = ci0 + rc;
                                if (ci < p.ncx) base[(int64_t)cj * row_ld + ci] = g[rc];
                                g[rc] = 0.0;
                            }
                        }
                    }
                    belowQ_prev = belowQ;
                }
            }
            __syncwarp();
            if (lane == 0 && b > 0) {
                bP[m + 1] = 0.0;
                bQ[m + 1] = 0.0;
            }
            __syncwarp();
        }
    }
}

// Increments of pairwise pairs (x path = y path = x0 + item) in per-pair
// blocks [item][cj][ci] (ci < rows_x; rows ci >= ncx are 0), summed as
// fma(dx_k, dy_k, acc) for k = 0 .. d-1 from zero like the other producers.
template <int V = 0> // instantiated once, in kernels_grad.cu
__global__ void grad_pair_inc_kernel(const double *dx, const double *dy, int64_t nitems, int64_t x0, int64_t ncx,
                                     int64_t ncy, int64_t rows_x, int64_t d, double *out)
{
    const int64_t total = nitems * ncy * rows_x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t item = e / (ncy * rows_x), r = e - item * ncy * rows_x;
        const int64_t cj = r / rows_x, ci = r - cj * rows_x;
        double acc = 0.0;
        if (ci < ncx) {
            const double *a = dx + (x0 + item) * d * ncx + ci;
            const double *b = dy + (x0 + item) * d * ncy + cj;
            for (int64_t k = 0; k < d; ++k) acc = fma(a[k * ncx], b[k * ncy], acc);
        }
        out[e] = acc;
    }
}

// Caller's increments (npairs, ncx, ncy) with element strides, times the
// pair's scales, into per-pair blocks [item][cj][ci] (rows ci >= ncx are 0);
// with `back`, the reverse: out = block * scales written with the strides.
template <int V = 0> // instantiated once, in kernels_grad.cu
__global__ void grad_inc_blocks_kernel(const void *inc, int in64, int64_t s0, int64_t s1, int64_t s2, int64_t nitems,
                                       int64_t b0, int64_t ncx, int64_t ncy, int64_t rows_x, const void *sx,
                                       const void *sy, double *blocks, void *out, int back)
{
    const int64_t total = nitems * ncy * rows_x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t item = e / (ncy * rows_x), r = e - item * ncy * rows_x;
        const int64_t cj = r / rows_x, ci = r - cj * rows_x;
        const int64_t b = b0 + item;
        double sc = 1.0;
        if (sx) sc *= in64 ? reinterpret_cast<const double *>(sx)[b] : (double)reinterpret_cast<const float *>(sx)[b];
        if (sy) sc *= in64 ? reinterpret_cast<const double *>(sy)[b] : (double)reinterpret_cast<const float *>(sy)[b];
        const int64_t off = b * s0 + ci * s1 + cj * s2;
        if (!back) {
            double v = 0.0;
            if (ci < ncx)
                v = in64 ? reinterpret_cast<const double *>(inc)[off] : (double)reinterpret_cast<const float *>(inc)[off];
            blocks[e] = v * sc;
        } else if (ci < ncx) {
            const double v = blocks[e] * sc;
            if (in64)
                reinterpret_cast<double *>(out)[off] = v;
            else
                reinterpret_cast<float *>(out)[off] = (float)v;
        }
    }
}

// Gradients with respect to the x side's scaled-difference rows: for each
// matrix row m (x path il, cell ci), part[slice][m][k] = sum over the slice's
// y cells n paired with it (Gram: all of them; pairwise: its own pair's) of
// G[n][m] * dyt[n][k].  grad_reduce_kernel adds the slices in order.
// dxt / dyt are the scaled differences in row layout (one row of d values per
// cell; x rows padded to rows_x per path with zeros), so that the inner loops
// index them directly.
struct GradContractParams {
    int op;
    const double *mat;     // dk/dc
    int64_t ld, rows_x, ncx, ncy;
    int64_t nrows_m;       // Gram: ld; pairwise: nitems * rows_x
    int64_t ncols_n;       // Gram: ny * ncy; pairwise: ncy (per pair)
    const double *dxt;     // x differences, rows m of the chunk: [m][k]
    const double *dyt;     // y differences, all y cells: [y path * ncy + cj][k]
    int64_t d;
    double *part;          // gx: [slice][nrows_m][d] partial sums
    int64_t slice;         // columns per slice
    double *gdy;           // gy: (ny, ncy, d) accumulated (+=) over chunks
    int64_t x0;
};

// Row layout of scaled differences: dst[(path * rows + r) * d + k] =
// src[(path * d + k) * nc + r] for r < nc, 0 for nc <= r < rows.
template <int V = 0> // instantiated once, in kernels_grad.cu
__global__ void grad_rows_kernel(const double *src, int64_t npaths, int64_t nc, int64_t rows, int64_t d, double *dst)
{
    const int64_t total = npaths * rows * d;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t path = e / (rows * d), rem = e - path * rows * d, r = rem / d, k = rem - r * d;
        dst[e] = r < nc ? src[(path * d + k) * nc + r] : 0.0;
    }
}

template <int V = 0> // instantiated once, in kernels_grad.cu
__global__ void grad_gx_kernel(GradContractParams p)
{
    const int64_t mm = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (mm >= p.nrows_m) return;
    const int64_t n0 = (int64_t)blockIdx.y * p.slice;
    const int64_t n1 = n0 + p.slice < p.ncols_n ? n0 + p.slice : p.ncols_n;
    const double *col;     // G[n][mm] = col[n * stride]
    int64_t stride;
    const double *dyt;     // dyt[n * d + k] for the n of this row
    if (p.op == kOpPairwise) {
        const int64_t item = mm / p.rows_x, ci = mm - item * p.rows_x;
        col = p.mat + item * p.ncy * p.rows_x + ci;
        stride = p.rows_x;
        dyt = p.dyt + (p.x0 + item) * p.ncy * p.d; // the pair's own y path
    } else {
        col = p.mat + mm;
        stride = p.ld;
        dyt = p.dyt;
    }
    double *out = p.part + ((int64_t)blockIdx.y * p.nrows_m + mm) * p.d;
    for (int64_t k0 = 0; k0 < p.d; k0 += 8) {
        double acc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = 0.0;
        const double *yk = dyt + k0;
        for (int64_t n = n0; n < n1; ++n) {
            const double gv = col[n * stride];
            const double *yn = yk + n * p.d;
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (k0 + k < p.d) acc[k] = fma(gv, yn[k], acc[k]);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (k0 + k < p.d) out[k0 + k] = acc[k];
    }
}

// gy: one warp per y cell n (Gram: n = y path * ncy + cj over all y paths;
// pairwise: n = pair * ncy + cj), lanes over the x cells paired with it.
template <int V = 0> // instantiated once, in kernels_grad.cu
__global__ void grad_gy_kernel(GradContractParams p)
{
    const int lane = threadIdx.x & 31;
    const int64_t n = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nrows = p.op == kOpPairwise ? (p.nrows_m / p.rows_x) * p.ncy : p.ncols_n;
    if (n >= nrows) return;
    const double *row;
    const double *xt;
    int64_t mlen, yrow;
    if (p.op == kOpPairwise) {
        const int64_t item = n / p.ncy, cj = n - item * p.ncy;
        row = p.mat + item * p.ncy * p.rows_x + cj * p.rows_x;
        mlen = p.rows_x;
        xt = p.dxt + item * p.rows_x * p.d;
        yrow = (p.x0 + item) * p.ncy + cj;
    } else {
        row = p.mat + n * p.ld;
        mlen = p.ld;
        xt = p.dxt;
        yrow = n;
    }
    for (int64_t k0 = 0; k0 < p.d; k0 += 8) {
        double acc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = 0.0;
        for (int64_t mm = lane; mm < mlen; mm += 32) {
            const double gv = row[mm]; // padding rows hold 0, as do their differences
            const double *xm = xt + mm * p.d + k0;
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (k0 + k < p.d) acc[k] = fma(gv, xm[k], acc[k]);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            double v = acc[k];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if (lane == 0 && k0 + k < p.d) p.gdy[yrow * p.d + k0 + k] += v;
        }
    }
}

// gy for the Gram: gdy[n][k] += sum_m G[n][m] dxt[m][k], a tall-skinny GEMM
// (rows n: all y cells, m: the chunk's x cells, k < d).  A CTA owns 32 rows
// and k-chunks of up to 32; m goes in tiles of 64 staged in shared memory
// (G rows coalesced along m; dxt transposed to [k][m] with a padded stride so
// that the 8 k-groups of a warp hit different banks).  Each (n, k) has one
// owner thread, so the sum over chunks stays in order.
constexpr int kGyRows = 32, kGyTile = 64, kGyK = 32;

template <int V = 0> // instantiated once, in kernels_grad.cu
__global__ void __launch_bounds__(256) grad_gy_gram_kernel(GradContractParams p)
{
    __shared__ double gs[kGyRows][kGyTile + 1];
    __shared__ double xs[kGyK][kGyTile + 1];
    const int tid = threadIdx.x;
    const int row = tid >> 3, kg = tid & 7; // 32 rows x 8 k-groups; k = kg + 8 j
    const int64_t n0 = (int64_t)blockIdx.x * kGyRows;
    const int64_t nrows = p.ncols_n;
    for (int64_t k0 = 0; k0 < p.d; k0 += kGyK) {
        const int kn = (int)((p.d - k0) < kGyK ? (p.d - k0) : kGyK);
        double acc[kGyK / 8];
#pragma unroll
        for (int j = 0; j < kGyK / 8; ++j) acc[j] = 0.0;
        for (int64_t m0 = 0; m0 < p.ld; m0 += kGyTile) {
            __syncthreads();
            for (int e = tid; e < kGyRows * kGyTile; e += 256) {
                const int r = e / kGyTile, mm = e - r * kGyTile;
                const int64_t n = n0 + r, m = m0 + mm;
                gs[r][mm] = (n < nrows && m < p.ld) ? p.mat[n * p.ld + m] : 0.0;
            }
            for (int e = tid; e < kGyTile * kn; e += 256) {
                const int mm = e / kn, k = e - mm * kn;
                const int64_t m = m0 + mm;
                xs[k][mm] = m < p.ld ? p.dxt[m * p.d + k0 + k] : 0.0;
            }
            __syncthreads();
#pragma unroll 4
            for (int mm = 0; mm < kGyTile; ++mm) {
                const double gv = gs[row][mm];
#pragma unroll
                for (int j = 0; j < kGyK / 8; ++j)
                    if (kg + 8 * j < kn) acc[j] = fma(gv, xs[kg + 8 * j][mm], acc[j]);
            }
        }
        const int64_t n = n0 + row;
        if (n < nrows) {
#pragma unroll
            for (int j = 0; j < kGyK / 8; ++j)
                if (kg + 8 * j < kn) p.gdy[n * p.d + k0 + kg + 8 * j] += acc[j];
        }
    }
}

// gdx[(x0 + il) * ncx + ci][k] = sum over slices of part (rows ci < ncx).
template <int V = 0> // instantiated once, in kernels_grad.cu
__global__ void grad_reduce_kernel(const double *part, int64_t nslices, int64_t nrows_m, int64_t rows_x, int64_t ncx,
                                   int64_t d, int64_t x0, double *gdx)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nrows_m * d) return;
    const int64_t mm = e / d, k = e - mm * d;
    const int64_t il = mm / rows_x, ci = mm - il * rows_x;
    if (ci >= ncx) return;
    double s = 0.0;
    for (int64_t sl = 0; sl < nslices; ++sl) s += part[(sl * nrows_m + mm) * d + k];
    gdx[((x0 + il) * ncx + ci) * d + k] = s;
}

// grad at the points: g[path][t][k] = scale(path) * (gd[t-1][k] - gd[t][k]),
// gd of the path's coarse differences (ncells = len - 1), in the output dtype.
template <int V = 0> // instantiated once, in kernels_grad.cu
__global__ void grad_points_kernel(const double *gd, int64_t npaths, int64_t len, int64_t d, double f,
                                   const void *sc, int in64, void *out)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= npaths * len * d) return;
    const int64_t pth = e / (len * d), r = e - pth * len * d, t = r / d, k = r - t * d;
    const int64_t nc = len - 1;
    const double *g = gd + pth * nc * d;
    const double a = t >= 1 ? g[(t - 1) * d + k] : 0.0;
    const double b = t < nc ? g[t * d + k] : 0.0;
    const double s = sc ? (in64 ? reinterpret_cast<const double *>(sc)[pth]
                                : (double)reinterpret_cast<const float *>(sc)[pth]) : 1.0;
    const double v = (a - b) * f * s;
    if (in64)
        reinterpret_cast<double *>(out)[e] = v;
    else
        reinterpret_cast<float *>(out)[e] = (float)v;
}

} // namespace sigk
