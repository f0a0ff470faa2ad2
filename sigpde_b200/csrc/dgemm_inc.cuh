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

// The same entries for d <= KD (16 or 32), pipelined: a CTA stages its A
// tile (64 x-rows by d) once and walks the n tiles blockIdx.y,
// blockIdx.y + gridDim.y, ... (for kTcLower only those below the diagonal, a
// prefix of the walk); the next n tile's B values are loaded into registers
// while the current tile is computed and stored, and B is double-buffered in
// shared memory with one barrier per tile.  dgemm_inc_kernel stages, waits,
// computes and stores each tile in turn (one tile per CTA), so its loads are
// never overlapped with its own math.  Summation order and results are those
// of dgemm_inc_kernel.
template <int KD>
__global__ void __launch_bounds__(256, 3) dgemm_inc_pipe_kernel(DgemmIncParams p)
{
    constexpr int TILE = kDgTile;
    constexpr int LPT = KD * TILE / 256; // B (and A) values a thread stages per tile
    extern __shared__ __align__(16) double dg_smem[];
    double(*As)[TILE + 1] = reinterpret_cast<double(*)[TILE + 1]>(dg_smem);
    double(*Bs)[KD][TILE + 1] = reinterpret_cast<double(*)[KD][TILE + 1]>(dg_smem + KD * (TILE + 1));
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int mm = threadIdx.x & (TILE - 1), kq = threadIdx.x / TILE;
    const int64_t m0 = (int64_t)blockIdx.x * TILE;
    const int64_t n_rows = p.npaths_y * p.ncy;
    const int kd = (int)p.d;
    int64_t n_end = n_rows;
    if (p.mode == kTcLower) { // tiles with n0 / ncy > i_hi + x0 lie above the diagonal of path pairs
        int64_t i_hi = (m0 + TILE - 1) / p.rows_x;
        if (i_hi >= p.npaths_x) i_hi = p.npaths_x - 1;
        const int64_t lim = (i_hi + p.x0 + 1) * p.ncy;
        if (lim < n_end) n_end = lim;
    }
    const int64_t step = (int64_t)gridDim.y * TILE;
    int64_t n0 = (int64_t)blockIdx.y * TILE;
    if (n0 >= n_end) return; // uniform across the CTA, before any barrier
    {
        const int64_t m = m0 + mm;
        const int64_t px = m / p.rows_x, cx = m - px * p.rows_x;
        const bool a_ok = px < p.npaths_x && cx < p.ncx;
        const double *a_src = p.dx + (a_ok ? px * p.d * p.ncx + cx : 0);
#pragma unroll
        for (int r = 0; r < LPT; ++r) {
            const int kk = kq + r * (256 / TILE);
            As[kk][mm] = (a_ok && kk < kd) ? a_src[kk * p.ncx] : 0.0;
        }
    }
    double bv[LPT];
    auto load_b = [&](int64_t nb) {
        const int64_t n = nb + mm;
        const int64_t qy = n / p.ncy, cy = n - qy * p.ncy;
        const bool b_ok = n < n_rows;
        const double *b_src = p.dy + (b_ok ? qy * p.d * p.ncy + cy : 0);
#pragma unroll
        for (int r = 0; r < LPT; ++r) {
            const int kk = kq + r * (256 / TILE);
            bv[r] = 0.0;
            if (b_ok && kk < kd) bv[r] = b_src[kk * p.ncy];
        }
    };
    load_b(n0);
    int buf = 0;
    for (; n0 < n_end; n0 += step) {
#pragma unroll
        for (int r = 0; r < LPT; ++r) Bs[buf][kq + r * (256 / TILE)][mm] = bv[r];
        __syncthreads(); // this tile's B (and, the first time, A) is visible; the other buffer is free
        if (n0 + step < n_end) load_b(n0 + step);
        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
        for (int kk = 0; kk < kd; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
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
        buf ^= 1;
    }
}

constexpr size_t dgemm_pipe_smem_bytes(int kd) { return (size_t)3 * kd * (kDgTile + 1) * sizeof(double); }

// ------------------------------------------------------------------ uneven batches
// Float64 increments of an uneven batch from the tensor-core plan's tables
// (fp64 cells with d >= 16): the pairs' scaled differences as float64 row
// images, [image row][k], with the same rows and scalings as the tensor-core
// operand images (row path on side 0 with the static scale and 4^-order),
// then one FP64 GEMM over the plan's 128 x 256 tiles in 64 x 64 pieces.
template <typename TIN>
__global__ void ragged_image64_kernel(TcRaggedImageParams p, double *img)
{
    for (int64_t b = blockIdx.y; b < p.npairs; b += gridDim.y) {
        const int64_t lx = p.x_len[b], ly = p.y_len[b];
        const bool use_y = (p.side == 0) == (lx > ly);
        const TIN *pack = reinterpret_cast<const TIN *>(use_y ? p.y_pack : p.x_pack);
        const TIN *sc = reinterpret_cast<const TIN *>(use_y ? p.sy : p.sx);
        const int64_t off = use_y ? p.y_off[b] : p.x_off[b];
        const int64_t nc = (use_y ? ly : lx) - 1;
        const int ord = p.order[b];
        const int64_t r0 = p.row0[b];
        const int64_t rows8 = (nc + 7) & ~7LL;
        // a pair the plan cannot hold is skipped; the wavefront refuses it too
        if (nc < 1 || ord < 0 || ord > 12 || r0 < 0 || (r0 & 7) != 0 || r0 + rows8 > p.rows_alloc) continue;
        double g = sc ? (double)sc[b] : 1.0;
        if (p.side == 0) g *= p.f * ldexp(1.0, -2 * ord);
        const TIN *xp0 = pack + off * p.d;
        double *out = img + r0 * p.d;
        const int64_t total = rows8 * p.d;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
             e += (int64_t)gridDim.x * blockDim.x) {
            const int64_t c = e / p.d, k = e - c * p.d;
            double v = 0.0;
            if (c < nc) {
                const TIN *xp = xp0 + c * p.d + k;
                v = ((double)xp[p.d] - (double)xp[0]) * g;
            }
            out[e] = v;
        }
    }
}

struct RaggedDgemmParams {
    const double *a, *b;   // row images [row][d]
    int64_t a_rows, b_rows, d;
    const int64_t *tiles;  // ntiles x (a_row, b_row, m_valid, n_valid, out_off, ld), the tensor-core plan's
    int64_t ntiles;
    double *out;
    int64_t out_elems;
    unsigned *err;         // set when a tile lies outside the buffers (that tile is skipped)
};

template <int TILE = kDgTile>
__global__ void __launch_bounds__(256, 3) ragged_dgemm_kernel(RaggedDgemmParams p)
{
    static_assert(TILE == 64, "4x4 outputs per thread of a 16x16 block");
    __shared__ double As[kDgK][TILE + 1];
    __shared__ double Bs[kDgK][TILE + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t nsub = p.ntiles * 8; // 2 x 4 pieces of 64 x 64 per 128 x 256 tile
    for (int64_t w = blockIdx.x; w < nsub; w += gridDim.x) {
        const int64_t t = w >> 3;
        const int mi = (int)(w & 7) >> 2, nj = (int)(w & 3);
        const int64_t *te = p.tiles + t * 6;
        const int64_t a_row = te[0], b_row = te[1], m_valid = te[2], n_valid = te[3], out_off = te[4], ld = te[5];
        const int64_t m0 = (int64_t)mi * TILE, n0 = (int64_t)nj * TILE;
        // rows to store: the pair's rows rounded up to 4 (its own zero padding), within this piece
        const int64_t m_store = ((m_valid + 3) & ~3LL);
        if (m0 >= m_store || n0 >= n_valid) continue; // uniform across the CTA
        const bool ok = a_row >= 0 && b_row >= 0 && a_row + m_store <= p.a_rows &&
                        b_row + n_valid <= p.b_rows && out_off >= 0 && ld >= m_store &&
                        out_off + (n_valid - 1) * ld + m_store <= p.out_elems;
        if (!ok) {
            if (threadIdx.x == 0) atomicExch(p.err, 1u);
            continue;
        }
        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
        for (int64_t k0 = 0; k0 < p.d; k0 += kDgK) {
            // stage A[k][m] and B[k][n]: consecutive threads read consecutive k of one image row
            for (int e = threadIdx.x; e < kDgK * TILE; e += 256) {
                const int mm = e / kDgK, kk = e - mm * kDgK;
                const int64_t k = k0 + kk;
                const int64_t m = m0 + mm, n = n0 + mm;
                As[kk][mm] = (k < p.d && m < m_store) ? p.a[(a_row + m) * p.d + k] : 0.0;
                Bs[kk][mm] = (k < p.d && n < n_valid) ? p.b[(b_row + n) * p.d + k] : 0.0;
            }
            __syncthreads();
            const int kn = (int)((p.d - k0) < kDgK ? (p.d - k0) : kDgK);
            for (int kk = 0; kk < kn; ++kk) {
                double a[4], bb[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
                for (int j = 0; j < 4; ++j) bb[j] = Bs[kk][ty + 16 * j];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t n = n0 + ty + 16 * j;
            if (n >= n_valid) continue;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t m = m0 + tx + 16 * i;
                if (m < m_store) p.out[out_off + n * ld + m] = acc[i][j];
            }
        }
    }
}

// ragged_dgemm_kernel for d <= KD (16 or 32), pipelined: the unit of work is
// the half-tile (tile t, A block mi) whose 4 pieces share their 64 A rows.
// The CTA stages those rows (all of K) once and walks the half-tile's pieces,
// loading the next piece's B rows into registers during the current piece's
// FMAs and stores (B single-buffered in shared memory, two barriers a piece,
// so that KD = 32 stays within 48 KB of static shared memory).  Summation
// order, stored rows and error reporting are those of ragged_dgemm_kernel.
template <int KD>
__global__ void __launch_bounds__(256, 3) ragged_dgemm_pipe_kernel(RaggedDgemmParams p)
{
    constexpr int TILE = kDgTile;
    constexpr int LPT = KD * TILE / 256; // values a thread stages per block of A or B
    __shared__ double As[KD][TILE + 1];
    __shared__ double Bs[KD][TILE + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int kd = (int)p.d;
    const int64_t nunits = p.ntiles * 2;
    double bv[LPT];
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int64_t t = u >> 1;
        const int mi = (int)(u & 1);
        const int64_t *te = p.tiles + t * 6;
        const int64_t a_row = te[0], b_row = te[1], m_valid = te[2], n_valid = te[3], out_off = te[4], ld = te[5];
        const int64_t m0 = (int64_t)mi * TILE;
        const int64_t m_store = ((m_valid + 3) & ~3LL);
        if (m0 >= m_store || n_valid <= 0) continue; // uniform across the CTA
        const bool ok = a_row >= 0 && b_row >= 0 && a_row + m_store <= p.a_rows &&
                        b_row + n_valid <= p.b_rows && out_off >= 0 && ld >= m_store &&
                        out_off + (n_valid - 1) * ld + m_store <= p.out_elems;
        if (!ok) {
            if (threadIdx.x == 0) atomicExch(p.err, 1u);
            continue;
        }
        int npieces = (int)((n_valid + TILE - 1) / TILE);
        if (npieces > 4) npieces = 4;
        auto load_b = [&](int nj) {
            const int64_t n0 = (int64_t)nj * TILE;
#pragma unroll
            for (int r = 0; r < LPT; ++r) {
                const int e = threadIdx.x + r * 256;
                const int mm = e / KD, kk = e - mm * KD;
                const int64_t n = n0 + mm;
                bv[r] = 0.0;
                if (kk < kd && n < n_valid) bv[r] = p.b[(b_row + n) * p.d + kk];
            }
        };
        __syncthreads(); // the previous unit's reads of As and Bs are done
#pragma unroll
        for (int r = 0; r < LPT; ++r) {
            const int e = threadIdx.x + r * 256;
            const int mm = e / KD, kk = e - mm * KD;
            const int64_t m = m0 + mm;
            As[kk][mm] = (kk < kd && m < m_store) ? p.a[(a_row + m) * p.d + kk] : 0.0;
        }
        load_b(0);
        for (int nj = 0; nj < npieces; ++nj) {
            if (nj > 0) __syncthreads(); // the previous piece's reads of Bs are done
#pragma unroll
            for (int r = 0; r < LPT; ++r) {
                const int e = threadIdx.x + r * 256;
                const int mm = e / KD, kk = e - mm * KD;
                Bs[kk][mm] = bv[r];
            }
            __syncthreads(); // this piece's B (and the unit's A) is visible
            if (nj + 1 < npieces) load_b(nj + 1);
            double acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
            for (int kk = 0; kk < kd; ++kk) {
                double a[4], bb[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
                for (int j = 0; j < 4; ++j) bb[j] = Bs[kk][ty + 16 * j];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
            }
            const int64_t n0 = (int64_t)nj * TILE;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = n0 + ty + 16 * j;
                if (n >= n_valid) continue;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int64_t m = m0 + tx + 16 * i;
                    if (m < m_store) p.out[out_off + n * ld + m] = acc[i][j];
                }
            }
        }
    }
}

} // namespace sigk
