// Robust normalisation with one CTA per path: the path's refined grid is cut
// into bands of 32 R rows, one warp per band, and the warps solve it as a
// pipeline (the warp on band w reads band w-1's bottom row as it is published,
// ragged.cuh's band_solve).  Every Chandrupatla iteration re-solves the whole
// grid this way, so a path's ~10 sequential solves each take about one
// band's time plus the pipeline fill instead of all bands in sequence on one
// warp: the latency of a robust request shrinks with its path length.
//
// The bracket arithmetic (normalize_path) runs in every thread on the value
// the last band returns, shared through shared memory, so all threads take the
// same branches and the CTA-wide barriers stay uniform.
#pragma once

#include "ragged.cuh"

namespace sigk {

constexpr int kNormPipeMaxWarps = 16;
constexpr int kNormPipeStride = 4; // column blocks between band publications (the bands of a CTA are close)

template <typename TIN, int R, int O, int MODE>
__global__ void __launch_bounds__(kNormPipeMaxWarps * 32) normalize_pipe_kernel(NormParams p)
{
    using T = double;
    using BS = BlockShape<R, O>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_val;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5; // bands of every path
    const SolveGeom g = make_geom<R, O>(p.nc, p.nc, p.order);
    T *bnd = reinterpret_cast<T *>(p.bnd) + (int64_t)blockIdx.x * (nw - 1) * p.bnd_stride;
    int *prog = p.prog + (int64_t)blockIdx.x * kNormPipeMaxWarps;
    TIN *lam_out = reinterpret_cast<TIN *>(p.lam);
    int solves = 0; // solves done by this CTA: progress values continue across them

    for (int64_t b = blockIdx.x; b < p.n; b += gridDim.x) {
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
            dsrc.dxs = p.stage_smem ? reinterpret_cast<T *>(smem_raw) + (int64_t)w * BS::RC * p.d * 32 : nullptr;
        } else {
            // the path's coarse increment tile, built once by the whole CTA: tile[cj][ci] = <dx_ci, dx_cj>
            T *tile = reinterpret_cast<T *>(smem_raw);
            const double *dxb = p.dx + b * p.d * p.nc;
            for (int64_t e = threadIdx.x; e < p.nc * p.nc; e += blockDim.x) {
                const int64_t cj = e / p.nc;
                const int64_t ci = e - cj * p.nc;
                T acc = T(0);
                for (int64_t k = 0; k < p.d; ++k) acc = fma(dxb[k * p.nc + ci], dxb[k * p.nc + cj], acc);
                tile[cj * p.tile_pitch + ci] = acc;
            }
            __syncthreads();
            tsrc.tile = tile;
            tsrc.pitch = p.tile_pitch;
        }
        auto solve = [&](double scale) -> double {
            const int base = solves * (int)(g.nsteps + 1);
            ++solves;
            const T *tb = w > 0 ? bnd + (int64_t)(w - 1) * p.bnd_stride : nullptr;
            const int *tp = w > 0 ? prog + (w - 1) : nullptr;
            T *bb = w < nw - 1 ? bnd + (int64_t)w * p.bnd_stride : nullptr;
            T v;
            if constexpr (MODE == kNormGiven) {
                gsrc.fscale = p.fscale * scale;
                v = band_solve<T, R, O>(g, gsrc, w, w == nw - 1, tb, tp, bb, prog + w, p.err, base, kNormPipeStride);
            } else if constexpr (MODE == kNormDelta) {
                dsrc.fscale = p.fscale * scale;
                v = band_solve<T, R, O>(g, dsrc, w, w == nw - 1, tb, tp, bb, prog + w, p.err, base, kNormPipeStride);
            } else {
                tsrc.fscale = p.fscale * scale;
                v = band_solve<T, R, O>(g, tsrc, w, w == nw - 1, tb, tp, bb, prog + w, p.err, base, kNormPipeStride);
            }
            if (w == nw - 1 && lane == 0) s_val = v;
            __syncthreads(); // every band is done; the last one's value is in s_val
            const double r = s_val;
            __syncthreads(); // s_val and the band rows are free for the next solve
            return r;
        };
        double out = 0.0;
        int it = 0;
        normalize_path(p, b, threadIdx.x == 0, solve, out, it);
        if (threadIdx.x == 0) {
            if (lam_out) lam_out[b] = TIN(out);
            if (p.iters) p.iters[b] = it;
        }
        __syncthreads(); // the tile / staging area is free for the next path
    }
}

} // namespace sigk
