// fused_tc.cuh -- tensor-core increments consumed on chip by the streaming
// wavefront: no increment matrix in HBM.
//
// The two-phase tensor-core path (tc.cuh) writes the coarse increments
// <dx_ci, dy_cj> of every Gram pair to HBM (4.26 GB at 256 x 256, L = 128) and
// a streaming wavefront reads them back.  Here one CTA does both.
//
//   * 4 wavefront warps each stream their own run of pairs: the CTA walks
//     groups (x_{4a..4a+3}, y_j), warp w takes (x_{4a+w}, y_j), so the four
//     pairs of a group share the y path (the MMA's B operand);
//   * warp 4 stages operands with cp.async.bulk and issues, every 16 steps (a
//     "chunk" of 16 coarse columns), split-TF32 tcgen05.mma into one of 4 TMEM
//     chunk slots: RC tiles of M = 128 rows, N = 16, where the A operand is
//     permuted so that TMEM lane 32 w + i of tile k holds coarse row RC i + k of
//     warp w's x path -- exactly the rows that wavefront lane i of warp w owns;
//   * so each warp finds ITS pair's increments in ITS TMEM lane quarter: at a
//     chunk boundary it reads them (tcgen05.ld) and writes them into its own
//     shared-memory ring, skewed (lane i runs i steps behind lane 0, so it
//     gets the columns of its next 16 steps, [16k - i, 16k - i + 16)), one
//     16-byte store per slot; lanes then read slot (step mod 32): 16 slots
//     being read, 16 written;
//   * no barrier couples the warps: they wait for the MMA of a chunk on an
//     mbarrier, and tell the producer that they are done with old chunks on
//     another; a lane lags lane 0 by up to 31 steps, so a boundary reads chunks
//     k-2, k-1 and k, and TMEM holds 4 chunk slots (256 columns, 2 CTAs per SM).
//
// The arithmetic is that of the two-phase path exactly: the same MMAs (lo*hi,
// hi*lo, hi*hi per K step, float32 accumulation) for each increment and the
// same float64 cells (stencil_coefs / stream_block), so the results are
// bitwise those of tc_gemm_kernel + stream_inc_kernel.
//
// Scope: Gram (x != y), tc64 (float64 cells), dyadic order <= 3, dim <= 16,
// x paths of at most 128 coarse cells in one band with R >= 2^order rows a
// lane (RC = R >> order coarse rows, at most 4).  Every wait is bounded: a wait
// that runs out sets the error word and the CTA's entries become NaN.
#pragma once

#include "tc.cuh"

namespace sigk {

constexpr int kFtWarps = 4;         // wavefront warps per CTA: one per TMEM lane quarter
constexpr int kFtChunk = 16;        // steps per MMA chunk (the MMA's N)
constexpr int kFtTmemSlots = 4;     // chunk slots in TMEM: k-2, k-1, k read at boundary k; k+1 in flight
constexpr int kFtSlotCols = 64;     // TMEM columns per chunk slot: RC <= 4 tiles of 16 columns
constexpr uint32_t kFtTmemCols = kFtTmemSlots * kFtSlotCols; // 256
constexpr int kFtRingSlots = 32;    // ring slots per lane row: 16 read, 16 written
constexpr int kFtBSlots = 4;        // B stages: chunk k + 2 is staged while chunks k, k + 1 wait for their MMAs
constexpr size_t kFtMinSmem = 80 * 1024; // at most two CTAs per SM (their 2 x 256 TMEM columns fit)

struct FusedTcParams {
    const float *a_hi, *a_lo; // A image: blocks of 4 x paths, RC tiles of 128 rows each (tc_image quad layout)
    const float *b_hi, *b_lo; // B image: T rows per y path (rows >= ncy zero)
    int64_t nx, ny;
    int ncx, ncy;
    int kp;                   // dimension padded to a multiple of 8
    int T;                    // time slots per pair: ncy rounded up to a multiple of kFtChunk
    int64_t ngroups;          // ceil(nx / 4) * ny; group g = (x block g / ny, y path g % ny)
    int64_t per_cta;          // groups per CTA (a contiguous run)
    int in64;                 // output float64 (else float32)
    void *out;
    int64_t out_ld;
    unsigned *err;            // set to 1 when a bounded wait ran out (those entries are NaN)
};

struct FtSmem {
    uint32_t ring, a, b, bars, misc, total;
};

__host__ __device__ __forceinline__ uint32_t ft_align(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

// Shared memory: 4 rings (32 slots x 32 RC rows of floats), one A block (RC
// tiles, hi and lo), kFtBSlots B slots (16 rows, hi and lo), mbarriers (a,
// b[kFtBSlots], mma[2], done[2]), the TMEM address and an error flag.
__host__ __device__ __forceinline__ FtSmem ft_smem_layout(int rc, int kp)
{
    FtSmem s{};
    s.ring = 0;
    s.a = ft_align((uint32_t)kFtWarps * kFtRingSlots * 32 * rc * 4, 1024);
    s.b = s.a + 2u * (uint32_t)rc * kTcM * kp * 4;
    s.bars = s.b + (uint32_t)kFtBSlots * 2u * (uint32_t)kFtChunk * kp * 4;
    s.misc = s.bars + (5 + kFtBSlots) * 8;
    s.total = s.misc + 16;
    return s;
}

__host__ __forceinline__ size_t fused_tc_smem(int rc, int kp)
{
    const size_t s = ft_smem_layout(rc, kp).total;
    return s < kFtMinSmem ? kFtMinSmem : s;
}

// Producer (lane 0 of warp 4): operand staging and MMA issue for one CTA's run.
struct FtProducer {
    const FusedTcParams *p;
    int64_t g0;          // first group of the run
    int rc;              // tiles per A block (coarse rows a lane)
    uint32_t a_base, b_base, bar_a, bar_b, bar_mma, tmem;
    uint32_t tile_bytes, b_bytes; // one 128-row A tile (hi or lo); one 16-row B slot (hi or lo)
    int a_phase = 0;     // stagings of the A block so far

    __device__ __forceinline__ int64_t group_of(int64_t k) const { return (k * kFtChunk) / p->T; }
    __device__ __forceinline__ int64_t block_of(int64_t k) const { return (g0 + group_of(k)) / p->ny; }

    // the A block (4 x paths) of x block a
    __device__ __forceinline__ void stage_a(int64_t a)
    {
        const uint32_t bytes = (uint32_t)rc * tile_bytes;
        const int64_t off = a * rc * kTcM * p->kp;
        mbar_expect_tx(bar_a, 2 * bytes);
        bulk_g2s(a_base, p->a_hi + off, bytes, bar_a);
        bulk_g2s(a_base + bytes, p->a_lo + off, bytes, bar_a);
        ++a_phase;
    }

    // the y path's 16 rows of chunk k into B slot k % kFtBSlots
    __device__ __forceinline__ void stage_b(int64_t k) const
    {
        const int64_t t0 = k * kFtChunk;
        const int64_t j = (g0 + t0 / p->T) % p->ny;
        const int64_t row = j * p->T + t0 % p->T;
        const uint32_t slot = (uint32_t)(k % kFtBSlots), bar = bar_b + 8 * slot;
        const uint32_t dst = b_base + slot * 2 * b_bytes;
        mbar_expect_tx(bar, 2 * b_bytes);
        bulk_g2s(dst, p->b_hi + row * p->kp, b_bytes, bar);
        bulk_g2s(dst + b_bytes, p->b_lo + row * p->kp, b_bytes, bar);
    }

    // chunk k: wait for its operands, then per A tile 3 split products per K step into TMEM slot k % 4
    __device__ __forceinline__ bool issue(int64_t k) const
    {
        const uint32_t sb = (uint32_t)(k % kFtBSlots);
        if (!mbar_wait(bar_a, (uint32_t)((a_phase - 1) & 1))) return false;
        if (!mbar_wait(bar_b + 8 * sb, (uint32_t)((k / kFtBSlots) & 1))) return false;
        tc_fence_after();
        const uint32_t sbo = (uint32_t)p->kp * 32; // bytes between 8-row groups
        const uint32_t idesc = tf32_idesc(kTcM, kFtChunk);
        const uint32_t bhi = b_base + sb * 2 * b_bytes, blo = bhi + b_bytes;
        const uint32_t a_lo_base = a_base + (uint32_t)rc * tile_bytes;
        for (int t = 0; t < rc; ++t) {
            const uint32_t d = tmem + (uint32_t)((k % kFtTmemSlots) * kFtSlotCols + t * kFtChunk);
            const uint32_t ahi = a_base + (uint32_t)t * tile_bytes, alo = a_lo_base + (uint32_t)t * tile_bytes;
            for (int ks = 0; ks < p->kp / 8; ++ks) {
                const uint32_t ko = (uint32_t)ks * 256; // two 128-byte K chunks per step
                mma_tf32(d, smem_desc(alo + ko, 128, sbo), smem_desc(bhi + ko, 128, sbo), idesc, ks > 0 ? 1u : 0u);
                mma_tf32(d, smem_desc(ahi + ko, 128, sbo), smem_desc(blo + ko, 128, sbo), idesc, 1u);
                mma_tf32(d, smem_desc(ahi + ko, 128, sbo), smem_desc(bhi + ko, 128, sbo), idesc, 1u);
            }
        }
        mma_commit(bar_mma + 8 * (uint32_t)(k & 1));
        return true;
    }
};

// A lane's RC coarse increments from its ring slot, and its RC values of one
// chunk column into a ring slot (16-, 8- or 4-byte accesses).
template <int RC>
__device__ __forceinline__ void ft_ring_read(const float *src, double (&c)[RC])
{
    if constexpr (RC == 4) {
        const float4 v = *reinterpret_cast<const float4 *>(src);
        c[0] = v.x;
        c[1] = v.y;
        c[2] = v.z;
        c[3] = v.w;
    } else if constexpr (RC == 2) {
        const float2 v = *reinterpret_cast<const float2 *>(src);
        c[0] = v.x;
        c[1] = v.y;
    } else {
        c[0] = src[0];
    }
}

template <int RC>
__device__ __forceinline__ void ft_ring_write(float *dst, const float (&v)[kFtSlotCols], int c)
{
    if constexpr (RC == 4)
        *reinterpret_cast<float4 *>(dst) = make_float4(v[c], v[16 + c], v[32 + c], v[48 + c]);
    else if constexpr (RC == 2)
        *reinterpret_cast<float2 *>(dst) = make_float2(v[c], v[16 + c]);
    else
        dst[0] = v[c];
}

// Warps 0..3 run the wavefront (and, at each chunk boundary, move their pair's
// increments from their TMEM lane quarter into their ring); warp 4 stages the
// operands and issues the MMAs.
template <int R, int O>
__global__ void __launch_bounds__((kFtWarps + 1) * 32, 2) fused_tc_kernel(FusedTcParams p)
{
    using T = double;
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    static_assert(O <= 3 && (R >> O) == RC && RC <= 4, "one coarse column a step, whole coarse rows a lane");
    constexpr int kRows = 32 * RC; // ring rows: the coarse rows of one pair's band
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t g0 = (int64_t)blockIdx.x * p.per_cta;
    if (g0 >= p.ngroups) return; // CTA-uniform, before anything is allocated
    const int64_t ng = (p.ngroups - g0) < p.per_cta ? (p.ngroups - g0) : p.per_cta;
    const int Tp = p.T;
    const int64_t nlocal = ng * Tp;            // time slots of each warp's run
    const int64_t nchunks = nlocal / kFtChunk; // T is a multiple of kFtChunk
    const int64_t S = nlocal + 31;             // steps: lane 31 runs 31 behind lane 0
    const int64_t nbound = (S + kFtChunk - 1) / kFtChunk;

    const FtSmem L = ft_smem_layout(RC, p.kp);
    const uint32_t sbase = smem_u32(smem);
    float *ring = reinterpret_cast<float *>(smem + L.ring);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L.misc);
    volatile int *cta_err = reinterpret_cast<volatile int *>(smem + L.misc + 4);
    const uint32_t bar_a = sbase + L.bars, bar_b = bar_a + 8, bar_mma = bar_b + 8 * kFtBSlots, bar_done = bar_mma + 16;
    const bool producer = warp == kFtWarps;

    if (producer) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kFtTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        if (lane == 0) {
            for (int i = 0; i < 3 + kFtBSlots; ++i) mbar_init(bar_a + 8 * i, 1); // a, b[], mma[2]
            mbar_init(bar_done, kFtWarps);
            mbar_init(bar_done + 8, kFtWarps);
            *cta_err = 0;
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (producer) {
        if (lane == 0) {
            // -------------------------------------------------------- operands and MMAs
            FtProducer prod;
            prod.p = &p;
            prod.g0 = g0;
            prod.rc = RC;
            prod.a_base = sbase + L.a;
            prod.b_base = sbase + L.b;
            prod.bar_a = bar_a;
            prod.bar_b = bar_b;
            prod.bar_mma = bar_mma;
            prod.tmem = tmem;
            prod.tile_bytes = (uint32_t)kTcM * p.kp * 4;
            prod.b_bytes = (uint32_t)kFtChunk * p.kp * 4;
            int64_t issued = -1, staged_b = -1;
            bool ok = true;
            prod.stage_a(prod.block_of(0));
            for (int64_t k = 0; k < 2 && k < nchunks; ++k) {
                prod.stage_b(k);
                staged_b = k;
            }
            for (int64_t k = 0; ok && k < nchunks; ++k) {
                if (k >= 2) {
                    // TMEM slot k % 4 held chunk k - 4, last read at boundary k - 2: every warp must be past it
                    if (!mbar_wait(bar_done + 8 * (uint32_t)((k - 2) & 1), (uint32_t)(((k - 2) >> 1) & 1))) {
                        ok = false;
                        break;
                    }
                    // B slot (k + 2) % 4 held chunk k - 2, whose MMAs must be done.  Waited before chunk k's
                    // MMAs are committed to the same mbarrier, so the phase cannot be mistaken for k's.
                    if (!mbar_wait(bar_mma + 8 * (uint32_t)(k & 1), (uint32_t)(((k - 2) >> 1) & 1))) {
                        ok = false;
                        break;
                    }
                }
                if (k + 2 < nchunks) { // slots 2, 3 are fresh; later ones held chunk k - 2 (done above)
                    prod.stage_b(k + 2);
                    staged_b = k + 2;
                }
                if (k >= 1 && prod.block_of(k) != prod.block_of(k - 1)) {
                    // a new A block: the MMAs of chunk k - 1, the last to read the old one, must be done
                    if (!mbar_wait(bar_mma + 8 * (uint32_t)((k - 1) & 1), (uint32_t)(((k - 1) >> 1) & 1))) {
                        ok = false;
                        break;
                    }
                    prod.stage_a(prod.block_of(k));
                }
                if (!prod.issue(k)) {
                    ok = false;
                    break;
                }
                issued = k;
                if (*cta_err) ok = false; // a consumer gave up a wait
            }
            if (!ok) {
                *cta_err = 1;
                // let the copies and MMAs started here land (bounded) before the CTA exits
                for (int64_t k = (staged_b > 2 ? staged_b - 2 : 0); k <= staged_b; ++k)
                    mbar_wait(bar_b + 8 * (uint32_t)(k % kFtBSlots), (uint32_t)((k / kFtBSlots) & 1));
                mbar_wait(bar_a, (uint32_t)((prod.a_phase - 1) & 1));
                if (issued >= 0) mbar_wait(bar_mma + 8 * (uint32_t)(issued & 1), (uint32_t)((issued >> 1) & 1));
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------ the wavefront (stream_inc_kernel's cells)
        // Lane `lane` of this warp reads TMEM lane 32 warp + lane: in tile k, coarse row RC lane + k of this
        // warp's x path, i.e. its own rows as a wavefront lane.
        float *myring = ring + (size_t)warp * kFtRingSlots * kRows;
        float *myrow = myring + RC * lane;

        auto boundary = [&](int64_t kb) {
            if (kb < nchunks && !*cta_err) {
                if (!mbar_wait(bar_mma + 8 * (uint32_t)(kb & 1), (uint32_t)((kb >> 1) & 1))) *cta_err = 1;
            }
            tc_fence_after();
            // tcgen05.ld is warp-collective: decide for the whole warp (another thread may set the flag)
            const bool werr = __any_sync(kFullMask, *cta_err != 0);
            if (!werr) {
#pragma unroll 1
                for (int64_t a = kb - 2; a <= kb; ++a) {
                    if (a < 0 || a >= nchunks) continue;
                    float v[kFtSlotCols];
                    const uint32_t col = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((a % kFtTmemSlots) * kFtSlotCols);
                    tmem_ld32(col, *reinterpret_cast<float(*)[32]>(v));
                    if constexpr (RC > 2) tmem_ld32(col + 32, *reinterpret_cast<float(*)[32]>(v + 32));
                    // time 16a + c of this lane belongs to its step 16a + c + lane; the steps after this boundary
                    // are [16kb, 16kb + 16), whose ring half nobody reads now
                    const int base = (int)(16 * (a - kb)) + lane;
#pragma unroll
                    for (int c = 0; c < kFtChunk; ++c) {
                        const int j = base + c;
                        if ((unsigned)j < (unsigned)kFtChunk)
                            ft_ring_write<RC>(myrow + (size_t)((int)((16 * kb + j) & (kFtRingSlots - 1)) * kRows), v, c);
                    }
                }
            }
            __syncwarp();
            tc_fence_before();
            if (lane == 0) mbar_arrive(bar_done + 8 * (uint32_t)(kb & 1)); // done with TMEM chunk kb - 2
        };

        StreamParams sp{};
        sp.op = kOpGram;
        sp.in64 = p.in64;
        sp.ny = p.ny;
        sp.out = p.out;
        sp.out_ld = p.out_ld;
        const int ncy = p.ncy;
        const int n = p.ncx << O;
        const int lstar = (n - 1) / R, rstar = (n - 1) % R;
        const float *rd = myring + RC * lane;
        T left[R];
#pragma unroll
        for (int i = 0; i < R; ++i) left[i] = T(1);
        T bot[C];
#pragma unroll
        for (int c = 0; c < C; ++c) bot[c] = T(1);
        T corner_next = T(1);
        int col = 0;
        int64_t grp = 0, xi = 0, yj = 0;
        for (int64_t kb = 0; kb < nbound; ++kb) {
            boundary(kb);
            const int64_t s1 = (kb + 1) * kFtChunk < S ? (kb + 1) * kFtChunk : S;
            for (int64_t s = kb * kFtChunk; s < s1; ++s) {
                T top[C];
#pragma unroll
                for (int c = 0; c < C; ++c) top[c] = __shfl_up_sync(kFullMask, bot[c], 1);
                if (lane == 0) {
#pragma unroll
                    for (int c = 0; c < C; ++c) top[c] = T(1);
                }
                const int64_t u = s - lane;
                if (u >= 0 && u < nlocal) {
                    if (col == 0) {
                        const int64_t g = g0 + grp;
                        xi = kFtWarps * (g / p.ny) + warp;
                        yj = g % p.ny;
#pragma unroll
                        for (int i = 0; i < R; ++i) left[i] = T(1);
                    }
                    if (col < ncy) {
                        const T corner = (col == 0) ? T(1) : corner_next;
                        corner_next = top[C - 1];
                        T cv[RC];
                        ft_ring_read<RC>(rd + (size_t)(s & (kFtRingSlots - 1)) * kRows, cv);
                        T A[RC], B[RC];
#pragma unroll
                        for (int rc = 0; rc < RC; ++rc) stencil_coefs(cv[rc], A[rc], B[rc]);
                        stream_block<T, R, O>(left, top, corner, A, B, bot);
                        if (col == ncy - 1 && lane == lstar && xi < p.nx)
                            stream_store(sp, 0, xi, yj, pick_row(left, rstar));
                    }
                    if (++col == Tp) {
                        col = 0;
                        ++grp;
                    }
                }
            }
        }
    }

    // ---------------------------------------------------------------- teardown
    __syncthreads();
    if (*cta_err) { // the CTA's entries are incomplete: NaN, and the launch's error word
        StreamParams sp{};
        sp.op = kOpGram;
        sp.in64 = p.in64;
        sp.ny = p.ny;
        sp.out = p.out;
        sp.out_ld = p.out_ld;
        if (tid == 0) atomicOr(p.err, 1u);
        for (int64_t e = tid; e < ng * kFtWarps; e += blockDim.x) {
            const int64_t g = g0 + e / kFtWarps, i = kFtWarps * (g / p.ny) + e % kFtWarps;
            if (i < p.nx) stream_store(sp, 0, i, g % p.ny, T(__longlong_as_double(0x7ff8000000000000LL)));
        }
    }
    if (producer) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kFtTmemCols) : "memory");
    }
}

} // namespace sigk
