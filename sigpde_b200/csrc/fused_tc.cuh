// fused_tc.cuh -- tensor-core increments consumed on chip by a two-entry
// streaming wavefront: no increment matrix in HBM.
//
// The two-phase tensor-core path (tc.cuh) writes the coarse increments
// <dx_ci, dy_cj> of every Gram pair to HBM (4.26 GB at 256 x 256, L = 128) and
// a streaming wavefront reads them back.  Here one CTA per SM does both.
//
// Work: the CTA walks a contiguous run of groups; group g = (x block a, y pair
// b) holds the 16 entries (x_{8a+4h+q}, y_{2b+r}), h, r in {0, 1}, q in 0..3.
// Warp w = 4h + q streams x_{8a+4h+q} against y_{2b} and y_{2b+1} at once,
// each cell operation an independent float64 pair (stream_reg_dual_kernel's
// cells, minus the dot products): 8 warps, 16 pair streams per SM.
//
// Skew halves.  Lane l of a wavefront runs l steps behind lane 0, so within
// 16 steps its 32 lanes need increments from a 47-column window of times.
// Chunks of 16 times come from split-TF32 tcgen05.mma (M = 128, N = 16) into
// TMEM; holding that window for every stream would take 4 chunk slots.  So
// each chunk k is two MMA families: LO, against the y rows of times
// [16k, 16k + 16), for wavefront lanes 0..15, and HI, against times
// [16k - 16, 16k), for lanes 16..31.  Within each half the skew is at most 15
// steps, so the 16 steps after a chunk boundary read only 2 chunks: 2 TMEM
// slots.
//
// Lane sharing.  A 32x32b TMEM load gives thread t of warp w lane
// 32 (w % 4) + t.  Set h = 0 plays wavefront lane t on thread t, set h = 1
// plays lane (t + 16) mod 32 (its shuffles rotate), so in every MMA row
// 32 q + t belongs to exactly one of the two warps of quarter q:
//     LO rows: t < 16 -> set 0, lane t;       t >= 16 -> set 1, lane t - 16
//     HI rows: t >= 16 -> set 0, lane t;      t < 16 -> set 1, lane t + 16
// and both sets share the same columns.  TMEM: 2 slots x 2 y paths x
// {LO, HI} x RC tiles x 16 columns = 128 RC columns (512 at RC = 4).
//
// Every RING steps (16, or 8 where a wide dimension leaves shared memory for
// only 8 ring slots) the two warps of a quarter wait for the current chunk's
// MMAs and split the copy of it and the chunk before out of TMEM: set 0 loads
// the LO family, set 1 the HI family, and thread t writes lane 32 q + t into
// the shared-memory ring of the warp that owns the row, skewed so that slot
// s % RING holds what each thread needs at step s (one 16-byte store per
// slot, between two 64-thread barriers of the pair).  Then each warp arrives
// on a counter.  At the last boundary that reads chunk m - 1, the last of the
// 8 warps to arrive issues chunk m + 1's MMAs (into the slot of chunk m - 1)
// and stages the y rows of chunk m + 2: no producer warp, no block-wide
// barrier.  The A operand (the x block's rows) changes only where the run
// moves to another x block; there the HI MMAs of that chunk, which still read
// the old block, are completed before the new block is staged.
//
// The arithmetic is that of the two-phase path exactly: the same MMAs (lo*hi,
// hi*lo, hi*hi per K step, float32 accumulation) for each increment and the
// same float64 cells (stencil_coefs / stream_block), so the results are
// bitwise those of tc_gemm_kernel + stream_inc_kernel.
//
// Scope: Gram (x != y), tc64 (float64 cells), dyadic order <= 3, x paths of
// one band with R = RC 2^order rows a lane, RC <= 4, shared memory within the
// device limit (RING = 16: dimension <= 8 at RC = 4, <= 16 below; RING = 8:
// dimension <= 16 at RC = 4, <= 32 at RC <= 2).  Every wait is
// bounded: a wait that runs out sets the error word and the CTA's entries
// become NaN.
#pragma once

#include "tc.cuh"

namespace sigk {

constexpr int kFtWarps = 8;      // two sets of four wavefront warps (one per TMEM lane quarter)
constexpr int kFtChunk = 16;     // times per MMA chunk (the MMA's N)
constexpr int kFtBSlots = 4;     // y-row stages: chunks k - 1, k (MMA k), k + 1 (next MMA), k + 2 (staging)

struct FusedTcParams {
    const float *a_hi, *a_lo; // A image: per block of 8 x paths, 2 RC tiles of 128 rows (RC LO, then RC HI)
    const float *b_hi, *b_lo; // B image: T rows per y path (rows >= ncy zero)
    int64_t nx, ny;
    int ncx, ncy;
    int kp;                   // dimension padded to a multiple of 8
    int T;                    // time slots per pair: ncy rounded up to a multiple of kFtChunk
    int64_t hy;               // y pairs, ceil(ny / 2)
    int64_t ngroups;          // ceil(nx / 8) * hy; group g = (x block g / hy, y pair g % hy)
    int64_t per_cta;          // groups per CTA (a contiguous run)
    int in64;                 // output float64 (else float32)
    void *out;
    int64_t out_ld;
    unsigned *err;            // set to 1 when a bounded wait ran out (those entries are NaN)
};

__host__ __device__ constexpr uint32_t ft_tmem_cols(int rc) { return (uint32_t)(128 * rc); }

struct FtSmem {
    uint32_t ring, a, b, bars, misc, total;
};

__host__ __device__ __forceinline__ uint32_t ft_align(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

// Shared memory: the rings (per warp: `ring` slots x 2 y paths x 32 threads x
// RC floats), the A block (2 RC tiles, hi then lo), kFtBSlots y-row stages
// (2 y paths x {hi, lo} x 16 rows), mbarriers (a, aux, b[kFtBSlots], mma[2])
// and the issuers' shared state.
__host__ __device__ __forceinline__ FtSmem ft_smem_layout(int rc, int kp, int ring)
{
    FtSmem s{};
    s.ring = 0;
    s.a = ft_align((uint32_t)kFtWarps * ring * 2 * 32 * rc * 4, 1024);
    s.b = s.a + 2u * 2u * (uint32_t)rc * kTcM * kp * 4;
    s.bars = s.b + (uint32_t)kFtBSlots * 2u * 2u * (uint32_t)kFtChunk * kp * 4;
    s.misc = s.bars + (4 + kFtBSlots) * 8;
    s.total = s.misc + 64;
    return s;
}

__host__ __forceinline__ size_t fused_tc_smem(int rc, int kp, int ring) { return ft_smem_layout(rc, kp, ring).total; }

// State shared by the threads that take turns issuing (shared memory; each
// issuer acquires it through the arrival counter, see FtIssuer).
struct FtState {
    uint32_t tmem;       // TMEM base address
    int err;             // a wait ran out in this CTA
    uint32_t arrive;     // arrivals at boundaries so far
    uint32_t aux_pending; // an HI-only commit (x block change) is in flight
    int64_t a_block;     // x block held in the A stage
    uint32_t a_phase;    // completed stagings of A (mbarrier phases)
    uint32_t aux_phase;  // completed HI-only commits (x block changes)
    int64_t staged_b;    // last chunk whose y rows were staged
    int64_t issued;      // last chunk whose MMAs were committed
};
static_assert(sizeof(FtState) <= 64, "issuer state fits the misc area");

__device__ __forceinline__ uint32_t atomic_add_acq_rel(uint32_t addr, uint32_t v)
{
    uint32_t old;
    asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(addr), "r"(v) : "memory");
    return old;
}

// Operand staging and MMA issue for one CTA's run.  Executed by one thread at
// a time: thread 0 for the prologue, then at each boundary the last warp to
// arrive (its lane 0).
struct FtIssuer {
    const FusedTcParams *p;
    FtState *st;
    int64_t g0, nlocal, nchunks;
    int rc;
    uint32_t a_base, b_base, bar_a, bar_aux, bar_b, bar_mma, tmem;
    uint32_t tile_bytes, b_bytes; // one 128-row A tile (hi or lo); 16 y rows of one path (hi or lo)

    // the group of chunk k's first time (times past the run clamp to its last chunk)
    __device__ __forceinline__ int64_t group_of(int64_t k) const
    {
        const int64_t kk = k < nchunks ? k : nchunks - 1;
        return g0 + (kk * kFtChunk) / p->T;
    }
    __device__ __forceinline__ int64_t block_of(int64_t k) const { return group_of(k) / p->hy; }

    __device__ __forceinline__ bool fail() const
    {
        st->err = 1;
        return false;
    }

    // the A block (x paths 8a .. 8a + 7): 2 RC tiles, hi and lo
    __device__ __forceinline__ void stage_a(int64_t a) const
    {
        const uint32_t bytes = 2u * (uint32_t)rc * tile_bytes;
        const int64_t off = a * 2 * rc * kTcM * p->kp;
        mbar_expect_tx(bar_a, 2 * bytes);
        bulk_g2s(a_base, p->a_hi + off, bytes, bar_a);
        bulk_g2s(a_base + bytes, p->a_lo + off, bytes, bar_a);
        st->a_block = a;
    }

    // y rows of chunk k (both paths of the pair, hi and lo) into stage k % kFtBSlots
    __device__ __forceinline__ void stage_b(int64_t k) const
    {
        const int64_t kk = k < nchunks ? k : nchunks - 1;
        const int64_t t0 = kk * kFtChunk;
        const int64_t g = g0 + t0 / p->T;
        const int64_t y0 = 2 * (g % p->hy);
        const int64_t y1 = y0 + 1 < p->ny ? y0 + 1 : y0;
        const int64_t row = t0 % p->T;
        const uint32_t slot = (uint32_t)(k % kFtBSlots), bar = bar_b + 8 * slot;
        const uint32_t dst = b_base + slot * 4 * b_bytes;
        mbar_expect_tx(bar, 4 * b_bytes);
        bulk_g2s(dst, p->b_hi + (y0 * p->T + row) * p->kp, b_bytes, bar);
        bulk_g2s(dst + b_bytes, p->b_lo + (y0 * p->T + row) * p->kp, b_bytes, bar);
        bulk_g2s(dst + 2 * b_bytes, p->b_hi + (y1 * p->T + row) * p->kp, b_bytes, bar);
        bulk_g2s(dst + 3 * b_bytes, p->b_lo + (y1 * p->T + row) * p->kp, b_bytes, bar);
        st->staged_b = k;
    }

    __device__ __forceinline__ bool wait_b(int64_t k) const
    {
        return mbar_wait(bar_b + 8 * (uint32_t)(k % kFtBSlots), (uint32_t)((k / kFtBSlots) & 1));
    }

    // one family (LO: y rows of chunk k; HI: of chunk k - 1) of chunk k, both y paths, into TMEM slot k % 2
    __device__ __forceinline__ void mma_family(int64_t k, int hi) const
    {
        const int64_t kb = (hi && k > 0) ? k - 1 : k;
        const uint32_t sb = b_base + (uint32_t)(kb % kFtBSlots) * 4 * b_bytes;
        const uint32_t sbo = (uint32_t)p->kp * 32; // bytes between 8-row groups
        const uint32_t idesc = tf32_idesc(kTcM, kFtChunk);
        const uint32_t a_lo_base = a_base + 2u * (uint32_t)rc * tile_bytes;
        for (int r = 0; r < 2; ++r) {
            const uint32_t bhi = sb + 2u * r * b_bytes, blo = bhi + b_bytes;
            for (int t = 0; t < rc; ++t) {
                const uint32_t d = tmem + (uint32_t)((k & 1) * 64 * rc + r * 32 * rc + hi * 16 * rc + t * 16);
                const uint32_t tile = (uint32_t)(hi * rc + t);
                const uint32_t ahi = a_base + tile * tile_bytes, alo = a_lo_base + tile * tile_bytes;
                for (int ks = 0; ks < p->kp / 8; ++ks) {
                    const uint32_t ko = (uint32_t)ks * 256; // two 128-byte K chunks per step
                    mma_tf32(d, smem_desc(alo + ko, 128, sbo), smem_desc(bhi + ko, 128, sbo), idesc, ks > 0 ? 1u : 0u);
                    mma_tf32(d, smem_desc(ahi + ko, 128, sbo), smem_desc(blo + ko, 128, sbo), idesc, 1u);
                    mma_tf32(d, smem_desc(ahi + ko, 128, sbo), smem_desc(bhi + ko, 128, sbo), idesc, 1u);
                }
            }
        }
    }

    // chunk k's MMAs, committed to mma[k % 2]
    __device__ __forceinline__ bool issue(int64_t k) const
    {
        if (st->err) return false;
        if (!wait_b(k) || (k > 0 && !wait_b(k - 1))) return fail();
        if (!mbar_wait(bar_a, (st->a_phase - 1) & 1)) return fail();
        tc_fence_after();
        const int64_t blk = block_of(k);
        if (blk != st->a_block) {
            // the HI family still reads the old x block: complete it, then stage the new block
            mma_family(k, 1);
            st->aux_pending = 1;
            mma_commit(bar_aux);
            if (!mbar_wait(bar_aux, st->aux_phase & 1)) return fail();
            st->aux_pending = 0;
            ++st->aux_phase;
            stage_a(blk);
            ++st->a_phase;
            if (!mbar_wait(bar_a, (st->a_phase - 1) & 1)) return fail();
            tc_fence_after();
            mma_family(k, 0);
        } else {
            mma_family(k, 0);
            mma_family(k, 1);
        }
        mma_commit(bar_mma + 8 * (uint32_t)(k & 1));
        st->issued = k;
        return true;
    }
};

// A thread's RC increments of one y path from its ring slot, and its RC values
// of one chunk column into a ring slot (16-, 8- or 4-byte accesses).
template <int RC>
__device__ __forceinline__ void ft_ring_read(const float *src, float (&c)[RC])
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
__device__ __forceinline__ void ft_ring_write(float *dst, const float (&v)[RC][kFtChunk], int c)
{
    if constexpr (RC == 4)
        *reinterpret_cast<float4 *>(dst) = make_float4(v[0][c], v[1][c], v[2][c], v[3][c]);
    else if constexpr (RC == 2)
        *reinterpret_cast<float2 *>(dst) = make_float2(v[0][c], v[1][c]);
    else
        dst[0] = v[0][c];
}

template <int R, int O, int RING>
__global__ void __launch_bounds__(kFtWarps * 32, 1) fused_tc_kernel(FusedTcParams p)
{
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    static_assert(O <= 3 && (R >> O) == RC && RC <= 4, "one coarse column a step, whole coarse rows a lane");
    static_assert(RING == 16 || RING == 8, "a boundary every 16 or 8 steps");
    constexpr uint32_t kCols = ft_tmem_cols(RC);
    constexpr int kSlotF = 2 * 32 * RC; // floats per ring slot (2 y paths x 32 threads x RC)
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int h = warp >> 2, q = warp & 3;
    const int lam = h ? ((lane + 16) & 31) : lane; // the wavefront lane this thread plays
    const int ii = lam & 15;                       // its skew within its half
    const int64_t g0 = (int64_t)blockIdx.x * p.per_cta;
    if (g0 >= p.ngroups) return; // CTA-uniform, before anything is allocated
    const int64_t ng = (p.ngroups - g0) < p.per_cta ? (p.ngroups - g0) : p.per_cta;
    const int Tp = p.T;
    const int64_t nlocal = ng * Tp;            // time slots of each warp's run
    const int64_t S = nlocal + 31;             // steps: lane 31 runs 31 behind lane 0
    const int64_t nbound = (S + RING - 1) / RING;             // boundaries: one every RING steps
    const int64_t nmma = (RING * (nbound - 1)) / kFtChunk + 1; // chunks read: up to the last boundary's

    const FtSmem L = ft_smem_layout(RC, p.kp, RING);
    const uint32_t sbase = smem_u32(smem);
    FtState *st = reinterpret_cast<FtState *>(smem + L.misc);
    volatile int *cta_err = &st->err;
    const uint32_t bar_a = sbase + L.bars, bar_aux = bar_a + 8, bar_b = bar_a + 16,
                   bar_mma = bar_b + 8 * kFtBSlots;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&st->tmem)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) {
        for (int i = 0; i < 4 + kFtBSlots; ++i) mbar_init(bar_a + 8 * i, 1); // a, aux, b[], mma[2]
        st->err = 0;
        st->arrive = 0;
        st->aux_pending = 0;
        st->a_block = -1;
        st->a_phase = 0;
        st->aux_phase = 0;
        st->staged_b = -1;
        st->issued = -1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = st->tmem;

    FtIssuer I;
    I.p = &p;
    I.st = st;
    I.g0 = g0;
    I.nlocal = nlocal;
    I.nchunks = nlocal / kFtChunk; // T is a multiple of kFtChunk
    I.rc = RC;
    I.a_base = sbase + L.a;
    I.b_base = sbase + L.b;
    I.bar_a = bar_a;
    I.bar_aux = bar_aux;
    I.bar_b = bar_b;
    I.bar_mma = bar_mma;
    I.tmem = tmem;
    I.tile_bytes = (uint32_t)kTcM * p.kp * 4;
    I.b_bytes = (uint32_t)kFtChunk * p.kp * 4;

    if (tid == 0) { // prologue: the first x block, y rows of chunks 0..2, MMAs of chunks 0 and 1
        I.stage_a(I.block_of(0));
        ++st->a_phase;
        I.stage_b(0);
        I.stage_b(1);
        if (I.issue(0) && I.issue(1) && nmma > 2) I.stage_b(2);
    }
    __syncwarp();

    // ---------------------------------------------------------------- the wavefront
    // ring slot j, y path r of this thread: myring[j * kSlotF + r * 32 * RC .. + RC)
    float *myring = reinterpret_cast<float *>(smem + L.ring) + (size_t)warp * RING * kSlotF + lane * RC;
    const uint32_t tq = tmem + ((uint32_t)(q * 32) << 16); // this warp's TMEM lane quarter
    const uint32_t arrive_addr = smem_u32(&st->arrive);

    // Boundary b, before steps [RING b, RING b + RING): chunk m = RING b / 16 is done (its MMAs waited for);
    // the increments of these steps come from chunks m - 1 and m (column c of chunk a is step
    // 16 a + c + ii of the thread that plays the row's lane, ring slot 16 a + c + ii - RING b).  The two
    // warps of a lane quarter share the copy: set 0 loads the LO family, set 1 the HI family, and thread t
    // writes the value of TMEM lane 32 q + t into the ring of the warp that owns the row (its own for
    // t < 16, its partner's for t >= 16; thread t of either warp plays a lane congruent to t mod 16, so
    // the ring offset and the skew ii are the same).  A 64-thread barrier of the pair before the copy
    // (both warps are done reading the previous period's slots) and one after it (the slots are written)
    // orders the cross-warp stores.  Then the arrival.  Chunk m - 1 is read for the last time at the
    // boundary whose period ends at step 16 m + 15 (b = m at RING = 16, b = 2m + 1 at RING = 8); the last
    // arrival there issues chunk m + 1 into its TMEM slot and stages the y rows of chunk m + 2.  No warp
    // arrives at a boundary before every warp has arrived at the previous one past the first chunk (the
    // next boundary's chunk is issued only at that last arrival), so the arrival that brings the count to
    // 8 (b + 1) is the last one of boundary b.
    float *dstring = lane < 16 ? myring : myring + (h ? -4 : 4) * RING * kSlotF; // the row owner's ring
    const int pair_bar = 1 + q; // named barrier of warps q and q + 4
    auto boundary = [&](int64_t b) {
        const int64_t m = (RING * b) / kFtChunk;
        if (!*cta_err && !mbar_wait(bar_mma + 8 * (uint32_t)(m & 1), (uint32_t)((m >> 1) & 1))) *cta_err = 1;
        tc_fence_after();
        named_bar(pair_bar, 64);
        // tcgen05.ld is warp-collective: decide for the whole warp (another thread may set the flag)
        if (!__any_sync(kFullMask, *cta_err != 0)) {
#pragma unroll 1
            for (int64_t a = (m > 0 ? m - 1 : 0); a <= m; ++a) {
                const int base = (int)(kFtChunk * a - RING * b) + ii;
#pragma unroll 1
                for (int r = 0; r < 2; ++r) {
                    float v[RC][kFtChunk]; // TMEM lane 32 q + lane of this warp's family, all RC tiles
                    const uint32_t col = (uint32_t)((a & 1) * 64 * RC + r * 32 * RC + h * 16 * RC);
#pragma unroll
                    for (int t = 0; t < RC; t += 2) {
                        if constexpr (RC == 1) {
                            uint32_t u[16], w[16];
                            tmem_ld16x2(tq + col, tq + col, u, w);
#pragma unroll
                            for (int c = 0; c < kFtChunk; ++c) v[0][c] = __uint_as_float(u[c]);
                        } else {
                            uint32_t u[16], w[16];
                            tmem_ld16x2(tq + col + t * 16, tq + col + (t + 1) * 16, u, w);
#pragma unroll
                            for (int c = 0; c < kFtChunk; ++c) {
                                v[t][c] = __uint_as_float(u[c]);
                                v[t + 1][c] = __uint_as_float(w[c]);
                            }
                        }
                    }
                    // one RC-float store per ring slot; a thread's slots are RC-float aligned and the slot
                    // stride is a multiple of 32 banks, so the warp's stores are conflict-free
#pragma unroll
                    for (int c = 0; c < kFtChunk; ++c) {
                        const int j = base + c;
                        if ((unsigned)j < (unsigned)RING) ft_ring_write<RC>(dstring + j * kSlotF + r * 32 * RC, v, c);
                    }
                }
            }
        }
        named_bar(pair_bar, 64);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
            const uint32_t old = atomic_add_acq_rel(arrive_addr, 1u);
            if (old + 1 == (uint32_t)(kFtWarps * (b + 1))) {
                tc_fence_after();
                const bool last_read_of_prev = RING == kFtChunk || (b & 1); // the last boundary reading m - 1
                if (last_read_of_prev && m >= 1 && m + 1 < nmma && I.issue(m + 1) && m + 2 < nmma) I.stage_b(m + 2);
            }
        }
        __syncwarp();
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
    const int src = (lane + 31) & 31; // the thread that plays wavefront lane lam - 1
    const Dbl2 one{1.0, 1.0};
    Dbl2 left[R];
#pragma unroll
    for (int i = 0; i < R; ++i) left[i] = one;
    Dbl2 bot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) bot[c] = one;
    Dbl2 corner_next = one;
    int col = 0;
    int64_t grp = 0, xi = 0, ya = 0;
    for (int64_t b = 0; b < nbound; ++b) {
        boundary(b);
        const int64_t s1 = (b + 1) * RING < S ? (b + 1) * RING : S;
        for (int64_t s = b * RING; s < s1; ++s) {
            Dbl2 top[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                top[c].x = __shfl_sync(kFullMask, bot[c].x, src);
                top[c].y = __shfl_sync(kFullMask, bot[c].y, src);
            }
            if (lam == 0) {
#pragma unroll
                for (int c = 0; c < C; ++c) top[c] = one;
            }
            const int64_t u = s - lam;
            if (u >= 0 && u < nlocal) {
                if (col == 0) {
                    const int64_t g = g0 + grp, a = g / p.hy;
                    xi = 8 * a + 4 * h + q;
                    ya = 2 * (g - a * p.hy);
#pragma unroll
                    for (int i = 0; i < R; ++i) left[i] = one;
                }
                if (col < ncy) {
                    const Dbl2 corner = (col == 0) ? one : corner_next;
                    corner_next = top[C - 1];
                    float ca[RC], cb[RC];
                    const float *rs = myring + (int)(s & (RING - 1)) * kSlotF;
                    ft_ring_read<RC>(rs, ca);
                    ft_ring_read<RC>(rs + 32 * RC, cb);
                    Dbl2 A[RC], B[RC];
#pragma unroll
                    for (int rc = 0; rc < RC; ++rc) stencil_coefs(Dbl2{(double)ca[rc], (double)cb[rc]}, A[rc], B[rc]);
                    stream_block<Dbl2, R, O>(left, top, corner, A, B, bot);
                    if (col == ncy - 1 && lam == lstar && xi < p.nx) {
                        const Dbl2 v = pick_row(left, rstar);
                        stream_store(sp, 0, xi, ya, v.x);
                        if (ya + 1 < p.ny) stream_store(sp, 0, xi, ya + 1, v.y);
                    }
                }
                if (++col == Tp) {
                    col = 0;
                    ++grp;
                }
            }
        }
    }

    // ---------------------------------------------------------------- teardown
    __syncthreads();
    if (*cta_err) { // the CTA's entries are incomplete: NaN, and the launch's error word
        if (tid == 0) {
            // let the copies and MMAs started here land (bounded) before the CTA exits
            const int64_t sb = st->staged_b;
            for (int64_t k = (sb > 3 ? sb - 3 : 0); k <= sb; ++k) I.wait_b(k);
            if (st->a_phase > 0) mbar_wait(bar_a, (st->a_phase - 1) & 1);
            if (st->aux_pending) mbar_wait(bar_aux, st->aux_phase & 1);
            if (st->issued >= 0) mbar_wait(bar_mma + 8 * (uint32_t)(st->issued & 1), (uint32_t)((st->issued >> 1) & 1));
            atomicOr(p.err, 1u);
        }
        for (int64_t e = tid; e < ng * 16; e += blockDim.x) {
            const int64_t g = g0 + e / 16, a = g / p.hy;
            const int r = (int)(e % 16);
            const int64_t i = 8 * a + (r >> 1), j = 2 * (g - a * p.hy) + (r & 1);
            if (i < p.nx && j < p.ny) stream_store(sp, 0, i, j, __longlong_as_double(0x7ff8000000000000LL));
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

} // namespace sigk
