// Tensor-core increments: the coarse increment matrix <dx_ci, dy_cj> of every
// pair, computed as one dense contraction over the path dimension on the
// 5th-generation tensor cores, then consumed by a streaming wavefront.
//
// The reference builds the increments with a static-kernel Gram and a 4-term
// second difference (sigpde/torch/kernel.py:13-21, static_kernels.py:3-11);
// for the linear kernel that is C = A * B^T with A the scaled differences of
// the x paths (one row per coarse cell) and B those of the y paths.
//
// Precision: split TF32.  Each difference v (exact in float64) is written as
// hi + lo with hi = tf32(v), lo = tf32(v - hi); the MMA sums hi*hi' + hi*lo' +
// lo*hi' in float32 (the lo*lo' term is below float32 resolution).  That keeps
// ~21 bits of each product instead of TF32's 11 (the "3xTF32" scheme).
//
// Kernels
//   tc_image_kernel     float64 differences -> hi/lo operand images laid out
//                       exactly as the MMA reads them from shared memory, so
//                       a whole operand tile is one contiguous bulk copy;
//   tc_gemm_kernel      persistent, one CTA per SM, warp-specialised: a
//                       producer lane stages each tile's operands with
//                       cp.async.bulk (TMA engine, completion on an mbarrier)
//                       and issues tcgen05.mma into one of two TMEM
//                       accumulators while 8 epilogue warps drain the other
//                       (tcgen05.ld -> shared memory -> 2-D TMA tensor store,
//                       cp.async.bulk.tensor, to HBM);
//   stream_inc_kernel   the streaming wavefront of stream.cuh reading its
//                       increments from that matrix (vector loads of the
//                       lane's coarse rows, or for long steps a cp.async ring
//                       two steps ahead) instead of forming dot products.
#pragma once

#include <cuda.h> // CUtensorMap

#include "ragged.cuh"
#include "stream.cuh"

namespace sigk {

constexpr int kTcM = 128;          // MMA M (rows of A per tile)
constexpr long kTcSpinLimit = 1L << 24;

enum : int { kTcAll = 0, kTcLower = 1, kTcDiag = 2, kTcTable = 3 };

// ------------------------------------------------------------------ TF32 split
// Round a float to the nearest TF32 value (10 explicit mantissa bits), ties to
// even, by integer arithmetic on the bit pattern.  Inputs here are finite and
// far from overflow (scaled path differences).
__device__ __forceinline__ float tf32_rne(float v)
{
    unsigned u = __float_as_uint(v);
    u += 0x0FFFu + ((u >> 13) & 1u);
    u &= 0xFFFFE000u;
    return __uint_as_float(u);
}

struct TcImageParams {
    const void *x;      // (npaths, len, d) in TIN
    int64_t npaths, len, d;
    int64_t rows_per_path; // rows of a path in the image (>= len - 1; extra rows are zero)
    int64_t tile_rows;     // rows per operand tile (128 for A, BN for B)
    int64_t ntiles;
    int kp;                // K padded to a multiple of 8
    double f;              // scale f * s[p]
    const void *s;         // per-path scale in TIN or null
    float *hi, *lo;
    // fused_rc > 0: the fused Gram's A layout (fused_tc.cuh).  Blocks of 8 x paths, each 2 fused_rc tiles
    // of 128 rows, LO tiles (f = 0) then HI tiles (f = 1): tile f fused_rc + k.  Row 32 q + t of tile
    // (f, k) holds coarse row fused_rc lam + k of path 8 a + 4 h + q, where lam = 16 f + t % 16 is
    // the wavefront lane and h = (t / 16) xor f the warp set that owns the row.
    int fused_rc;
};

// Image layout (group-major): element (row m, k) sits at float offset
// ((m/8 * kp/4 + k/4) * 8 + m%8) * 4 + k%4.  A group of 8 rows holds all of K
// as kp/4 core matrices of 8 rows x 16 bytes (128 bytes each), so any run of
// rows that starts at a multiple of 8 is one contiguous block: an operand
// tile is a single bulk copy wherever it starts.  For tcgen05.mma this is the
// canonical K-major, no-swizzle layout with 128 bytes between the two K
// chunks of one MMA (leading byte offset) and kp*32 bytes between 8-row
// groups (stride byte offset).
__host__ __device__ __forceinline__ int64_t image_offset(int64_t m, int64_t k, int kp)
{
    return (((m >> 3) * (kp >> 2) + (k >> 2)) * 8 + (m & 7)) * 4 + (k & 3);
}

template <typename TIN>
__global__ void tc_image_kernel(TcImageParams p)
{
    const TIN *__restrict__ x = reinterpret_cast<const TIN *>(p.x);
    const TIN *__restrict__ sc = reinterpret_cast<const TIN *>(p.s);
    const int64_t nkc = p.kp / 4;
    const int64_t total = p.ntiles * p.tile_rows * p.kp;
    const int64_t nc = p.len - 1;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        // e enumerates the image in memory order: group, K chunk, row in group, k in chunk
        const int64_t k4 = e & 3;
        const int64_t r8 = (e >> 2) & 7;
        const int64_t rest = e >> 5;
        const int64_t kc = rest % nkc;
        const int64_t g = rest / nkc;
        const int64_t m = g * 8 + r8;
        const int64_t k = kc * 4 + k4;
        int64_t path, c;
        if (p.fused_rc > 0) {
            const int64_t per_block = (int64_t)p.fused_rc * 256, rem = m % per_block;
            const int64_t tile = rem >> 7, fam = tile / p.fused_rc, tk = tile - fam * p.fused_rc;
            const int64_t t = rem & 31, h = (t >> 4) ^ fam, lam = 16 * fam + (t & 15);
            path = 8 * (m / per_block) + 4 * h + (rem >> 5 & 3);
            c = (int64_t)p.fused_rc * lam + tk;
        } else {
            path = m / p.rows_per_path;
            c = m - path * p.rows_per_path;
        }
        float hi = 0.f, lo = 0.f;
        if (path < p.npaths && c < nc && k < p.d) {
            const TIN *xp = x + (path * p.len + c) * p.d + k;
            const double g = sc ? p.f * (double)sc[path] : p.f;
            const double v = ((double)xp[p.d] - (double)xp[0]) * g;
            hi = tf32_rne((float)v);
            lo = tf32_rne((float)(v - (double)hi));
        }
        p.hi[e] = hi;
        p.lo[e] = lo;
    }
}

// Operand images of an uneven batch: pair b's row path (the shorter of its
// two paths, as the wavefront puts it on the rows) goes to the A image at
// row0[b] (side 0), its column path to the B image (side 1).  Rows of a pair
// are padded to a multiple of 8 with zeros.  The A side carries the static
// scale and 4^-order of the pair; each side carries its own path's scale.
struct TcRaggedImageParams {
    const void *x_pack, *y_pack;
    const int64_t *x_off, *x_len, *y_off, *y_len;
    const int *order;
    double f;
    const void *sx, *sy;  // per pair, TIN, or null
    const int64_t *row0;  // per pair: first image row (multiple of 8)
    int64_t rows_alloc;
    int64_t npairs, d;
    int kp;
    int side;
    float *hi, *lo;
};

template <typename TIN>
__global__ void tc_ragged_image_kernel(TcRaggedImageParams p)
{
    const int64_t nkc = p.kp / 4;
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
        float *hi = p.hi + r0 * p.kp, *lo = p.lo + r0 * p.kp;
        const int64_t total = rows8 * p.kp;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
             e += (int64_t)gridDim.x * blockDim.x) {
            const int64_t k4 = e & 3;
            const int64_t r8 = (e >> 2) & 7;
            const int64_t rest = e >> 5;
            const int64_t kc = rest % nkc;
            const int64_t c = (rest / nkc) * 8 + r8;
            const int64_t k = kc * 4 + k4;
            float h = 0.f, l = 0.f;
            if (c < nc && k < p.d) {
                const TIN *xp = xp0 + c * p.d + k;
                const double v = ((double)xp[p.d] - (double)xp[0]) * g;
                h = tf32_rne((float)v);
                l = tf32_rne((float)(v - (double)h));
            }
            hi[e] = h;
            lo[e] = l;
        }
    }
}

// ------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return done != 0;
}

// Bounded wait on an mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long i = 0; i < kTcSpinLimit; ++i) {
        if (mbar_test(bar, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor (tcgen05): start address, leading (K
// direction) and stride (M/N direction) byte offsets in 16-byte units, the
// sm_100 descriptor version (bit 46) and layout type 0 = no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor for kind::tf32: float32 accumulator (bits 4-5 = 1),
// A and B TF32 (bits 7-9 and 10-12 = 2), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
                 "l"(a), "l"(b), "r"(idesc), "r"(acc)
                 : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 consecutive TMEM columns of this warp's 32 lanes: v[j] = column col + j of lane (row) lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                 "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
                   "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
                   "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// Two 16-column loads of the warp's lane quarter (32x32b.x16 each) and one wait.
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, uint32_t (&a)[16], uint32_t (&b)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7]),
                   "=r"(a[8]), "=r"(a[9]), "=r"(a[10]), "=r"(a[11]), "=r"(a[12]), "=r"(a[13]), "=r"(a[14]),
                   "=r"(a[15])
                 : "r"(ta)
                 : "memory");
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7]),
                   "=r"(b[8]), "=r"(b[9]), "=r"(b[10]), "=r"(b[11]), "=r"(b[12]), "=r"(b[13]), "=r"(b[14]),
                   "=r"(b[15])
                 : "r"(tb)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ------------------------------------------------------------------ GEMM
struct TcGemmParams {
    const float *a_hi, *a_lo; // A image: mtiles tiles of 128 rows
    const float *b_hi, *b_lo; // B image: ntiles tiles of BN rows
    int64_t mtiles, ntiles;
    int kp;
    int mode;                 // kTcAll / kTcLower (symmetric Gram) / kTcDiag (pairwise)
    int64_t m_rows, n_rows;   // rows of A / B that are stored (the rest is tile padding)
    int64_t rows_x, rows_y;   // rows per x path (A) and per y path (B)
    int64_t npaths_x, npaths_y;
    int64_t x0;               // kTcLower: global index of the first x path of A (chunked symmetric Gram)
    float *out;
    int64_t ld;               // kTcAll/kTcLower: out[n * ld + m]; kTcDiag: out[n * rows_x + m % rows_x]
    unsigned *err;
    // kTcTable (uneven pairs): one entry of kTcTileWords per tile, {a_row, b_row, m_valid, n_valid,
    // out_off, ld}: the tile's first A and B image rows (multiples of 8), its valid rows and columns,
    // and where its (column-major, ld floats per column) block of increments starts in out
    const int64_t *table;
    int64_t ntable;
    int64_t a_rows, b_rows;   // image rows allocated (tiles must lie inside)
    int64_t out_elems;        // floats in out
};

constexpr int kTcTileWords = 6;

template <int BN>
__device__ __forceinline__ bool tc_tile_needed(const TcGemmParams &p, int64_t mt, int64_t nt)
{
    if (p.mode == kTcAll) return true;
    int64_t i_lo = (mt * kTcM) / p.rows_x;
    int64_t i_hi = (mt * kTcM + kTcM - 1) / p.rows_x;
    if (i_hi >= p.npaths_x) i_hi = p.npaths_x - 1;
    int64_t j_lo = (nt * BN) / p.rows_y;
    int64_t j_hi = (nt * BN + BN - 1) / p.rows_y;
    if (j_hi >= p.npaths_y) j_hi = p.npaths_y - 1;
    if (p.mode == kTcLower) return j_lo <= i_hi + p.x0;
    return j_lo <= i_hi && i_lo <= j_hi;
}

// A table entry that would read or write outside its buffers is refused
// (error bit 4) and skipped by both warp roles alike.
template <int BN>
__device__ __forceinline__ bool tc_table_entry_ok(const TcGemmParams &p, const int64_t *e)
{
    const int64_t a_row = e[0], b_row = e[1], mv = e[2], nv = e[3], off = e[4], ld = e[5];
    return a_row >= 0 && (a_row & 7) == 0 && a_row + kTcM <= p.a_rows && b_row >= 0 && (b_row & 7) == 0 &&
           b_row + BN <= p.b_rows && mv >= 1 && mv <= kTcM && nv >= 1 && nv <= BN && ld >= 4 && (ld & 3) == 0 &&
           ((mv + 3) & ~3LL) <= ld && off >= 0 && (off & 3) == 0 && off + (nv - 1) * ld + ((mv + 3) & ~3LL) <= p.out_elems;
}

template <int BN>
__device__ __forceinline__ int64_t tc_total_tiles(const TcGemmParams &p)
{
    return p.mode == kTcTable ? p.ntable : p.mtiles * p.ntiles;
}

template <int BN>
__device__ __forceinline__ int64_t tc_next_tile(const TcGemmParams &p, int64_t t)
{
    const int64_t total = tc_total_tiles<BN>(p);
    for (; t < total; t += gridDim.x) {
        if (p.mode == kTcTable) {
            if (tc_table_entry_ok<BN>(p, p.table + t * kTcTileWords)) return t;
            if (threadIdx.x == 0) atomicOr(p.err, 4u);
        } else if (tc_tile_needed<BN>(p, t / p.ntiles, t % p.ntiles)) {
            return t;
        }
    }
    return total;
}

__device__ __forceinline__ void named_bar(int id, int nthreads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}

// Contiguous bulk copy shared -> global (TMA engine); 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_s2g(void *dst, uint32_t src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
}

// 2-D tiled TMA store of a shared-memory box (x = innermost coordinate).
__device__ __forceinline__ void tma_store_2d(const void *map, uint32_t src, int x, int y)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(map), "r"(src),
                 "r"(x), "r"(y)
                 : "memory");
}

// Warp roles of tc_gemm_kernel: warps 0-7 drain the accumulators (two per
// TMEM lane quarter, one per half of the N columns); warp 8 owns the TMEM
// allocation and its lane 0 stages operands and issues the MMAs.
constexpr int kTcEpiWarps = 8;
constexpr int kTcThreads = (kTcEpiWarps + 1) * 32;
constexpr int kTcStageCols = 32; // columns per TMA store box (box = 128 rows x 32 columns)

// Shared-memory layout of tc_gemm_kernel<BN> (byte offsets).
struct TcSmem {
    uint32_t staging;  // 2 halves x 2 buffers x (32 columns x 128 rows) floats
    uint32_t operands; // a_hi, a_lo (128 x kp), b_hi, b_lo (BN x kp)
    uint32_t bars;     // full, mma_done[2], acc_empty[2]
    uint32_t misc;     // TMEM address, abort flag, per-warp ok flags
    uint32_t total;
};

__host__ __device__ __forceinline__ TcSmem tc_smem_layout(int bn, int kp)
{
    TcSmem s{};
    s.staging = 0;
    s.operands = 2 * 2 * kTcStageCols * kTcM * 4;
    s.bars = s.operands + (2 * kTcM + 2 * bn) * kp * 4;
    s.misc = s.bars + 5 * 8;
    s.total = s.misc + 16 + 4 * kTcEpiWarps;
    return s;
}

template <int BN>
__global__ void __launch_bounds__(kTcThreads, 1) tc_gemm_kernel(TcGemmParams p, const __grid_constant__ CUtensorMap out_map)
{
    static_assert(BN % 64 == 0 && BN >= 64 && BN <= 256, "N of a kind::tf32 MMA with M = 128, in 64-column halves");
    constexpr uint32_t kCols = 2 * BN; // two accumulators
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const TcSmem L = tc_smem_layout(BN, p.kp);
    const uint32_t a_bytes = (uint32_t)kTcM * p.kp * 4;
    const uint32_t b_bytes = (uint32_t)BN * p.kp * 4;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t s_ahi = sbase + L.operands, s_alo = s_ahi + a_bytes;
    const uint32_t s_bhi = s_alo + a_bytes, s_blo = s_bhi + b_bytes;
    const uint32_t bar_full = sbase + L.bars, bar_mma0 = bar_full + 8, bar_empty0 = bar_full + 24;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L.misc);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(smem + L.misc + 4);
    volatile int *ok_flags = reinterpret_cast<volatile int *>(smem + L.misc + 16);

    if (warp == kTcEpiWarps) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar_full, 1);
        mbar_init(bar_mma0, 1);
        mbar_init(bar_mma0 + 8, 1);
        mbar_init(bar_empty0, kTcEpiWarps);
        mbar_init(bar_empty0 + 8, kTcEpiWarps);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == kTcEpiWarps) {
        // ---------------------------------------------------------- producer / MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tf32_idesc(kTcM, BN);
            int it = 0;
            for (int64_t tile = tc_next_tile<BN>(p, blockIdx.x); tile < tc_total_tiles<BN>(p);
                 tile = tc_next_tile<BN>(p, tile + gridDim.x), ++it) {
                if (*abort_flag) break;
                const int b = it & 1;
                bool ok = true;
                if (it >= 2) ok = mbar_wait(bar_empty0 + 8 * b, ((it - 2) >> 1) & 1); // accumulator b drained
                if (ok && it >= 1) ok = mbar_wait(bar_mma0 + 8 * ((it - 1) & 1), ((it - 1) >> 1) & 1); // operands free
                if (!ok) {
                    atomicOr(p.err, 2u);
                    *abort_flag = 1;
                    break;
                }
                int64_t a_row, b_row; // first image rows of the tile (group-major: row r starts at float r * kp)
                if (p.mode == kTcTable) {
                    a_row = p.table[tile * kTcTileWords + 0];
                    b_row = p.table[tile * kTcTileWords + 1];
                } else {
                    a_row = (tile / p.ntiles) * kTcM;
                    b_row = (tile % p.ntiles) * BN;
                }
                mbar_expect_tx(bar_full, 2 * a_bytes + 2 * b_bytes);
                bulk_g2s(s_ahi, p.a_hi + a_row * p.kp, a_bytes, bar_full);
                bulk_g2s(s_alo, p.a_lo + a_row * p.kp, a_bytes, bar_full);
                bulk_g2s(s_bhi, p.b_hi + b_row * p.kp, b_bytes, bar_full);
                bulk_g2s(s_blo, p.b_lo + b_row * p.kp, b_bytes, bar_full);
                if (!mbar_wait(bar_full, it & 1)) {
                    atomicOr(p.err, 1u);
                    *abort_flag = 1;
                    mbar_wait(bar_full, it & 1); // a second bounded chance for copies in flight to land
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(b * BN);
                // K step ks covers K chunks 2ks and 2ks+1 (8 TF32 values); small terms first
                const uint32_t sbo = (uint32_t)p.kp * 32; // bytes between 8-row groups
                for (int ks = 0; ks < p.kp / 8; ++ks) {
                    const uint32_t ko = (uint32_t)ks * 256; // two 128-byte K chunks per step
                    const uint64_t ahi = smem_desc(s_ahi + ko, 128, sbo);
                    const uint64_t alo = smem_desc(s_alo + ko, 128, sbo);
                    const uint64_t bhi = smem_desc(s_bhi + ko, 128, sbo);
                    const uint64_t blo = smem_desc(s_blo + ko, 128, sbo);
                    mma_tf32(d, alo, bhi, idesc, ks > 0 ? 1u : 0u);
                    mma_tf32(d, ahi, blo, idesc, 1u);
                    mma_tf32(d, ahi, bhi, idesc, 1u);
                }
                mma_commit(bar_mma0 + 8 * b);
            }
            if (it >= 1) mbar_wait(bar_mma0 + 8 * ((it - 1) & 1), ((it - 1) >> 1) & 1); // last MMAs done
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- epilogue: TMEM -> HBM
        const int quarter = warp & 3, half = warp >> 2;
        const bool leader = quarter == 0 && lane == 0; // issues this half's TMA tensor stores
        // threads that issue bulk stores (and so wait on their groups): the leader, or with a tile table
        // every lane of the half's first warp (one column each)
        const bool issuer = p.mode == kTcTable ? quarter == 0 : leader;
        float *staging = reinterpret_cast<float *>(smem + L.staging);
        int ctr = 0; // chunks stored by this half (selects the staging buffer)
        int it = 0;
        for (int64_t tile = tc_next_tile<BN>(p, blockIdx.x); tile < tc_total_tiles<BN>(p);
             tile = tc_next_tile<BN>(p, tile + gridDim.x), ++it) {
            const int b = it & 1;
            bool ok = !*abort_flag && mbar_wait(bar_mma0 + 8 * b, (it >> 1) & 1);
            if (!ok) {
                atomicOr(p.err, 2u);
                *abort_flag = 1;
            }
            // the four warps of a half agree before any named barrier of the tile
            if (lane == 0) ok_flags[warp] = ok ? 1 : 0;
            named_bar(1 + half, 128);
            ok = ok_flags[4 * half] && ok_flags[4 * half + 1] && ok_flags[4 * half + 2] && ok_flags[4 * half + 3];
            named_bar(1 + half, 128);
            if (!ok) break;
            tc_fence_after();
            const int64_t mt = tile / p.ntiles, nt = tile % p.ntiles;
            const int64_t m = mt * kTcM + quarter * 32 + lane;
            const int64_t *te = p.mode == kTcTable ? p.table + tile * kTcTileWords : nullptr;
            for (int c = 0; c < BN / 64; ++c) {
                const int col = half * (BN / 2) + c * 32;
                if (te && col >= te[3]) continue; // no valid column in this chunk (the same for the whole half)
                // table tiles: a lane quarter without valid rows skips its TMEM load (the warp still
                // takes part in the half's barriers)
                const bool rows_here = !te || quarter * 32 < te[2];
                float v[32];
                if (rows_here) tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * BN + col), v);
                const int64_t n0 = nt * BN + col;
                if (p.mode != kTcDiag) {
                    float *buf = staging + (size_t)(half * 2 + (ctr & 1)) * (kTcStageCols * kTcM);
                    ++ctr;
                    if (issuer) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                    named_bar(1 + half, 128); // buf is no longer read by an earlier store
                    if (rows_here) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) buf[j * kTcM + quarter * 32 + lane] = v[j];
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    named_bar(1 + half, 128); // buf complete
                    if (te) {
                        // one bulk copy per valid column, issued by lane j of the half's first warp:
                        // rows 0 .. m_valid rounded up to 4 (the pair's own zero padding)
                        if (quarter == 0) {
                            if (lane < te[3] - col) {
                                const uint32_t seg = (uint32_t)(((te[2] + 3) & ~3LL) * 4);
                                bulk_s2g(p.out + te[4] + (col + lane) * te[5], smem_u32(buf + lane * kTcM), seg);
                            }
                            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                        }
                    } else if (leader) {
                        tma_store_2d(&out_map, smem_u32(buf), (int)(mt * kTcM), (int)n0);
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                    }
                } else {
                    const bool mok = m < p.m_rows;
                    const int64_t px = mok ? m / p.rows_x : 0;
                    const int64_t cx = m - px * p.rows_x;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int64_t n = n0 + j;
                        if (mok && n < p.n_rows && n / p.rows_y == px) p.out[n * p.rows_x + cx] = v[j];
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_empty0 + 8 * b);
        }
        if (issuer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    if (warp == kTcEpiWarps) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

// Dynamic shared memory of tc_gemm_kernel<BN>; at least 200 KB so that one
// CTA holds an SM (and all of its TMEM columns).
__host__ __forceinline__ size_t tc_gemm_smem(int bn, int kp)
{
    const size_t s = tc_smem_layout(bn, kp).total;
    return s < 200 * 1024 ? 200 * 1024 : s;
}

// ------------------------------------------------------------------ wavefront
// Prefetch ring of stream_inc_kernel: each lane keeps the matrix values of its
// next PF steps in flight as cp.async copies into its own shared-memory slots
// (zero-filled where the lane's coarse rows start at or beyond ncx, as
// load_mat_vals reads them), so a step waits for a copy issued PF steps
// earlier rather than for a fresh global load.  Only the issuing lane reads a
// slot, after cp.async.wait_group has made its copy visible to it.
constexpr int kIncRingLaneBytes = 160; // shared memory per lane for the ring

template <typename TM, int RC, int CELLS>
struct IncRing {
    static constexpr int VB = RC * (int)sizeof(TM);   // bytes per lane per step
    static constexpr int CP = VB < 16 ? VB : 16;      // bytes per copy
    // steps of lead: two for long steps (32 or more cells a lane); shorter steps measured slower
    // with a ring (its bookkeeping costs more than the load latency it hides there)
    static constexpr int STEPS = CELLS >= 32 ? 2 : 0;
    static constexpr int CAP = kIncRingLaneBytes / VB - 1;
    static constexpr int PF = STEPS < CAP ? STEPS : (CAP > 0 ? CAP : 0); // 0: plain loads (load_mat_vals)
    static constexpr int SLOTS = PF + 1;
};

template <int SZ>
__device__ __forceinline__ void cp_async_zfill(uint32_t dst, const void *src, int src_bytes)
{
    if constexpr (SZ == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(SZ), "r"(src_bytes)
                     : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Copy the lane's RC values of one matrix row (chunks starting at or beyond
// ncx are zero-filled without a read) into a ring slot.
template <typename TM, int RC>
__device__ __forceinline__ void ring_fill(uint32_t dst, const TM *row, int ci0, int ncx)
{
    constexpr int VB = RC * (int)sizeof(TM);
    constexpr int CP = VB < 16 ? VB : 16;
    constexpr int EPC = CP / (int)sizeof(TM);
#pragma unroll
    for (int q = 0; q < VB / CP; ++q) {
        const bool ok = ci0 + q * EPC < ncx;
        cp_async_zfill<CP>(dst + q * CP, ok ? row + ci0 + q * EPC : row, ok ? CP : 0);
    }
}

template <typename T, typename TM, int RC>
__device__ __forceinline__ void ring_read(const unsigned char *src, T (&c)[RC])
{
    if constexpr (RC == 1) {
        c[0] = T(*reinterpret_cast<const TM *>(src));
    } else if constexpr (sizeof(TM) == 8) {
#pragma unroll
        for (int q = 0; q < RC / 2; ++q) {
            const double2 v = reinterpret_cast<const double2 *>(src)[q];
            c[2 * q + 0] = T(v.x);
            c[2 * q + 1] = T(v.y);
        }
    } else if constexpr (RC == 2) {
        const float2 v = *reinterpret_cast<const float2 *>(src);
        c[0] = T(v.x);
        c[1] = T(v.y);
    } else {
#pragma unroll
        for (int q = 0; q < RC / 4; ++q) {
            const float4 v = reinterpret_cast<const float4 *>(src)[q];
            c[4 * q + 0] = T(v.x);
            c[4 * q + 1] = T(v.y);
            c[4 * q + 2] = T(v.z);
            c[4 * q + 3] = T(v.w);
        }
    }
}

struct StreamIncParams {
    int op;           // kOpPairwise / kOpGram / kOpGramSym
    int in64;         // output dtype
    const void *inc;  // increment matrix (see tc_gemm_kernel, dgemm_inc_kernel), TM elements
    int64_t ld;       // Gram ops: floats between rows cj of the matrix
    int64_t rows_x;   // rows per x path in the matrix (ncx rounded up to 4)
    int64_t x0;       // first x path of this chunk (Gram ops)
    int64_t nx, ny;
    int64_t ncx, ncy;
    int order;
    void *out;
    int64_t out_ld;
    int64_t item0;    // first item of this chunk
    int64_t nitems;   // items in this chunk
    int64_t per_warp;
    const unsigned *err; // non-zero: the GEMM gave up a wait; results are NaN
};

// W lanes a pair pipeline: 32, or 16 for short pairs (n <= 16 R), where each
// half-warp streams its own run of pairs (per_warp counts pairs per pipeline):
// twice the rows a lane for the same pairs and half the pipeline fill.
template <typename T, int R, int O, typename TM, int W = 32>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) stream_inc_kernel(StreamIncParams p)
{
    static_assert(W == 32 || W == 16, "a pipeline is a warp or a half-warp");
    using BS = BlockShape<R, O>;
    constexpr int C = BS::C;
    constexpr int RC = BS::RC;
    const int lane = threadIdx.x & 31;
    const int sl = lane & (W - 1); // lane within the pipeline
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = (int64_t)blockIdx.x * kWarpsPerBlock + wib;
    const int64_t wfirst = gwarp * (32 / W) * p.per_warp; // the warp's first item
    if (wfirst >= p.nitems) return;                        // warp-uniform: no pipeline of this warp has work
    const int64_t first = wfirst + (lane / W) * p.per_warp;
    const int64_t left_items = p.nitems - first;
    const int cnt = left_items <= 0 ? 0 : (int)(left_items < p.per_warp ? left_items : p.per_warp);
    // the warp's first pipeline has the longest run; all lanes loop over its steps (shuffles are warp-wide)
    const int cnt_max = (int)((p.nitems - wfirst) < p.per_warp ? (p.nitems - wfirst) : p.per_warp);
    const int ncx = (int)p.ncx, ncy = (int)p.ncy;
    const int n = ncx << p.order;
    const int nsteps = (ncy << p.order) / C;
    const int ci0 = (sl * R) >> p.order;
    const int lstar = (n - 1) / R, rstar = (n - 1) % R;
    const int64_t row_ld = p.op == kOpPairwise ? p.rows_x : p.ld;
    StreamParams sp{}; // for stream_decode / stream_store
    sp.op = p.op;
    sp.in64 = p.in64;
    sp.ny = p.ny;
    sp.out = p.out;
    sp.out_ld = p.out_ld;
    if (*p.err) { // the increments are incomplete: report NaN rather than wrong numbers
        for (int k2 = sl; k2 < cnt; k2 += W) {
            int64_t xi, yj;
            const int64_t item = p.item0 + first + k2;
            stream_decode(sp, item, xi, yj);
            stream_store(sp, item, xi, yj, T(NAN));
        }
        return;
    }

    T left[R];
#pragma unroll
    for (int r = 0; r < R; ++r) left[r] = T(1);
    T bot[C];
#pragma unroll
    for (int c = 0; c < C; ++c) bot[c] = T(1);
    T corner_next = T(1);
    int q = 0, k = 0;
    int64_t item = 0, xi = 0, yj = 0;
    const TM *inc = reinterpret_cast<const TM *>(p.inc);
    const TM *base = inc;
    const int total = cnt_max * nsteps + (W - 1);

    // prefetch ring: the copy for the lane's step t + PF is issued at step t
    using Ring = IncRing<TM, RC, R * C>;
    // without a ring, float64 matrices load each step's values one step ahead into registers
    // (config 3 fp64: 3.70 -> 3.27 ms); float32 matrices measured no gain (2.22 vs 2.25 ms)
    constexpr bool kRegPrefetch = sizeof(TM) == 8;
    constexpr int PF = Ring::PF;
    __shared__ __align__(16) unsigned char ring_mem[PF > 0 ? kWarpsPerBlock * Ring::SLOTS * 32 * Ring::VB : 16];
    unsigned char *ring = ring_mem + ((size_t)wib * Ring::SLOTS * 32 + lane) * Ring::VB;
    constexpr int kSlot = 32 * Ring::VB; // bytes between the slots of one lane
    int rd = 0, wr = 0;                  // slots to read / fill next
    int tp = 0, kp = 0, qp = 0;          // step, item and column of the next copy
    const TM *bp = inc;
    const int tsteps = cnt * nsteps;
    auto issue = [&]() {
        if (tp < tsteps) {
            if (qp == 0) {
                int64_t a, b;
                const int64_t it = p.item0 + first + kp;
                stream_decode(sp, it, a, b);
                bp = p.op == kOpPairwise ? inc + (it - p.item0) * (int64_t)ncy * p.rows_x
                                         : inc + b * (int64_t)ncy * p.ld + (a - p.x0) * p.rows_x;
            }
            const int cj = (O <= 3) ? qp : ((qp * C) >> p.order);
            ring_fill<TM, RC>((uint32_t)__cvta_generic_to_shared(ring + wr * kSlot), bp + (int64_t)cj * row_ld, ci0,
                              ncx);
            if (++qp == nsteps) {
                qp = 0;
                ++kp;
            }
            ++tp;
        }
        cp_async_commit(); // empty groups past the end keep the count uniform
        if (++wr == Ring::SLOTS) wr = 0;
    };
    if constexpr (PF > 0) {
#pragma unroll 1
        for (int i = 0; i < PF; ++i) issue();
    }
    TM nxt[RC]; // the lane's next step's values (kRegPrefetch)
    auto fetch = [&]() {
        if (tp < tsteps) {
            if (qp == 0) {
                int64_t a, b;
                const int64_t it = p.item0 + first + kp;
                stream_decode(sp, it, a, b);
                bp = p.op == kOpPairwise ? inc + (it - p.item0) * (int64_t)ncy * p.rows_x
                                         : inc + b * (int64_t)ncy * p.ld + (a - p.x0) * p.rows_x;
            }
            const int cj = (O <= 3) ? qp : ((qp * C) >> p.order);
            load_mat_raw<TM, RC>(bp + (int64_t)cj * row_ld, ci0, ncx, nxt);
            if (++qp == nsteps) {
                qp = 0;
                ++kp;
            }
            ++tp;
        }
    };
    if constexpr (PF == 0) {
        if (kRegPrefetch) fetch();
    }

    for (int s = 0; s < total; ++s) {
        T top[C];
#pragma unroll
        for (int c = 0; c < C; ++c) top[c] = __shfl_up_sync(kFullMask, bot[c], 1, W);
        if (sl == 0) {
#pragma unroll
            for (int c = 0; c < C; ++c) top[c] = T(1);
        }
        if (s >= sl && k < cnt) {
            if (q == 0) {
                item = p.item0 + first + k;
                stream_decode(sp, item, xi, yj);
                if constexpr (PF == 0)
                    base = p.op == kOpPairwise ? inc + (item - p.item0) * (int64_t)ncy * p.rows_x
                                               : inc + yj * (int64_t)ncy * p.ld + (xi - p.x0) * p.rows_x;
#pragma unroll
                for (int r = 0; r < R; ++r) left[r] = T(1);
            }
            const T corner = (q == 0) ? T(1) : corner_next;
            corner_next = top[C - 1];
            T cur[RC];
            if constexpr (PF > 0) {
                cp_async_wait<PF - 1>(); // this step's copy has landed
                ring_read<T, TM, RC>(ring + rd * kSlot, cur);
                if (++rd == Ring::SLOTS) rd = 0;
                issue();
            } else if (kRegPrefetch) {
#pragma unroll
                for (int rc = 0; rc < RC; ++rc) cur[rc] = T(nxt[rc]);
                fetch();
            } else {
                const int cj = (O <= 3) ? q : ((q * C) >> p.order);
                load_mat_vals<T, TM, RC>(base + (int64_t)cj * row_ld, ci0, ncx, cur);
            }
            T A[RC], B[RC];
#pragma unroll
            for (int rc = 0; rc < RC; ++rc) stencil_coefs(cur[rc], A[rc], B[rc]);
            stream_block<T, R, O>(left, top, corner, A, B, bot);
            if (q == nsteps - 1 && sl == lstar) stream_store(sp, item, xi, yj, pick_row(left, rstar));
            if (++q == nsteps) {
                q = 0;
                ++k;
            }
        }
    }
    if constexpr (PF > 0) cp_async_wait<0>();
}

} // namespace sigk
