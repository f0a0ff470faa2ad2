// sigk_api.cu -- C ABI of libsigk.so (declared in include/sigk.h).
//
// Validates arguments on the host, picks a kernel variant from the problem
// shape (rows per lane R, dyadic order O, cell precision T, input dtype TIN),
// sizes a persistent grid to the device's resident capacity and enqueues the
// launch on the caller's stream.  Nothing here allocates device memory.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <unordered_map>

#include "../../include/sigk.h"
#include "dispatch.h"
#include "ragged.cuh"
#include "stream.cuh"
#include "tc.cuh"
#include "norm_pipe.cuh"
#include "dgemm_inc.cuh"
#include "static_inc.cuh"
#include "grad.cuh"
#include "fused_tc.cuh"

namespace sigk {
namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *where)
{
    return fail(SIGK_ELAUNCH, "%s: %s (%s)", where, cudaGetErrorString(e), cudaGetErrorName(e));
}

constexpr int kMaxBlocksPerSM = 8;
constexpr size_t kMaxStageBytesPerWarp = 24 * 1024;

int sm_count()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
    return n;
}

int64_t warp_cap() { return (int64_t)sm_count() * kMaxBlocksPerSM * kWarpsPerBlock; }

// Rows per lane: the smallest power of two in {2,4,8,16} that covers the
// refined rows with one band of 32*R rows, else 16 (several bands).
int pick_rows(int64_t n)
{
    if (n <= 64) return 2;
    if (n <= 128) return 4;
    if (n <= 256) return 8;
    return 16;
}

int rows_per_coarse_lane(int R, int order)
{
    if (order >= 4) return 1;
    int rc = R >> order;
    return rc > 0 ? rc : 1;
}

constexpr size_t kMaxStreamStageBytesPerWarp = 32 * 1024;

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Kernels enqueued by this library since load (sigk_launch_count).
std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
// Polls of a ragged band wait before it gives up (sigk_set_wait_limit; < 0: kProgressPollLimit).
std::atomic<long long> g_wait_limit{-1};
long long wait_limit()
{
    const long long v = g_wait_limit.load(std::memory_order_relaxed);
    return v < 0 ? kProgressPollLimit : v;
}

bool env_flag(const char *name)
{
    const char *v = getenv(name);
    return v && v[0] && v[0] != '0';
}

struct Plan {
    int R;
    int O;
    int nbands;
    int64_t n, m;
    bool stream;                 // streaming kernel (one band, >= 32 column blocks)
    int D;                       // stream: padded dimension of the register variant, 0 = shared-memory variant
    size_t stage_bytes_per_warp; // shared memory per warp (0 = none)
    size_t dx_off, dy_off;       // stream: precomputed path differences in the workspace
    size_t bnd_off;              // multi-band: boundary rows in the workspace
    int64_t bnd_stride;          // elements per warp
    size_t ws_bytes;             // total workspace
};

// Kernel choice and workspace layout for one request.  sigk_workspace_size()
// and the entry points call this with the same arguments, so the size a
// caller allocates is the size the launch uses.
Plan make_plan(int op, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t d, int order, size_t tsize,
               bool from_inc)
{
    Plan pl{};
    pl.n = ncx << order;
    pl.m = ncy << order;
    pl.O = order >= 4 ? 4 : order;
    const int C = order >= 4 ? 8 : (1 << order);

    const int Rs = pick_rows(pl.n);
    const int rc = rows_per_coarse_lane(Rs, order);
    int Dp = 2;
    while (Dp < d) Dp <<= 1;
    const bool reg_ok = rc * Dp <= 32 && !env_flag("SIGK_NO_REG_DX");
    const size_t sbytes = reg_ok ? 0 : 2 * (size_t)rc * (size_t)d * 32 * tsize;
    if (!from_inc && op != SIGK_OP_NORMALIZE && pl.n <= 32 * Rs && pl.m / C >= 32 &&
        sbytes <= kMaxStreamStageBytesPerWarp && !env_flag("SIGK_NO_STREAM")) {
        pl.stream = true;
        pl.R = Rs;
        pl.D = reg_ok ? Dp : 0;
        pl.nbands = 1;
        pl.stage_bytes_per_warp = sbytes;
        const int64_t dp = reg_ok ? Dp : d;
        const size_t dxb = align256((size_t)nx * ncx * dp * tsize);
        const size_t dyb = align256((size_t)ny * ncy * dp * tsize);
        pl.dx_off = 0;
        pl.dy_off = dxb;
        pl.ws_bytes = dxb + dyb;
        return pl;
    }

    pl.R = Rs;
    if (!from_inc) {
        // shrink R (more bands) until the dx staging fits; if even R=2 does not fit, read dx from global
        int R = pl.R;
        while (true) {
            size_t bytes = (size_t)rows_per_coarse_lane(R, order) * (size_t)d * 32 * tsize;
            if (bytes <= kMaxStageBytesPerWarp) {
                pl.R = R;
                pl.stage_bytes_per_warp = bytes;
                break;
            }
            if (R == 2) break;
            R >>= 1;
        }
    }
    pl.nbands = (int)((pl.n + 32 * pl.R - 1) / (32 * pl.R));
    if (pl.nbands > 1) {
        pl.bnd_stride = ((pl.m + 1 + 31) / 32) * 32;
        pl.bnd_off = 0;
        pl.ws_bytes = (size_t)warp_cap() * (size_t)pl.bnd_stride * tsize;
    }
    if (!from_inc && op != SIGK_OP_NORMALIZE) {
        // the per-pair kernel reads precomputed, scaled, dimension-major differences (delta_kernel)
        pl.dx_off = align256(pl.ws_bytes);
        pl.dy_off = pl.dx_off + align256((size_t)nx * ncx * d * tsize);
        pl.ws_bytes = pl.dy_off + align256((size_t)ny * ncy * d * tsize);
    }
    return pl;
}

PairFn pick_pair(int precision, int dtype, int mode, int R, int O)
{
    const bool in64 = (dtype == SIGK_F64);
    return (precision == SIGK_PREC_FP64 || precision == SIGK_PREC_TC64) ? get_pair_kernel_f64(in64, mode, R, O)
                                                                         : get_pair_kernel_f32(in64, mode, R, O);
}


// ------------------------------------------------------------------ launching
struct OccKey {
    const void *fn;
    size_t smem;
    int dev;
    bool operator==(const OccKey &o) const { return fn == o.fn && smem == o.smem && dev == o.dev; }
};
struct OccHash {
    size_t operator()(const OccKey &k) const
    {
        return std::hash<const void *>()(k.fn) ^ (k.smem * 1315423911u) ^ ((size_t)k.dev << 48);
    }
};
std::mutex g_occ_mu;
std::unordered_map<OccKey, int, OccHash> g_occ;

int blocks_per_sm(const void *fn, size_t smem, int *out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    OccKey key{fn, smem, dev};
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        auto it = g_occ.find(key);
        if (it != g_occ.end()) {
            *out = it->second;
            return SIGK_OK;
        }
    }
    if (smem > 48 * 1024) {
        // Opt the kernel in to the device maximum (not to this request's size): the
        // attribute is per function, and a later, smaller request must not lower it
        // below the size of an earlier one that is still cached above.
        int optin = 0;
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
        cudaFuncAttributes fa{};
        e = cudaFuncGetAttributes(&fa, fn);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncGetAttributes");
        optin -= (int)fa.sharedSizeBytes; // static shared memory counts against the same limit
        if (smem > (size_t)optin) return fail(SIGK_ELAUNCH, "kernel needs %zu bytes of shared memory (max %d)", smem, optin);
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    }
    int nb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kWarpsPerBlock * 32, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (nb <= 0) return fail(SIGK_ELAUNCH, "kernel cannot be resident (smem=%zu bytes)", smem);
    if (nb > kMaxBlocksPerSM) nb = kMaxBlocksPerSM;
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        g_occ[key] = nb;
    }
    *out = nb;
    return SIGK_OK;
}

template <class P>
int launch(void (*fn)(P), P params, int64_t nitems, size_t smem, cudaStream_t stream)
{
    int nb = 0;
    int st = blocks_per_sm((const void *)fn, smem, &nb);
    if (st != SIGK_OK) return st;
    const int64_t want = (nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const int64_t cap = (int64_t)sm_count() * nb;
    const int64_t blocks = want < cap ? want : cap;
    if (blocks <= 0) return SIGK_OK;
    fn<<<(unsigned)blocks, kWarpsPerBlock * 32, smem, stream>>>(params);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return SIGK_OK;
}

bool is_device_ptr(const void *p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int check_common(int dtype, int precision, int order)
{
    if (dtype != SIGK_F32 && dtype != SIGK_F64) return fail(SIGK_EINVAL, "dtype must be SIGK_F32 or SIGK_F64");
    if (precision != SIGK_PREC_FP64 && precision != SIGK_PREC_FP32 && precision != SIGK_PREC_TC32 &&
        precision != SIGK_PREC_TC64)
        return fail(SIGK_EINVAL, "precision must be SIGK_PREC_FP64, _FP32, _TC32 or _TC64");
    if (order < 0 || order > 12) return fail(SIGK_EINVAL, "dyadic order %d outside [0, 12]", order);
    return SIGK_OK;
}

int check_dev(const void *p, const char *name, bool nullable)
{
    if (!p) return nullable ? SIGK_OK : fail(SIGK_EINVAL, "%s is NULL", name);
    if (!is_device_ptr(p)) return fail(SIGK_EINVAL, "%s is not a device pointer", name);
    return SIGK_OK;
}

// Cell precision of a mode: the tensor-core modes differ from FP64 / FP32 only
// in how the increments of linear-kernel pairs are formed.
int cell_prec(int precision)
{
    return (precision == SIGK_PREC_FP64 || precision == SIGK_PREC_TC64) ? SIGK_PREC_FP64 : SIGK_PREC_FP32;
}
bool is_tc(int precision) { return precision == SIGK_PREC_TC32 || precision == SIGK_PREC_TC64; }

size_t tsize_of(int precision) { return cell_prec(precision) == SIGK_PREC_FP64 ? 8 : 4; }

int check_ws(const Plan &pl, void *ws, size_t ws_bytes)
{
    if (pl.ws_bytes == 0) return SIGK_OK;
    if (!ws || ws_bytes < pl.ws_bytes)
        return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", pl.ws_bytes, ws ? ws_bytes : 0);
    if (((uintptr_t)ws & 15) != 0) return fail(SIGK_EINVAL, "workspace must be 16-byte aligned");
    return SIGK_OK;
}


// ------------------------------------------------------------------ tensor-core increments
// Plan of a linear-kernel request in a TC mode: the increments of every pair
// come from one TF32x3 tensor-core GEMM (tc.cuh) into an fp32 matrix in the
// workspace, which a streaming wavefront then reads.  Eligible: one band of
// rows per pair (the streaming kernel's shapes) and dim <= 32 (the operand
// tiles of both stages fit shared memory).  The x paths are cut into chunks
// so that the matrix stays under kTcChunkBytes (SIGK_TC_CHUNK_MB overrides).
constexpr size_t kTcChunkBytes = size_t(6) << 30;

struct TcPlan {
    bool ok;
    bool stream;              // streaming consumer (one band, >= 32 column blocks); else the per-pair kernel
    int R, O, nbands;
    int64_t bnd_stride;
    size_t bnd_off;
    int kp;
    int64_t rows_x, rows_y;   // matrix rows per x path (ncx rounded up to 4) and per y path
    int64_t chunk, nchunks;   // x paths per chunk
    int64_t a_tiles, b_tiles; // operand tiles per image
    size_t a_bytes, b_bytes;  // bytes of one (hi or lo) image
    size_t err_off, a_off, b_off, ct_off, ws_bytes;
};

// Float matrices read by half-warp pipelines at order 1 (at most 128 refined rows) run faster in
// chunks of at most 1 GiB: RobustSigPDE.gram N=512, L=64, d=16, tc64 2.23 -> 2.04 ms; a 512 x 512
// order-1 Gram 3.64 -> 3.33 ms (tc32 symmetric 1.93 -> 1.73 ms).  Orders 0 and 2 and float64
// matrices measured slower with small chunks, so they keep kTcChunkBytes.
constexpr size_t kTcChunkBytesHalfWarpO1 = size_t(1) << 30;

size_t tc_chunk_cap(bool half_warp_order1 = false)
{
    const char *v = getenv("SIGK_TC_CHUNK_MB");
    if (v && v[0]) {
        long long mb = atoll(v);
        if (mb > 0) return (size_t)mb << 20;
    }
    return half_warp_order1 ? kTcChunkBytesHalfWarpO1 : kTcChunkBytes;
}

TcPlan make_tc_plan(int op, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t d, int order, size_t tsize)
{
    TcPlan t{};
    const int64_t n = ncx << order, m = ncy << order;
    const int C = order >= 4 ? 8 : (1 << order);
    const int Rs = pick_rows(n);
    if (d > 32 || env_flag("SIGK_NO_TC")) return t;
    t.ok = true;
    t.stream = n <= 32 * Rs && m / C >= 32;
    t.R = Rs;
    t.O = order >= 4 ? 4 : order;
    t.nbands = (int)((n + 32 * Rs - 1) / (32 * Rs));
    size_t bnd_bytes = 0;
    if (!t.stream && t.nbands > 1) { // one boundary row per warp of the per-pair kernel
        t.bnd_stride = ((m + 1 + 31) / 32) * 32;
        bnd_bytes = align256((size_t)warp_cap() * (size_t)t.bnd_stride * tsize);
    }
    t.kp = (int)((d + 7) / 8 * 8);
    t.rows_x = (ncx + 3) / 4 * 4;
    t.rows_y = ncy;
    const int64_t width = op == kOpPairwise ? ncy : (op == kOpGram ? ny : nx) * ncy; // matrix rows per x path
    const size_t per_x = (size_t)t.rows_x * (size_t)width * sizeof(float);
    int64_t chunk = (int64_t)(tc_chunk_cap(order == 1 && n <= 128) / per_x);
    if (chunk < 1) chunk = 1;
    if (chunk > nx) chunk = nx;
    t.chunk = chunk;
    t.nchunks = (nx + chunk - 1) / chunk;
    t.a_tiles = (chunk * t.rows_x + kTcM - 1) / kTcM;
    const int64_t b_rows = op == kOpPairwise ? chunk * ncy : (op == kOpGram ? ny : nx) * ncy;
    t.b_tiles = (b_rows + kTcBN - 1) / kTcBN;
    t.a_bytes = align256((size_t)t.a_tiles * kTcM * t.kp * sizeof(float));
    t.b_bytes = align256((size_t)t.b_tiles * kTcBN * t.kp * sizeof(float));
    t.err_off = 0;
    t.bnd_off = 256;
    t.a_off = t.bnd_off + bnd_bytes;
    t.b_off = t.a_off + 2 * t.a_bytes;
    t.ct_off = t.b_off + 2 * t.b_bytes;
    t.ws_bytes = t.ct_off + align256((size_t)chunk * per_x);
    return t;
}

// fused_rc > 0: the fused Gram's permuted A layout (TcImageParams::fused_rc)
int tc_image(bool in64, const void *x, int64_t npaths, int64_t len, int64_t d, int64_t rows_per_path, int64_t tile_rows,
             int64_t ntiles, int kp, double f, const void *s, float *hi, float *lo, cudaStream_t stream, int fused_rc = 0)
{
    TcImageParams ip{};
    ip.fused_rc = fused_rc;
    ip.x = x;
    ip.npaths = npaths;
    ip.len = len;
    ip.d = d;
    ip.rows_per_path = rows_per_path;
    ip.tile_rows = tile_rows;
    ip.ntiles = ntiles;
    ip.kp = kp;
    ip.f = f;
    ip.s = s;
    ip.hi = hi;
    ip.lo = lo;
    const int64_t total = ntiles * tile_rows * kp;
    int64_t blocks = (total + 255) / 256;
    if (blocks > (int64_t)sm_count() * 8) blocks = (int64_t)sm_count() * 8;
    get_tc_image_kernel(in64)<<<(unsigned)blocks, 256, 0, stream>>>(ip);
    count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "operand image kernel launch");
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_out_map(CUtensorMap *map, float *out, int64_t ld, int64_t n_rows)
{
    static std::mutex mu;
    static EncodeTiledFn encode = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!encode) {
            void *fn = nullptr;
            cudaDriverEntryPointQueryResult q{};
            cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
            if (e != cudaSuccess || !fn || q != cudaDriverEntryPointSuccess)
                return fail(SIGK_ELAUNCH, "cuTensorMapEncodeTiled is not available from the driver");
            encode = reinterpret_cast<EncodeTiledFn>(fn);
        }
    }
    // the increment matrix: n_rows rows of ld floats; boxes of 128 floats x 32 rows
    const cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)n_rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kTcM, (cuuint32_t)kTcStageCols};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, out, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(SIGK_ELAUNCH, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SIGK_OK;
}

// bn: tile width of the GEMM (kTcBN = 256; 128 for the uneven-batch plans that ask for it).
int tc_gemm(const TcGemmParams &gp, cudaStream_t stream, int bn = kTcBN)
{
    TcGemmFn fn = get_tc_gemm_kernel(bn);
    const size_t smem = tc_gemm_smem(bn, gp.kp);
    const int w = bn == 128 ? 0 : 1;
    static std::mutex mu;
    static bool attr_set[2][64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < 0 || dev >= 64) return fail(SIGK_EINVAL, "device index %d out of range", dev);
        if (!attr_set[w][dev]) {
            int optin = 0;
            e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
            if ((size_t)optin < smem) return fail(SIGK_ELAUNCH, "GEMM needs %zu bytes of shared memory", smem);
            e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
            if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
            attr_set[w][dev] = true;
        }
    }
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    if (gp.mode == kTcAll || gp.mode == kTcLower) { // 2-D TMA stores into the Gram's increment matrix
        if ((gp.ld & 3) != 0 || ((uintptr_t)gp.out & 15) != 0)
            return fail(SIGK_EINVAL, "increment matrix rows must be 16-byte aligned");
        int st = encode_out_map(&map, gp.out, gp.ld, gp.n_rows);
        if (st) return st;
    }
    int64_t grid = gp.mtiles * gp.ntiles;
    if (grid > sm_count()) grid = sm_count();
    fn<<<(unsigned)grid, kTcThreads, smem, stream>>>(gp, map);
    count_launch();
    e = cudaGetLastError();
    return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "tensor-core GEMM launch");
}


// The wavefront over one chunk of x paths [i0, i1) reading an increment matrix
// (out[n * ld + m], float32 from the tensor cores or float64 from
// dgemm_inc_kernel): the streaming kernel for single-band pairs with enough
// column blocks, else one pair per warp.
int consume_matrix(const TcPlan &t, int op, const void *mat, bool mat64, int64_t ld, const unsigned *err, int64_t i0,
                   int64_t i1, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t d, int order, void *out,
                   int64_t out_ld, bool in64, int precision, int dtype, unsigned char *wsb, cudaStream_t stream)
{
    int st;
    const int64_t nxc = i1 - i0;
    int64_t item0, nitems;
    if (op == kOpPairwise) {
        item0 = i0;
        nitems = nxc;
    } else if (op == kOpGram) {
        item0 = i0 * ny;
        nitems = nxc * ny;
    } else {
        item0 = i0 * (i0 + 1) / 2;
        nitems = i1 * (i1 + 1) / 2 - item0;
    }
    if (!t.stream) { // several bands or few column blocks: one pair per warp reading the matrix
        PairParams p{};
        p.op = op;
        p.nx = nx;
        p.ny = ny;
        p.ncx = ncx;
        p.ncy = ncy;
        p.d = d;
        p.order = order;
        p.fscale = 1.0;
        p.out = out;
        p.out_ld = out_ld;
        p.nitems = nitems;
        p.item0 = item0;
        p.mat = mat;
        p.mat_err = err;
        p.mat_ld = ld;
        p.mat_rows_x = t.rows_x;
        p.x0 = i0;
        p.bnd = t.nbands > 1 ? wsb + t.bnd_off : nullptr;
        p.bnd_stride = t.bnd_stride;
        PairFn pfn = pick_pair(precision, dtype, mat64 ? kPairMat64 : kPairMat, t.R, t.O);
        return launch(pfn, p, p.nitems, 0, stream);
    }
    const bool f64 = cell_prec(precision) == SIGK_PREC_FP64;
    // pairs of at most 128 refined rows run as half-warp pipelines (two pairs a warp, twice the rows a
    // lane, half the pipeline fill): measured faster except for float64 matrices at order 0 (one
    // column a step, where twice the rows a lane doubles each step's loads: 1.11 vs 1.02 ms at
    // N=128 L=128 d=32)
    const int64_t nrows = ncx << order;
    int W = 32, R = t.R;
    if (nrows <= 128 && !(mat64 && order == 0) && !env_flag("SIGK_NO_HALF_WARP")) {
        W = 16;
        R = 2;
        while (16 * R < nrows) R *= 2;
    }
    StreamIncFn fn = get_stream_inc_kernel(f64, R, t.O, mat64, W);
    int nb = 0;
    if ((st = blocks_per_sm((const void *)fn, 0, &nb))) return st;
    const int64_t warps = (int64_t)sm_count() * nb * kWarpsPerBlock * (32 / W); // pair pipelines
    StreamIncParams sp{};
    sp.op = op;
    sp.in64 = in64;
    sp.inc = mat;
    sp.ld = ld;
    sp.rows_x = t.rows_x;
    sp.x0 = i0;
    sp.nx = nx;
    sp.ny = ny;
    sp.ncx = ncx;
    sp.ncy = ncy;
    sp.order = order;
    sp.out = out;
    sp.out_ld = out_ld;
    sp.err = err;
    sp.item0 = item0;
    sp.nitems = nitems;
    const int64_t nw = warps < nitems ? warps : nitems;
    sp.per_warp = (nitems + nw - 1) / nw; // pairs a pipeline
    const int64_t used = (nitems + sp.per_warp - 1) / sp.per_warp;
    const int64_t used_warps = (used + (32 / W) - 1) / (32 / W);
    const int64_t blocks = (used_warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
    fn<<<(unsigned)blocks, kWarpsPerBlock * 32, 0, stream>>>(sp);
    count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "stream increment kernel launch");
}

// Fused tensor-core Gram (fused_tc.cuh): the tcgen05 increments go from TMEM
// through shared memory to the wavefront, never to HBM.  Workspace: error word,
// then the hi / lo operand images (2 RC tiles of 128 rows per block of 8 x
// paths, T rows per y path).
constexpr size_t kFtMaxSmem = 227 * 1024; // the B200's per-block opt-in limit
struct FtPlan {
    bool ok = false;
    int R = 0, O = 0, kp = 0, T = 0, ring = 16;
    size_t err_off = 0, a_off = 0, a_bytes = 0, b_off = 0, b_bytes = 0, ws_bytes = 0;
};

FtPlan make_fused_plan(int op, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t d, int order, int precision)
{
    FtPlan f;
    // The route where it is eligible and the order is 2 or more (cells outweigh the per-chunk boundary: config 2
    // 5.15 ms fused vs 5.59 two-phase; at orders 0-1 the two-phase route measured faster).  SIGK_FUSED_TC=1
    // takes it at every eligible order, SIGK_FUSED_TC=0 never.
    const char *force = getenv("SIGK_FUSED_TC");
    const int mode = (force && force[0]) ? (force[0] != '0' ? 1 : 0) : -1;
    if (op != kOpGram || precision != SIGK_PREC_TC64 || d > 32 || order > 3 || mode == 0 || (mode < 0 && order < 2))
        return f;
    const int64_t n = ncx << order;
    if (n > 32 * 16) return f; // one band
    const int R = pick_rows(n);
    const int rc = R >> order;
    if (rc < 1 || (rc << order) != R || rc > 4 || 32 * R < n) return f;
    // a boundary every 16 steps, or every 8 (half the ring) where the operands of a wide dimension need the room
    const int kpd = (int)((d + 7) / 8 * 8);
    const int ring = fused_tc_smem(rc, kpd, 16) <= kFtMaxSmem ? 16 : fused_tc_smem(rc, kpd, 8) <= kFtMaxSmem ? 8 : 0;
    if (!ring || !get_fused_tc_kernel(R, order, ring)) return f;
    // at 4 coarse rows a lane the 8-step boundary's copy outweighs the matrix round trip (256 x 256, L = 128,
    // d = 16, order 2: 5.93 vs 5.63 ms two-phase); at 2 it wins (L = 64, d = 32, order 3: 4.30 vs 4.44 ms)
    if (mode < 0 && ring == 8 && rc > 2) return f;
    f.ok = true;
    f.R = R;
    f.ring = ring;
    f.O = order;
    f.kp = (int)((d + 7) / 8 * 8);
    f.T = (int)((ncy + kFtChunk - 1) / kFtChunk * kFtChunk);
    f.err_off = 0;
    f.a_off = 256;
    f.a_bytes = align256((size_t)((nx + 7) / 8) * 2 * rc * kTcM * f.kp * sizeof(float));
    f.b_off = f.a_off + 2 * f.a_bytes;
    f.b_bytes = align256((size_t)ny * f.T * f.kp * sizeof(float));
    f.ws_bytes = f.b_off + 2 * f.b_bytes;
    return f;
}

int run_pairs_fused(const FtPlan &f, const void *x, const void *y, int64_t nx, int64_t ny, int64_t lx, int64_t ly,
                    int64_t d, int dtype, int order, double static_scale, const void *sx, const void *sy, void *out,
                    int64_t out_ld, void *ws, cudaStream_t stream)
{
    int st;
    const bool in64 = dtype == SIGK_F64;
    unsigned char *wsb = reinterpret_cast<unsigned char *>(ws);
    unsigned *err = reinterpret_cast<unsigned *>(wsb + f.err_off);
    float *a_hi = reinterpret_cast<float *>(wsb + f.a_off), *a_lo = reinterpret_cast<float *>(wsb + f.a_off + f.a_bytes);
    float *b_hi = reinterpret_cast<float *>(wsb + f.b_off), *b_lo = reinterpret_cast<float *>(wsb + f.b_off + f.b_bytes);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    const double fs = static_scale * std::ldexp(1.0, -2 * order); // x side: static scale * 4^-order * scale_x
    const int rc = f.R >> f.O;
    if ((st = tc_image(in64, x, nx, lx, d, kTcM, kTcM, (nx + 7) / 8 * 2 * rc, f.kp, fs, sx, a_hi, a_lo, stream, rc)))
        return st;
    if ((st = tc_image(in64, y, ny, ly, d, f.T, f.T, ny, f.kp, 1.0, sy, b_hi, b_lo, stream))) return st;
    FusedTcFn fn = get_fused_tc_kernel(f.R, f.O, f.ring);
    const size_t smem = fused_tc_smem(rc, f.kp, f.ring);
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    {
        static std::mutex mu;
        static std::unordered_map<uint64_t, bool> done; // (device, function) opted in to the maximum
        const uint64_t key = ((uint64_t)(uintptr_t)fn << 8) ^ (uint64_t)dev;
        std::lock_guard<std::mutex> lk(mu);
        if (!done[key]) {
            int optin = 0;
            e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
            if ((size_t)optin < smem) return fail(SIGK_ELAUNCH, "fused kernel needs %zu bytes of shared memory", smem);
            // the device maximum, not this call's size: a later call with a wider dimension needs more
            e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
            if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
            done[key] = true;
        }
    }
    FusedTcParams fp{};
    fp.a_hi = a_hi;
    fp.a_lo = a_lo;
    fp.b_hi = b_hi;
    fp.b_lo = b_lo;
    fp.nx = nx;
    fp.ny = ny;
    fp.ncx = (int)(lx - 1);
    fp.ncy = (int)(ly - 1);
    fp.kp = f.kp;
    fp.T = f.T;
    fp.hy = (ny + 1) / 2;
    fp.ngroups = (nx + 7) / 8 * fp.hy;
    const int64_t cap = (int64_t)sm_count(); // one CTA per SM (TMEM: up to 512 columns)
    const int64_t ctas0 = fp.ngroups < cap ? fp.ngroups : cap;
    fp.per_cta = (fp.ngroups + ctas0 - 1) / ctas0;
    const int64_t ctas = (fp.ngroups + fp.per_cta - 1) / fp.per_cta;
    fp.in64 = in64;
    fp.out = out;
    fp.out_ld = out_ld;
    fp.err = err;
    fn<<<(unsigned)ctas, kFtWarps * 32, smem, stream>>>(fp);
    count_launch();
    e = cudaGetLastError();
    return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "fused tensor-core kernel launch");
}

int run_pairs_tc(const TcPlan &t, int op, const void *x, const void *y, int64_t nx, int64_t ny, int64_t lx, int64_t ly,
                 int64_t d, int dtype, int order, double static_scale, const void *sx, const void *sy, void *out,
                 int64_t out_ld, int precision, void *ws, cudaStream_t stream)
{
    int st;
    const bool in64 = dtype == SIGK_F64;
    const size_t es = in64 ? 8 : 4;
    const int64_t ncx = lx - 1, ncy = ly - 1;
    unsigned char *wsb = reinterpret_cast<unsigned char *>(ws);
    unsigned *err = reinterpret_cast<unsigned *>(wsb + t.err_off);
    float *a_hi = reinterpret_cast<float *>(wsb + t.a_off), *a_lo = reinterpret_cast<float *>(wsb + t.a_off + t.a_bytes);
    float *b_hi = reinterpret_cast<float *>(wsb + t.b_off), *b_lo = reinterpret_cast<float *>(wsb + t.b_off + t.b_bytes);
    float *ct = reinterpret_cast<float *>(wsb + t.ct_off);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    const double fs = static_scale * std::ldexp(1.0, -2 * order); // x side: static scale * 4^-order * scale_x
    const char *xb = reinterpret_cast<const char *>(x);
    const char *yb = reinterpret_cast<const char *>(y);
    const char *sxb = reinterpret_cast<const char *>(sx);
    const char *syb = reinterpret_cast<const char *>(sy);
    if (op != kOpPairwise) { // the y side image is shared by all chunks
        const bool sym = op == kOpGramSym;
        if ((st = tc_image(in64, sym ? x : y, sym ? nx : ny, ly, d, ncy, kTcBN, t.b_tiles, t.kp, 1.0, sym ? sx : sy,
                           b_hi, b_lo, stream)))
            return st;
    }

    for (int64_t c = 0; c < t.nchunks; ++c) {
        const int64_t i0 = c * t.chunk, i1 = (i0 + t.chunk < nx) ? i0 + t.chunk : nx, nxc = i1 - i0;
        const int64_t a_tiles = (nxc * t.rows_x + kTcM - 1) / kTcM;
        if ((st = tc_image(in64, xb + i0 * lx * d * es, nxc, lx, d, t.rows_x, kTcM, a_tiles, t.kp, fs,
                           sx ? sxb + i0 * es : nullptr, a_hi, a_lo, stream)))
            return st;
        int64_t ny_rows;
        if (op == kOpPairwise) {
            ny_rows = nxc * ncy;
            if ((st = tc_image(in64, yb + i0 * ly * d * es, nxc, ly, d, ncy, kTcBN, (ny_rows + kTcBN - 1) / kTcBN,
                               t.kp, 1.0, sy ? syb + i0 * es : nullptr, b_hi, b_lo, stream)))
                return st;
        } else {
            ny_rows = (op == kOpGram ? ny : i1) * ncy;
        }
        TcGemmParams gp{};
        gp.a_hi = a_hi;
        gp.a_lo = a_lo;
        gp.b_hi = b_hi;
        gp.b_lo = b_lo;
        gp.mtiles = a_tiles;
        gp.ntiles = (ny_rows + kTcBN - 1) / kTcBN;
        gp.kp = t.kp;
        gp.mode = op == kOpPairwise ? kTcDiag : (op == kOpGramSym ? kTcLower : kTcAll);
        gp.m_rows = nxc * t.rows_x;
        gp.n_rows = ny_rows;
        gp.rows_x = t.rows_x;
        gp.rows_y = ncy;
        gp.npaths_x = nxc;
        gp.npaths_y = op == kOpPairwise ? nxc : (op == kOpGram ? ny : i1);
        gp.x0 = op == kOpGramSym ? i0 : 0;
        gp.out = ct;
        gp.ld = nxc * t.rows_x;
        gp.err = err;
        if ((st = tc_gemm(gp, stream))) return st;

        if ((st = consume_matrix(t, op, ct, false, gp.ld, err, i0, i1, nx, ny, ncx, ncy, d, order, out, out_ld,
                                 in64, precision, dtype, wsb, stream)))
            return st;
    }
    return SIGK_OK;
}


// ------------------------------------------------------------------ float64 increment matrix
// fp64 mode, Gram ops, dim >= kDgMinDim: the increments of all pairs from one
// FP64 GEMM on the CUDA cores (dgemm_inc.cuh), then the wavefront reads them;
// bitwise the results of the fused kernels, faster when the d FMAs per coarse
// cell dominate.  Workspace: a zero word (the consumers' error flag), boundary
// rows, the scaled differences of both sides, the matrix (x paths in chunks of
// at most kTcChunkBytes).
constexpr int kDgMinDim = 16;

// Layout of a float64 increment matrix plan; diffs: room for the scaled
// differences of both sides (the linear kernel's GEMM operands).
// The float64 increment GEMM over gp's matrix: pipelined (dgemm_inc_pipe_kernel,
// about 8 waves of 3 CTAs per SM, each CTA walking a share of the n tiles) for
// d <= 32, else one tile per CTA.  SIGK_NO_DGEMM_PIPE=1 selects the latter always.
int launch_dgemm_inc(const DgemmIncParams &gp, cudaStream_t stream)
{
    const int64_t mt = (gp.ld + kDgTile - 1) / kDgTile;
    int64_t nt = (gp.npaths_y * gp.ncy + kDgTile - 1) / kDgTile;
    if (mt > 0x7fffffffLL) return fail(SIGK_EUNSUPPORTED, "increment matrix too large");
    DgemmIncFn pipe = env_flag("SIGK_NO_DGEMM_PIPE") ? nullptr : get_dgemm_inc_pipe_kernel(gp.d);
    if (pipe) {
        const size_t smem = dgemm_inc_pipe_smem(gp.d);
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute((const void *)pipe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        }
        int64_t g = ((int64_t)sm_count() * 3 * 8 + mt - 1) / mt;
        if (g > nt) g = nt;
        if (g > 65535) g = 65535;
        if (g < 1) g = 1;
        pipe<<<dim3((unsigned)mt, (unsigned)g), 256, smem, stream>>>(gp);
    } else {
        if (nt > 65535) nt = 65535;
        get_dgemm_inc_kernel()<<<dim3((unsigned)mt, (unsigned)nt), 256, 0, stream>>>(gp);
    }
    count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "float64 increment GEMM launch");
}

// es: bytes per element of the increment matrix (8 for float64 cells, 4 for float32 cells); the chunk of x
// paths per launch and the matrix's share of the workspace follow it.
TcPlan mat64_layout(int op, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t d, int order, bool diffs,
                    size_t es = sizeof(double))
{
    TcPlan t{};
    const int64_t n = ncx << order, m = ncy << order;
    const int C = order >= 4 ? 8 : (1 << order);
    const int Rs = pick_rows(n);
    t.ok = true;
    t.stream = n <= 32 * Rs && m / C >= 32;
    t.R = Rs;
    t.O = order >= 4 ? 4 : order;
    t.nbands = (int)((n + 32 * Rs - 1) / (32 * Rs));
    size_t bnd_bytes = 0;
    if (!t.stream && t.nbands > 1) {
        t.bnd_stride = ((m + 1 + 31) / 32) * 32;
        bnd_bytes = align256((size_t)warp_cap() * (size_t)t.bnd_stride * sizeof(double));
    }
    t.rows_x = (ncx + 3) / 4 * 4;
    t.rows_y = ncy;
    const int64_t ny_paths = op == kOpGram ? ny : nx;
    const size_t per_x = (size_t)t.rows_x * (size_t)(ny_paths * ncy) * es;
    int64_t chunk = (int64_t)(tc_chunk_cap() / per_x);
    if (chunk < 1) chunk = 1;
    if (chunk > nx) chunk = nx;
    t.chunk = chunk;
    t.nchunks = (nx + chunk - 1) / chunk;
    t.err_off = 0;
    t.bnd_off = 256;
    t.a_off = t.bnd_off + bnd_bytes; // x differences
    t.b_off = t.a_off + (diffs ? align256((size_t)nx * ncx * d * sizeof(double)) : 0); // y differences
    t.ct_off = t.b_off + (diffs ? align256((size_t)ny_paths * ncy * d * sizeof(double)) : 0);
    t.ws_bytes = t.ct_off + align256((size_t)chunk * per_x);
    return t;
}

TcPlan make_mat64_plan(int op, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t d, int order)
{
    if (op == kOpPairwise || d < kDgMinDim || env_flag("SIGK_NO_DGEMM_INC")) return TcPlan{};
    // A Gram of order 2-3 whose lanes hold dx in registers runs faster on the two-entry register kernel,
    // which forms the dot products a step ahead of the cells (256 x 256, L = 64, d = 16, order 2: 1.97 vs
    // 2.19 ms; the same values).  Orders 0-1 (few cells a coarse column) and wider dx tiles keep the matrix.
    if (op == kOpGram && order >= 2 && order <= 3 && !env_flag("SIGK_NO_REG_DX")) {
        const int64_t n = ncx << order;
        const int Rs = pick_rows(n);
        int Dp = 2;
        while (Dp < d) Dp <<= 1;
        if (n <= 32 * Rs && rows_per_coarse_lane(Rs, order) * Dp <= 32 && ncy >= 32) return TcPlan{};
    }
    return mat64_layout(op, nx, ny, ncx, ncy, d, order, true);
}

// RBF / L1-RBF Grams (fp64 cells, dim <= kStaticMaxDim): the increments of
// all pairs straight from the path points (static_inc.cuh) into the same
// matrix layout, read by the same wavefront kernels.
constexpr int64_t kStaticMaxDim = 32;

TcPlan make_static_plan(int op, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t d, int order, int precision)
{
    if (op == kOpPairwise || d > kStaticMaxDim) return TcPlan{};
    const size_t es = cell_prec(precision) == SIGK_PREC_FP64 ? sizeof(double) : sizeof(float);
    return mat64_layout(op, nx, ny, ncx, ncy, d, order, false, es);
}

int run_pairs_mat64(const TcPlan &t, int op, const void *x, const void *y, int64_t nx, int64_t ny, int64_t lx,
                    int64_t ly, int64_t d, int dtype, int order, double static_scale, const void *sx, const void *sy,
                    void *out, int64_t out_ld, int precision, void *ws, cudaStream_t stream)
{
    int st;
    const bool in64 = dtype == SIGK_F64;
    const int64_t ncx = lx - 1, ncy = ly - 1;
    unsigned char *wsb = reinterpret_cast<unsigned char *>(ws);
    unsigned *err = reinterpret_cast<unsigned *>(wsb + t.err_off);
    double *dx = reinterpret_cast<double *>(wsb + t.a_off);
    double *dy = reinterpret_cast<double *>(wsb + t.b_off);
    double *mat = reinterpret_cast<double *>(wsb + t.ct_off);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    // scaled differences, as the fused path: static scale * 4^-order * scale_x on x, scale_y on y
    // (the symmetric Gram: both from x, scale_x on each side)
    DeltaFn delta = get_delta_kernel(true, in64);
    auto run_delta = [&](const void *src, int64_t npaths, int64_t len, double f, const void *sc, double *dst) -> int {
        const int64_t total = npaths * (len - 1) * d;
        int64_t blocks = (total + 255) / 256;
        if (blocks > (int64_t)sm_count() * 8) blocks = (int64_t)sm_count() * 8;
        delta<<<(unsigned)blocks, 256, 0, stream>>>(src, npaths, len, d, d, f, sc, dst);
        count_launch();
        cudaError_t e2 = cudaGetLastError();
        return e2 == cudaSuccess ? SIGK_OK : cuda_fail(e2, "delta kernel launch");
    };
    const double fs = static_scale * std::ldexp(1.0, -2 * order);
    const bool sym = op == kOpGramSym;
    if ((st = run_delta(x, nx, lx, fs, sx, dx))) return st;
    if (sym) {
        if (fs == 1.0)
            dy = dx;
        else if ((st = run_delta(x, nx, lx, 1.0, sx, dy)))
            return st;
    } else if ((st = run_delta(y, ny, ly, 1.0, sy, dy))) {
        return st;
    }
    for (int64_t c = 0; c < t.nchunks; ++c) {
        const int64_t i0 = c * t.chunk, i1 = (i0 + t.chunk < nx) ? i0 + t.chunk : nx, nxc = i1 - i0;
        DgemmIncParams gp{};
        gp.dx = dx + i0 * d * ncx;
        gp.dy = dy;
        gp.npaths_x = nxc;
        gp.ncx = ncx;
        gp.rows_x = t.rows_x;
        gp.npaths_y = sym ? i1 : ny;
        gp.ncy = ncy;
        gp.d = d;
        gp.mode = sym ? kTcLower : kTcAll;
        gp.x0 = i0;
        gp.out = mat;
        gp.ld = nxc * t.rows_x;
        if ((st = launch_dgemm_inc(gp, stream))) return st;
        if ((st = consume_matrix(t, op, mat, true, gp.ld, err, i0, i1, nx, ny, ncx, ncy, d, order, out, out_ld, in64,
                                 precision, dtype, wsb, stream)))
            return st;
    }
    return SIGK_OK;
}

int run_pairs_static(const TcPlan &t, int op, int kind, double param, const void *x, const void *y, int64_t nx,
                     int64_t ny, int64_t lx, int64_t ly, int64_t d, int dtype, int order, const void *sx,
                     const void *sy, void *out, int64_t out_ld, int precision, void *ws, cudaStream_t stream)
{
    int st;
    const bool in64 = dtype == SIGK_F64;
    const size_t es = in64 ? 8 : 4;
    const int64_t ncx = lx - 1, ncy = ly - 1;
    unsigned char *wsb = reinterpret_cast<unsigned char *>(ws);
    unsigned *err = reinterpret_cast<unsigned *>(wsb + t.err_off);
    void *mat = wsb + t.ct_off; // float64 elements for float64 cells, float32 for float32 cells
    const bool f64cells = cell_prec(precision) == SIGK_PREC_FP64;
    StaticIncFn fn = get_static_inc_kernel(kind, d, f64cells);
    if (!fn) return fail(SIGK_EUNSUPPORTED, "no static-kernel increment kernel for kind %d, dim %lld", kind,
                         (long long)d);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    const bool sym = op == kOpGramSym;
    for (int64_t c = 0; c < t.nchunks; ++c) {
        const int64_t i0 = c * t.chunk, i1 = (i0 + t.chunk < nx) ? i0 + t.chunk : nx, nxc = i1 - i0;
        StaticIncParams sp{};
        sp.x = reinterpret_cast<const unsigned char *>(x) + (size_t)i0 * lx * d * es;
        sp.y = sym ? x : y;
        sp.in64 = in64;
        sp.npaths_x = nxc;
        sp.lx = lx;
        sp.rows_x = t.rows_x;
        sp.npaths_y = sym ? i1 : ny;
        sp.ly = ly;
        sp.d = d;
        sp.inv_param = 1.0 / param;
        sp.f = std::ldexp(1.0, -2 * order);
        sp.sx = sx ? reinterpret_cast<const unsigned char *>(sx) + (size_t)i0 * es : nullptr;
        sp.sy = sym ? sx : sy;
        sp.mode = sym ? kTcLower : kTcAll;
        sp.x0 = i0;
        sp.out = mat;
        sp.ld = nxc * t.rows_x;
        const int64_t warps = (nxc * lx + kStRowsPerWarp - 1) / kStRowsPerWarp;
        const int64_t bx = (warps + kStWarps - 1) / kStWarps;
        int64_t by = (sp.npaths_y * ncy + kStTileN - 1) / kStTileN;
        if (by > 65535) by = 65535;
        if (bx > 0x7fffffffLL) return fail(SIGK_EUNSUPPORTED, "increment matrix too large");
        fn<<<dim3((unsigned)bx, (unsigned)by), kStWarps * 32, 0, stream>>>(sp);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "static-kernel increment launch");
        if ((st = consume_matrix(t, op, mat, f64cells, sp.ld, err, i0, i1, nx, ny, ncx, ncy, d, order, out, out_ld,
                                 in64, precision, dtype, wsb, stream)))
            return st;
    }
    return SIGK_OK;
}

// ------------------------------------------------------------------ backward pass
// Gradients of sum w * k with respect to the points (grad.cuh).  Pairs are
// processed in chunks of x paths so that the per-cell derivatives D (one
// float64 per fine cell of every pair in the chunk) and the chunk's increment
// matrix stay under kGradChunkBytes (SIGK_GRAD_CHUNK_MB overrides).
// Workspace: zero word | x, y differences | dk/d(x diff), dk/d(y diff) |
// partial sums of the x contraction | increment matrix | D | boundary rows.
constexpr size_t kGradChunkBytes = 8ull << 30;
constexpr int kGradMaxOrder = 4;
constexpr int64_t kGradSlices = 64;

struct GradPlan {
    bool ok = false;
    int R = 0, O = 0, nb = 0;
    int64_t rows_x = 0, chunk = 0, nchunks = 0, slice = 0, nslices = 0;
    size_t dx_off = 0, dy_off = 0, gdx_off = 0, gdy_off = 0, part_off = 0, mat_off = 0, d_off = 0, bnd_off = 0,
           xt_off = 0, yt_off = 0, ws_bytes = 0;
};

GradPlan make_grad_plan(int op, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t d, int order)
{
    GradPlan g;
    if (order > kGradMaxOrder) return g;
    const int64_t n = ncx << order, m = ncy << order;
    // rows per lane: the smallest power of two with 32R >= n, at most 8 (bands of 256 rows keep the
    // adjoint's registers near 128), and at least 2^order (a lane holds whole coarse rows)
    int R = 1;
    while (R < 8 && 32 * R < n) R *= 2;
    while (R < (1 << order)) R *= 2;
    g.R = R;
    g.O = order;
    g.nb = (int)((n + 32 * R - 1) / (32 * R));
    g.rows_x = (ncx + 3) / 4 * 4;
    const size_t dbytes = (size_t)g.nb * grad_band_doubles((int)m, R) * sizeof(double);
    const size_t bbytes = 2 * (size_t)(m + 2) * sizeof(double);
    const size_t mbytes = (size_t)ncy * g.rows_x * sizeof(double);
    const int64_t items_per_x = op == kOpPairwise ? 1 : ny;
    const size_t per_x = (size_t)items_per_x * (dbytes + bbytes + mbytes);
    size_t cap = kGradChunkBytes;
    if (const char *v = getenv("SIGK_GRAD_CHUNK_MB")) {
        const long long mb = atoll(v);
        if (mb > 0) cap = (size_t)mb << 20;
    }
    int64_t chunk = (int64_t)(cap / per_x);
    if (chunk < 1) chunk = 1;
    if (chunk > nx) chunk = nx;
    g.chunk = chunk;
    g.nchunks = (nx + chunk - 1) / chunk;
    const int64_t ncols = op == kOpPairwise ? ncy : ny * ncy;
    g.slice = (ncols + kGradSlices - 1) / kGradSlices;
    if (g.slice < 32) g.slice = ncols < 32 ? ncols : 32;
    g.nslices = (ncols + g.slice - 1) / g.slice;
    const int64_t ny_paths = op == kOpPairwise ? nx : ny;
    size_t off = 256;
    g.dx_off = off;
    off += align256((size_t)nx * d * ncx * sizeof(double));
    g.dy_off = off;
    off += align256((size_t)ny_paths * d * ncy * sizeof(double));
    g.gdx_off = off;
    off += align256((size_t)nx * ncx * d * sizeof(double));
    g.gdy_off = off;
    off += align256((size_t)ny_paths * ncy * d * sizeof(double));
    g.part_off = off;
    off += align256((size_t)g.nslices * chunk * g.rows_x * d * sizeof(double));
    g.xt_off = off; // the chunk's x differences in row layout
    off += align256((size_t)chunk * g.rows_x * d * sizeof(double));
    g.yt_off = off; // all y differences in row layout
    off += align256((size_t)ny_paths * ncy * d * sizeof(double));
    g.mat_off = off;
    off += align256((size_t)chunk * items_per_x * mbytes);
    g.d_off = off;
    off += align256((size_t)chunk * items_per_x * dbytes);
    g.bnd_off = off;
    off += align256((size_t)chunk * items_per_x * bbytes);
    g.ws_bytes = off;
    g.ok = true;
    return g;
}

int run_backward(const GradPlan &g, int op, const void *x, const void *y, int64_t nx, int64_t ny, int64_t lx,
                 int64_t ly, int64_t d, int dtype, int order, double static_scale, const void *sx, const void *sy,
                 const void *w, void *gx, void *gy, void *ws, cudaStream_t stream)
{
    const bool in64 = dtype == SIGK_F64;
    const int64_t ncx = lx - 1, ncy = ly - 1;
    unsigned char *wsb = reinterpret_cast<unsigned char *>(ws);
    double *dx = reinterpret_cast<double *>(wsb + g.dx_off);
    double *dy = reinterpret_cast<double *>(wsb + g.dy_off);
    double *gdx = reinterpret_cast<double *>(wsb + g.gdx_off);
    double *gdy = reinterpret_cast<double *>(wsb + g.gdy_off);
    double *part = reinterpret_cast<double *>(wsb + g.part_off);
    double *mat = reinterpret_cast<double *>(wsb + g.mat_off);
    const int64_t ny_paths = op == kOpPairwise ? nx : ny;
    cudaError_t e = cudaMemsetAsync(gdy, 0, (size_t)ny_paths * ncy * d * sizeof(double), stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    DeltaFn delta = get_delta_kernel(true, in64);
    auto run_delta = [&](const void *src, int64_t npaths, int64_t len, double f, const void *sc, double *dst) -> int {
        const int64_t total = npaths * (len - 1) * d;
        int64_t blocks = (total + 255) / 256;
        if (blocks > (int64_t)sm_count() * 8) blocks = (int64_t)sm_count() * 8;
        delta<<<(unsigned)blocks, 256, 0, stream>>>(src, npaths, len, d, d, f, sc, dst);
        count_launch();
        cudaError_t e2 = cudaGetLastError();
        return e2 == cudaSuccess ? SIGK_OK : cuda_fail(e2, "delta kernel launch");
    };
    const double fs = static_scale * std::ldexp(1.0, -2 * order);
    int st;
    if ((st = run_delta(x, nx, lx, fs, sx, dx))) return st;
    if ((st = run_delta(y, ny_paths, ly, 1.0, sy, dy))) return st;
    double *dxt = reinterpret_cast<double *>(wsb + g.xt_off);
    double *dyt = reinterpret_cast<double *>(wsb + g.yt_off);
    auto run_rows = [&](const double *src, int64_t npaths, int64_t nc, int64_t rows, double *dst) -> int {
        const int64_t total = npaths * rows * d;
        int64_t blocks = (total + 255) / 256;
        if (blocks > (int64_t)sm_count() * 8) blocks = (int64_t)sm_count() * 8;
        get_grad_aux_kernels().rows<<<(unsigned)blocks, 256, 0, stream>>>(src, npaths, nc, rows, d, dst);
        count_launch();
        cudaError_t e2 = cudaGetLastError();
        return e2 == cudaSuccess ? SIGK_OK : cuda_fail(e2, "row-layout launch");
    };
    if ((st = run_rows(dy, ny_paths, ncy, ncy, dyt))) return st;
    GradFns kf = get_grad_kernels(g.R, g.O);
    GradAuxFns aux = get_grad_aux_kernels();
    if (!kf.fwd || !kf.bwd) return fail(SIGK_EUNSUPPORTED, "no backward kernels for R=%d order=%d", g.R, g.O);
    int nbf = 0, nbb = 0;
    if ((st = blocks_per_sm((const void *)kf.fwd, 0, &nbf)) || (st = blocks_per_sm((const void *)kf.bwd, 0, &nbb)))
        return st;
    auto launched = [&](const char *what) -> int {
        count_launch();
        cudaError_t e2 = cudaGetLastError();
        return e2 == cudaSuccess ? SIGK_OK : cuda_fail(e2, what);
    };
    for (int64_t c = 0; c < g.nchunks; ++c) {
        const int64_t i0 = c * g.chunk, i1 = (i0 + g.chunk < nx) ? i0 + g.chunk : nx, nxc = i1 - i0;
        const int64_t items = op == kOpPairwise ? nxc : nxc * ny;
        const int64_t ld = op == kOpPairwise ? g.rows_x : nxc * g.rows_x;
        // increments of the chunk's pairs, in the layout the wavefronts read
        if (op == kOpPairwise) {
            const int64_t total = items * ncy * g.rows_x;
            int64_t blocks = (total + 255) / 256;
            if (blocks > (int64_t)sm_count() * 16) blocks = (int64_t)sm_count() * 16;
            aux.pair_inc<<<(unsigned)blocks, 256, 0, stream>>>(dx, dy, items, i0, ncx, ncy, g.rows_x, d, mat);
            if ((st = launched("pairwise increment launch"))) return st;
        } else {
            DgemmIncParams gp{};
            gp.dx = dx + i0 * d * ncx;
            gp.dy = dy;
            gp.npaths_x = nxc;
            gp.ncx = ncx;
            gp.rows_x = g.rows_x;
            gp.npaths_y = ny;
            gp.ncy = ncy;
            gp.d = d;
            gp.mode = kTcAll;
            gp.x0 = i0;
            gp.out = mat;
            gp.ld = ld;
            if ((st = launch_dgemm_inc(gp, stream))) return st;
        }
        if ((st = run_rows(dx + i0 * d * ncx, nxc, ncx, g.rows_x, dxt))) return st;
        GradParams gp{};
        gp.op = op;
        gp.mat = mat;
        gp.ld = ld;
        gp.rows_x = g.rows_x;
        gp.ncx = ncx;
        gp.ncy = ncy;
        gp.order = order;
        gp.nitems = items;
        gp.ny = ny;
        gp.w = w;
        gp.in64 = in64;
        gp.x0 = i0;
        gp.dbuf = reinterpret_cast<double *>(wsb + g.d_off);
        gp.bnd = reinterpret_cast<double *>(wsb + g.bnd_off);
        auto grid_for = [&](int nb) -> unsigned {
            int64_t warps = (int64_t)sm_count() * nb * kWarpsPerBlock;
            if (warps > items) warps = items;
            return (unsigned)((warps + kWarpsPerBlock - 1) / kWarpsPerBlock);
        };
        kf.fwd<<<grid_for(nbf), kWarpsPerBlock * 32, 0, stream>>>(gp);
        if ((st = launched("backward forward-pass launch"))) return st;
        kf.bwd<<<grid_for(nbb), kWarpsPerBlock * 32, 0, stream>>>(gp);
        if ((st = launched("adjoint launch"))) return st;
        // contractions: x side (partial slices, then their ordered sum) and y side
        GradContractParams cp{};
        cp.op = op;
        cp.mat = mat;
        cp.ld = ld;
        cp.rows_x = g.rows_x;
        cp.ncx = ncx;
        cp.ncy = ncy;
        cp.nrows_m = op == kOpPairwise ? items * g.rows_x : ld;
        cp.ncols_n = op == kOpPairwise ? ncy : ny * ncy;
        cp.dxt = dxt;
        cp.dyt = dyt;
        cp.d = d;
        cp.part = part;
        cp.slice = g.slice;
        cp.gdy = gdy;
        cp.x0 = i0;
        const int64_t nsl = (cp.ncols_n + g.slice - 1) / g.slice;
        if (gx) {
            aux.gx<<<dim3((unsigned)((cp.nrows_m + 127) / 128), (unsigned)nsl), 128, 0, stream>>>(cp);
            if ((st = launched("x contraction launch"))) return st;
            const int64_t tot = cp.nrows_m * d;
            aux.reduce<<<(unsigned)((tot + 255) / 256), 256, 0, stream>>>(part, nsl, cp.nrows_m, g.rows_x, ncx, d, i0,
                                                                        gdx);
            if ((st = launched("x reduction launch"))) return st;
        }
        if (gy) {
            if (op == kOpPairwise) {
                const int64_t rows = items * ncy;
                aux.gy<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, stream>>>(cp);
            } else {
                aux.gy_gram<<<(unsigned)((ny * ncy + kGyRows - 1) / kGyRows), 256, 0, stream>>>(cp);
            }
            if ((st = launched("y contraction launch"))) return st;
        }
    }
    if (gx) {
        const int64_t tot = nx * lx * d;
        aux.points<<<(unsigned)((tot + 255) / 256), 256, 0, stream>>>(gdx, nx, lx, d, fs, sx, in64, gx);
        if ((st = launched("x point-gradient launch"))) return st;
    }
    if (gy) {
        const int64_t tot = ny_paths * ly * d;
        aux.points<<<(unsigned)((tot + 255) / 256), 256, 0, stream>>>(gdy, ny_paths, ly, d, 1.0, sy, in64, gy);
        if ((st = launched("y point-gradient launch"))) return st;
    }
    return SIGK_OK;
}

// Backward over caller's increments: per chunk of pairs, the scaled increments
// in per-pair blocks, then the same forward / adjoint kernels (pairwise
// layout, weight of pair b = grad_out[b]), then dk/dc * scales back out.
GradPlan make_grad_inc_plan(int64_t npairs, int64_t ncx, int64_t ncy, int order)
{
    GradPlan g = make_grad_plan(kOpPairwise, npairs, npairs, ncx, ncy, 1, order);
    if (!g.ok) return g;
    // only the matrix, the per-step records and the boundary rows are used
    const int64_t m = ncy << order;
    const size_t dbytes = (size_t)g.nb * grad_band_doubles((int)m, g.R) * sizeof(double);
    const size_t bbytes = 2 * (size_t)(m + 2) * sizeof(double);
    const size_t mbytes = (size_t)ncy * g.rows_x * sizeof(double);
    size_t off = 256;
    g.mat_off = off;
    off += align256((size_t)g.chunk * mbytes);
    g.d_off = off;
    off += align256((size_t)g.chunk * dbytes);
    g.bnd_off = off;
    off += align256((size_t)g.chunk * bbytes);
    g.ws_bytes = off;
    return g;
}

int run_backward_inc(const GradPlan &g, const void *inc, int64_t npairs, int64_t ncx, int64_t ncy, int64_t s0,
                     int64_t s1, int64_t s2, int dtype, int order, const void *sx, const void *sy, const void *w,
                     void *ginc, int64_t g0, int64_t g1, int64_t g2, void *ws, cudaStream_t stream)
{
    const bool in64 = dtype == SIGK_F64;
    unsigned char *wsb = reinterpret_cast<unsigned char *>(ws);
    double *mat = reinterpret_cast<double *>(wsb + g.mat_off);
    GradFns kf = get_grad_kernels(g.R, g.O);
    GradAuxFns aux = get_grad_aux_kernels();
    if (!kf.fwd || !kf.bwd) return fail(SIGK_EUNSUPPORTED, "no backward kernels for R=%d order=%d", g.R, g.O);
    int st, nbf = 0, nbb = 0;
    if ((st = blocks_per_sm((const void *)kf.fwd, 0, &nbf)) || (st = blocks_per_sm((const void *)kf.bwd, 0, &nbb)))
        return st;
    auto launched = [&](const char *what) -> int {
        count_launch();
        cudaError_t e2 = cudaGetLastError();
        return e2 == cudaSuccess ? SIGK_OK : cuda_fail(e2, what);
    };
    for (int64_t c = 0; c < g.nchunks; ++c) {
        const int64_t b0 = c * g.chunk, b1 = (b0 + g.chunk < npairs) ? b0 + g.chunk : npairs, items = b1 - b0;
        const int64_t total = items * ncy * g.rows_x;
        int64_t blocks = (total + 255) / 256;
        if (blocks > (int64_t)sm_count() * 16) blocks = (int64_t)sm_count() * 16;
        aux.inc_blocks<<<(unsigned)blocks, 256, 0, stream>>>(inc, in64, s0, s1, s2, items, b0, ncx, ncy, g.rows_x,
                                                             sx, sy, mat, nullptr, 0);
        if ((st = launched("increment blocks launch"))) return st;
        GradParams gp{};
        gp.op = kOpPairwise;
        gp.mat = mat;
        gp.ld = g.rows_x;
        gp.rows_x = g.rows_x;
        gp.ncx = ncx;
        gp.ncy = ncy;
        gp.order = order;
        gp.nitems = items;
        gp.ny = npairs;
        gp.w = w;
        gp.in64 = in64;
        gp.x0 = b0;
        gp.dbuf = reinterpret_cast<double *>(wsb + g.d_off);
        gp.bnd = reinterpret_cast<double *>(wsb + g.bnd_off);
        auto grid_for = [&](int nb) -> unsigned {
            int64_t warps = (int64_t)sm_count() * nb * kWarpsPerBlock;
            if (warps > items) warps = items;
            return (unsigned)((warps + kWarpsPerBlock - 1) / kWarpsPerBlock);
        };
        kf.fwd<<<grid_for(nbf), kWarpsPerBlock * 32, 0, stream>>>(gp);
        if ((st = launched("backward forward-pass launch"))) return st;
        kf.bwd<<<grid_for(nbb), kWarpsPerBlock * 32, 0, stream>>>(gp);
        if ((st = launched("adjoint launch"))) return st;
        aux.inc_blocks<<<(unsigned)blocks, 256, 0, stream>>>(nullptr, in64, g0, g1, g2, items, b0, ncx, ncy, g.rows_x,
                                                             sx, sy, mat, ginc, 1);
        if ((st = launched("increment gradient launch"))) return st;
    }
    return SIGK_OK;
}

int run_pairs(int op, const void *x, const void *y, int64_t nx, int64_t ny, int64_t lx, int64_t ly, int64_t d,
              int dtype, int order, double static_scale, const void *sx, const void *sy, void *out, int64_t out_ld,
              int precision, void *ws, size_t ws_bytes, cudaStream_t stream)
{
    int st = check_common(dtype, precision, order);
    if (st) return st;
    if (nx < 1 || ny < 1) return fail(SIGK_EINVAL, "path counts must be >= 1 (got %lld, %lld)", (long long)nx,
                                      (long long)ny);
    if (lx < 2 || ly < 2) return fail(SIGK_EINVAL, "path lengths must be >= 2 (got %lld, %lld)", (long long)lx,
                                      (long long)ly);
    if (d < 1) return fail(SIGK_EINVAL, "dim must be >= 1");
    if ((st = check_dev(x, "x", false)) || (st = check_dev(y, "y", false)) || (st = check_dev(out, "out", false)) ||
        (st = check_dev(sx, "scale_x", true)) || (st = check_dev(sy, "scale_y", true)))
        return st;
    if (is_tc(precision)) {
        const FtPlan f = make_fused_plan(op, nx, ny, lx - 1, ly - 1, d, order, precision);
        if (f.ok) {
            if (!ws || ws_bytes < f.ws_bytes)
                return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", f.ws_bytes, ws ? ws_bytes : 0);
            if (((uintptr_t)ws & 255) != 0) return fail(SIGK_EINVAL, "workspace must be 256-byte aligned");
            return run_pairs_fused(f, x, y, nx, ny, lx, ly, d, dtype, order, static_scale, sx, sy, out, out_ld, ws,
                                   stream);
        }
        TcPlan t = make_tc_plan(op, nx, ny, lx - 1, ly - 1, d, order, tsize_of(precision));
        if (t.ok) {
            if (!ws || ws_bytes < t.ws_bytes)
                return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", t.ws_bytes, ws ? ws_bytes : 0);
            if (((uintptr_t)ws & 255) != 0) return fail(SIGK_EINVAL, "workspace must be 256-byte aligned");
            return run_pairs_tc(t, op, x, y, nx, ny, lx, ly, d, dtype, order, static_scale, sx, sy, out, out_ld,
                                precision, ws, stream);
        }
        precision = cell_prec(precision); // shapes outside the TC plan: CUDA-core increments, same cells
    }
    if (precision == SIGK_PREC_FP64) {
        TcPlan t = make_mat64_plan(op, nx, ny, lx - 1, ly - 1, d, order);
        if (t.ok) {
            if (!ws || ws_bytes < t.ws_bytes)
                return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", t.ws_bytes, ws ? ws_bytes : 0);
            if (((uintptr_t)ws & 255) != 0) return fail(SIGK_EINVAL, "workspace must be 256-byte aligned");
            return run_pairs_mat64(t, op, x, y, nx, ny, lx, ly, d, dtype, order, static_scale, sx, sy, out, out_ld,
                                   precision, ws, stream);
        }
    }
    const size_t ts = tsize_of(precision);
    const int64_t nitems = op == kOpPairwise ? nx : (op == kOpGram ? nx * ny : nx * (nx + 1) / 2);
    Plan pl = make_plan(op, nx, ny, lx - 1, ly - 1, d, order, ts, false);
    if ((st = check_ws(pl, ws, ws_bytes))) return st;
    const bool in64 = dtype == SIGK_F64;
    const bool f64 = precision == SIGK_PREC_FP64;

    {
        unsigned char *wsb = reinterpret_cast<unsigned char *>(ws);
        void *dx = wsb + pl.dx_off;
        void *dy = wsb + pl.dy_off;
        DeltaFn delta = get_delta_kernel(f64, in64);
        const int nsm = sm_count();
        const int64_t dp = pl.stream && pl.D ? pl.D : d;
        auto run_delta = [&](const void *src, int64_t npaths, int64_t len, double f, const void *sc,
                             void *dst) -> int {
            const int64_t total = npaths * (len - 1) * dp;
            int64_t blocks = (total + 255) / 256;
            if (blocks > (int64_t)nsm * 8) blocks = (int64_t)nsm * 8;
            delta<<<(unsigned)blocks, 256, 0, stream>>>(src, npaths, len, d, dp, f, sc, dst);
            count_launch();
            cudaError_t e = cudaGetLastError();
            return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "delta kernel launch");
        };
        // static scale * 4^-order and scale_x go into dX, scale_y into dY; the
        // symmetric Gram reads one buffer for both sides, scaled by scale_x
        const double fs = static_scale * std::ldexp(1.0, -2 * order);
        if (op == kOpGramSym) {
            // f goes on the row side only, so a second buffer is needed unless f == 1
            if (fs == 1.0) {
                if ((st = run_delta(x, nx, lx, 1.0, sx, dx))) return st;
                dy = dx;
            } else {
                if ((st = run_delta(x, nx, lx, fs, sx, dx))) return st;
                if ((st = run_delta(x, nx, lx, 1.0, sx, dy))) return st;
            }
        } else {
            if ((st = run_delta(x, nx, lx, fs, sx, dx))) return st;
            if ((st = run_delta(y, ny, ly, 1.0, sy, dy))) return st;
        }

        if (!pl.stream) { // one pair per warp, any number of bands
            PairParams p{};
            p.op = op;
            p.x = x;
            p.y = y;
            p.dx = dx;
            p.dy = dy;
            p.nx = nx;
            p.ny = ny;
            p.ncx = lx - 1;
            p.ncy = ly - 1;
            p.d = d;
            p.order = order;
            p.fscale = 1.0; // folded into the differences
            p.out = out;
            p.out_ld = out_ld;
            p.nitems = nitems;
            p.bnd = pl.nbands > 1 ? ws : nullptr;
            p.bnd_stride = pl.bnd_stride;
            p.stage_smem = pl.stage_bytes_per_warp > 0;
            PairFn fn = pick_pair(precision, dtype, kPairDelta, pl.R, pl.O);
            return launch(fn, p, p.nitems, pl.stage_bytes_per_warp * kWarpsPerBlock, stream);
        }

        StreamParams sp{};
        sp.op = op;
        sp.in64 = in64;
        sp.dx = dx;
        sp.dy = dy;
        sp.nx = nx;
        sp.ny = ny;
        sp.ncx = lx - 1;
        sp.ncy = ly - 1;
        sp.d = d;
        sp.dp = dp;
        sp.order = order;
        sp.out = out;
        sp.out_ld = out_ld;
        sp.nitems = nitems;
        // float32 cells with register dx: two pairs per lane on paired instructions
        const bool paired = !f64 && pl.D && nitems >= 2 && !env_flag("SIGK_NO_PAIRED_F32");
        // float64 cells of a Gram with register dx: two entries of one x path per lane
        StreamFn dual_fn = (f64 && pl.D && op == kOpGram && ny >= 2 && !env_flag("SIGK_NO_DUAL_F64"))
                               ? get_stream_reg_kernel_f64x2(pl.R, pl.O, pl.D)
                               : nullptr;
        const bool dual = dual_fn != nullptr;
        StreamFn fn = paired  ? get_stream_reg_kernel_f32x2(pl.R, pl.O, pl.D)
                      : dual  ? dual_fn
                      : pl.D ? get_stream_reg_kernel(f64, pl.R, pl.O, pl.D)
                             : get_stream_smem_kernel(f64, pl.R, pl.O);
        if (!fn) return fail(SIGK_EUNSUPPORTED, "no stream kernel for R=%d O=%d D=%d", pl.R, pl.O, pl.D);
        const size_t smem = pl.stage_bytes_per_warp * kWarpsPerBlock;
        int nb = 0;
        if ((st = blocks_per_sm((const void *)fn, smem, &nb))) return st;
        int64_t nwarps = (int64_t)nsm * nb * kWarpsPerBlock;
        const int64_t units = paired ? (nitems + 1) / 2 : dual ? nx * ((ny + 1) / 2) : nitems; // pipeline slots
        if (nwarps > units) nwarps = units;
        sp.per_warp = (units + nwarps - 1) / nwarps;
        if (paired) sp.per_warp *= 2; // an even run per warp: no half-empty slot but the last warp's
        if (dual) sp.nitems = units;  // the dual kernel walks entry pairs
        const int64_t used = (sp.nitems + sp.per_warp - 1) / sp.per_warp;
        const int64_t blocks = (used + kWarpsPerBlock - 1) / kWarpsPerBlock;
        fn<<<(unsigned)blocks, kWarpsPerBlock * 32, smem, stream>>>(sp);
        count_launch();
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "stream kernel launch");
    }
}

// Normalisation plan: the increment source (a shared-memory tile of the
// path's coarse increments when it fits, else precomputed differences, or the
// caller's increments), the variant, shared memory and workspace layout
// (boundary rows for multi-band paths, then the float64 differences).
constexpr size_t kNormTileBytesPerWarp = 48 * 1024;

struct NormPlan {
    int mode, R, O, nbands;
    int64_t tile_pitch, bnd_stride;
    size_t smem_per_warp, bnd_bytes, dx_off, ws_bytes;
    // pipelined kernel (one CTA per path, `nw` bands as warps): its shared memory per CTA and the
    // workspace offsets of the progress counters, the wait flag and the band rows
    bool pipe;
    int nw;
    size_t smem_cta, prog_off, err_off;
};

constexpr size_t kNormPipeSmemBytes = 160 * 1024;

NormPlan norm_plan(int64_t n, int64_t nc, int64_t d, int order, bool from_inc)
{
    NormPlan q{};
    const int64_t tile_pitch = nc | 1; // odd pitch: neighbouring lanes' rows fall in different banks
    const size_t tile = (size_t)nc * (size_t)tile_pitch * sizeof(double);
    if (from_inc)
        q.mode = kNormGiven;
    else if (tile <= kNormTileBytesPerWarp && !env_flag("SIGK_NO_NORM_TILE"))
        q.mode = kNormTile;
    else
        q.mode = kNormDelta;
    // only the difference mode stages rows of dx (and may shrink R to fit them)
    Plan pl = make_plan(SIGK_OP_NORMALIZE, n, n, nc, nc, d, order, 8, q.mode != kNormDelta);
    q.R = pl.R;
    q.O = pl.O;
    q.nbands = pl.nbands;
    q.bnd_stride = pl.bnd_stride;
    q.bnd_bytes = align256(pl.ws_bytes);
    q.tile_pitch = tile_pitch;
    q.smem_per_warp = q.mode == kNormTile ? tile : q.mode == kNormDelta ? pl.stage_bytes_per_warp : 0;
    q.dx_off = q.bnd_bytes;
    q.ws_bytes = from_inc ? q.bnd_bytes : q.dx_off + align256((size_t)n * (size_t)d * (size_t)nc * sizeof(double));

    // Pipelined variant (one CTA per path, R = 2 rows per lane grown until the bands fit one CTA).
    // Measured on B200 it wins only where it can hold the path's increment tile in shared memory
    // for the whole CTA while the one-warp-per-path kernel cannot (tile above 48 KB) and the
    // increments are expensive to re-form (d >= 16): N=32 L=128 d=32 o=1, 1.64 ms vs 6.58 ms.
    // Elsewhere its band hand-offs cost more than they save (N=512 L=64 d=16 o=1: 0.74 vs 0.29 ms;
    // N=8 L=256 d=8 o=2: 8.5 vs 5.3 ms), so it is used for that case only (SIGK_NORM_PIPE=1 forces
    // it when possible, SIGK_NO_NORM_PIPE=1 disables it).
    const int64_t nref = nc << order;
    int R = 2;
    while (R < 16 && (nref + 32 * R - 1) / (32 * R) > kNormPipeMaxWarps) R <<= 1;
    const int64_t nw = (nref + 32 * R - 1) / (32 * R);
    const bool wins = !from_inc && d >= 16 && tile > kNormTileBytesPerWarp && tile <= kNormPipeSmemBytes;
    if (nw >= 2 && nw <= kNormPipeMaxWarps && (wins || env_flag("SIGK_NORM_PIPE")) && !env_flag("SIGK_NO_NORM_PIPE")) {
        const int rc = rows_per_coarse_lane(R, order);
        int mode = q.mode;
        size_t smem = 0;
        if (mode == kNormTile || mode == kNormDelta) {
            // one shared tile per CTA when it fits, else per-warp staged differences (or none)
            mode = (tile <= kNormPipeSmemBytes && !env_flag("SIGK_NO_NORM_TILE")) ? kNormTile : kNormDelta;
            if (mode == kNormTile) {
                smem = tile;
            } else {
                const size_t st = (size_t)rc * (size_t)d * 32 * sizeof(double) * (size_t)nw;
                smem = st <= kNormPipeSmemBytes ? st : 0;
            }
        }
        const int64_t m = nc << order;
        q.pipe = true;
        q.mode = mode;
        q.R = R;
        q.nw = (int)nw;
        q.smem_cta = smem;
        q.bnd_stride = ((m + 1 + 31) / 32) * 32;
        q.prog_off = 0;
        q.err_off = align256((size_t)n * kNormPipeMaxWarps * sizeof(int));
        q.bnd_bytes = q.err_off + 256; // counters and flag, zeroed before each launch
        const size_t rows = align256((size_t)n * (size_t)(nw - 1) * (size_t)q.bnd_stride * sizeof(double));
        q.dx_off = q.bnd_bytes + rows;
        q.ws_bytes = from_inc ? q.dx_off
                              : q.dx_off + align256((size_t)n * (size_t)d * (size_t)nc * sizeof(double));
    }
    return q;
}

} // namespace
} // namespace sigk

using namespace sigk;

extern "C" {

const char *sigk_version(void) { return "sigk 0.1.0 sm_100a"; }

const char *sigk_last_error_string(void) { return g_last_error.c_str(); }

uint64_t sigk_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int64_t sigk_set_wait_limit(int64_t polls)
{
    return (int64_t)g_wait_limit.exchange(polls < 0 ? -1 : (long long)polls, std::memory_order_relaxed);
}

size_t sigk_workspace_size(int op, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y, int64_t dim, int order,
                           int dtype, int precision)
{
    (void)dtype;
    if (len_x < 2 || len_y < 2 || order < 0 || order > 12 || dim < 0 || n_x < 1 || n_y < 1) return 0;
    if (op == SIGK_OP_NORMALIZE) precision = SIGK_PREC_FP64;
    if (op == SIGK_OP_GRAM_SYM || op == SIGK_OP_NORMALIZE) {
        len_y = len_x;
        n_y = n_x;
    }
    if (op == SIGK_OP_PAIRWISE) n_y = n_x;
    if (op == SIGK_OP_NORMALIZE) return norm_plan(n_x, len_x - 1, dim > 0 ? dim : 1, order, dim == 0).ws_bytes;
    if (is_tc(precision) && dim > 0) {
        const int kop = op == SIGK_OP_PAIRWISE ? kOpPairwise : op == SIGK_OP_GRAM ? kOpGram : kOpGramSym;
        const FtPlan f = make_fused_plan(kop, n_x, n_y, len_x - 1, len_y - 1, dim, order, precision);
        if (f.ok) return f.ws_bytes;
        TcPlan t = make_tc_plan(op, n_x, n_y, len_x - 1, len_y - 1, dim, order, tsize_of(precision));
        if (t.ok) return t.ws_bytes;
        precision = cell_prec(precision); // as the entry points: CUDA-core increments, same cells
    }
    if (precision == SIGK_PREC_FP64 && dim > 0) {
        const int kop = op == SIGK_OP_PAIRWISE ? kOpPairwise : op == SIGK_OP_GRAM ? kOpGram : kOpGramSym;
        TcPlan t = make_mat64_plan(kop, n_x, n_y, len_x - 1, len_y - 1, dim, order);
        if (t.ok) return t.ws_bytes;
    }
    // dim == 0 selects the plan of the *_inc entry points (no dx staging)
    Plan pl = make_plan(op, n_x, n_y, len_x - 1, len_y - 1, dim > 0 ? dim : 1, order, tsize_of(precision), dim == 0);
    return pl.ws_bytes;
}

int sigk_pairwise(const void *x, const void *y, int64_t batch, int64_t len_x, int64_t len_y, int64_t dim, int dtype,
                  int order, double static_scale, const void *scale_x, const void *scale_y, void *out, int precision,
                  void *workspace, size_t workspace_bytes, sigk_stream_t stream)
{
    return run_pairs(kOpPairwise, x, y, batch, batch, len_x, len_y, dim, dtype, order, static_scale, scale_x, scale_y,
                     out, 1, precision, workspace, workspace_bytes, (cudaStream_t)stream);
}

int sigk_gram(const void *x, const void *y, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y, int64_t dim,
              int dtype, int order, double static_scale, const void *scale_x, const void *scale_y, void *out,
              int precision, void *workspace, size_t workspace_bytes, sigk_stream_t stream)
{
    return run_pairs(kOpGram, x, y, n_x, n_y, len_x, len_y, dim, dtype, order, static_scale, scale_x, scale_y, out,
                     n_y, precision, workspace, workspace_bytes, (cudaStream_t)stream);
}

int sigk_gram_sym(const void *x, int64_t n, int64_t len, int64_t dim, int dtype, int order, double static_scale,
                  const void *scale, void *out, int precision, void *workspace, size_t workspace_bytes,
                  sigk_stream_t stream)
{
    return run_pairs(kOpGramSym, x, x, n, n, len, len, dim, dtype, order, static_scale, scale, scale, out, n,
                     precision, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t sigk_static_workspace_size(int op, int kind, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y,
                                  int64_t dim, int order, int dtype, int precision)
{
    if (kind == SIGK_STATIC_LINEAR) return sigk_workspace_size(op, n_x, n_y, len_x, len_y, dim, order, dtype, precision);
    if (kind != SIGK_STATIC_RBF && kind != SIGK_STATIC_L1RBF) return 0;
    if (op != SIGK_OP_GRAM && op != SIGK_OP_GRAM_SYM) return 0;
    if (len_x < 2 || len_y < 2 || order < 0 || order > 12 || dim < 1 || n_x < 1 || n_y < 1) return 0;
    if (op == SIGK_OP_GRAM_SYM) {
        n_y = n_x;
        len_y = len_x;
    }
    TcPlan t = make_static_plan(op == SIGK_OP_GRAM ? kOpGram : kOpGramSym, n_x, n_y, len_x - 1, len_y - 1, dim, order,
                                precision);
    return t.ok ? t.ws_bytes : 0;
}

int sigk_gram_static(int op, int kind, double param, const void *x, const void *y, int64_t n_x, int64_t n_y,
                     int64_t len_x, int64_t len_y, int64_t dim, int dtype, int order, const void *scale_x,
                     const void *scale_y, void *out, int precision, void *workspace, size_t workspace_bytes,
                     sigk_stream_t stream)
{
    if (op != SIGK_OP_GRAM && op != SIGK_OP_GRAM_SYM)
        return fail(SIGK_EINVAL, "op must be SIGK_OP_GRAM or SIGK_OP_GRAM_SYM (got %d)", op);
    const bool sym = op == SIGK_OP_GRAM_SYM;
    if (sym) {
        if (y && y != x) return fail(SIGK_EINVAL, "SIGK_OP_GRAM_SYM takes y = NULL (or y = x)");
        y = x;
        n_y = n_x;
        len_y = len_x;
        scale_y = scale_x;
    }
    const int kop = sym ? kOpGramSym : kOpGram;
    if (kind == SIGK_STATIC_LINEAR)
        return run_pairs(kop, x, y, n_x, n_y, len_x, len_y, dim, dtype, order, param, scale_x, scale_y, out, n_y,
                         precision, workspace, workspace_bytes, (cudaStream_t)stream);
    if (kind != SIGK_STATIC_RBF && kind != SIGK_STATIC_L1RBF)
        return fail(SIGK_EINVAL, "unknown static kernel kind %d", kind);
    int st = check_common(dtype, precision, order);
    if (st) return st;
    if (!(param > 0.0) || !std::isfinite(param)) return fail(SIGK_EINVAL, "sigma must be finite and > 0");
    if (n_x < 1 || n_y < 1) return fail(SIGK_EINVAL, "path counts must be >= 1 (got %lld, %lld)", (long long)n_x,
                                        (long long)n_y);
    if (len_x < 2 || len_y < 2) return fail(SIGK_EINVAL, "path lengths must be >= 2 (got %lld, %lld)",
                                            (long long)len_x, (long long)len_y);
    if (dim < 1) return fail(SIGK_EINVAL, "dim must be >= 1");
    if (dim > kStaticMaxDim)
        return fail(SIGK_EUNSUPPORTED, "RBF / L1-RBF increments from points take dim <= %lld (got %lld); use "
                                       "sigk_gram_inc", (long long)kStaticMaxDim, (long long)dim);
    if ((st = check_dev(x, "x", false)) || (st = check_dev(y, "y", false)) || (st = check_dev(out, "out", false)) ||
        (st = check_dev(scale_x, "scale_x", true)) || (st = check_dev(scale_y, "scale_y", true)))
        return st;
    TcPlan t = make_static_plan(kop, n_x, n_y, len_x - 1, len_y - 1, dim, order, precision);
    if (!t.ok) return fail(SIGK_EUNSUPPORTED, "no static-kernel plan");
    if (!workspace || workspace_bytes < t.ws_bytes)
        return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", t.ws_bytes,
                    workspace ? workspace_bytes : 0);
    if (((uintptr_t)workspace & 255) != 0) return fail(SIGK_EINVAL, "workspace must be 256-byte aligned");
    return run_pairs_static(t, kop, kind, param, x, y, n_x, n_y, len_x, len_y, dim, dtype, order, scale_x, scale_y,
                            out, n_y, precision, workspace, (cudaStream_t)stream);
}

size_t sigk_backward_workspace_size(int op, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y, int64_t dim,
                                    int order, int dtype)
{
    (void)dtype;
    if (op != SIGK_OP_PAIRWISE && op != SIGK_OP_GRAM) return 0;
    if (len_x < 2 || len_y < 2 || order < 0 || order > 12 || dim < 1 || n_x < 1 || n_y < 1) return 0;
    if (op == SIGK_OP_PAIRWISE) n_y = n_x;
    GradPlan g = make_grad_plan(op == SIGK_OP_PAIRWISE ? kOpPairwise : kOpGram, n_x, n_y, len_x - 1, len_y - 1, dim,
                                order);
    return g.ok ? g.ws_bytes : 0;
}

int sigk_backward(int op, const void *x, const void *y, int64_t n_x, int64_t n_y, int64_t len_x, int64_t len_y,
                  int64_t dim, int dtype, int order, double static_scale, const void *scale_x, const void *scale_y,
                  const void *grad_out, void *grad_x, void *grad_y, void *workspace, size_t workspace_bytes,
                  sigk_stream_t stream)
{
    if (op != SIGK_OP_PAIRWISE && op != SIGK_OP_GRAM)
        return fail(SIGK_EINVAL, "op must be SIGK_OP_PAIRWISE or SIGK_OP_GRAM (got %d)", op);
    int st = check_common(dtype, SIGK_PREC_FP64, order);
    if (st) return st;
    if (op == SIGK_OP_PAIRWISE) n_y = n_x;
    if (n_x < 1 || n_y < 1) return fail(SIGK_EINVAL, "path counts must be >= 1 (got %lld, %lld)", (long long)n_x,
                                        (long long)n_y);
    if (len_x < 2 || len_y < 2) return fail(SIGK_EINVAL, "path lengths must be >= 2 (got %lld, %lld)",
                                            (long long)len_x, (long long)len_y);
    if (dim < 1) return fail(SIGK_EINVAL, "dim must be >= 1");
    if (order > kGradMaxOrder)
        return fail(SIGK_EUNSUPPORTED, "the backward pass takes dyadic order <= %d (got %d)", kGradMaxOrder, order);
    if (!grad_x && !grad_y) return SIGK_OK;
    if ((st = check_dev(x, "x", false)) || (st = check_dev(y, "y", false)) ||
        (st = check_dev(grad_out, "grad_out", false)) || (st = check_dev(grad_x, "grad_x", true)) ||
        (st = check_dev(grad_y, "grad_y", true)) || (st = check_dev(scale_x, "scale_x", true)) ||
        (st = check_dev(scale_y, "scale_y", true)))
        return st;
    const int kop = op == SIGK_OP_PAIRWISE ? kOpPairwise : kOpGram;
    GradPlan g = make_grad_plan(kop, n_x, n_y, len_x - 1, len_y - 1, dim, order);
    if (!g.ok) return fail(SIGK_EUNSUPPORTED, "no backward plan");
    if (!workspace || workspace_bytes < g.ws_bytes)
        return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", g.ws_bytes,
                    workspace ? workspace_bytes : 0);
    if (((uintptr_t)workspace & 255) != 0) return fail(SIGK_EINVAL, "workspace must be 256-byte aligned");
    return run_backward(g, kop, x, y, n_x, n_y, len_x, len_y, dim, dtype, order, static_scale, scale_x, scale_y,
                        grad_out, grad_x, grad_y, workspace, (cudaStream_t)stream);
}

size_t sigk_backward_inc_workspace_size(int64_t npairs, int64_t nc_x, int64_t nc_y, int order)
{
    if (npairs < 1 || nc_x < 1 || nc_y < 1 || order < 0 || order > kGradMaxOrder) return 0;
    GradPlan g = make_grad_inc_plan(npairs, nc_x, nc_y, order);
    return g.ok ? g.ws_bytes : 0;
}

int sigk_backward_inc(const void *inc, int64_t npairs, int64_t nc_x, int64_t nc_y, int64_t s0, int64_t s1, int64_t s2,
                      int dtype, int order, const void *scale_x, const void *scale_y, const void *grad_out,
                      void *grad_inc, int64_t g0, int64_t g1, int64_t g2, void *workspace, size_t workspace_bytes,
                      sigk_stream_t stream)
{
    int st = check_common(dtype, SIGK_PREC_FP64, order);
    if (st) return st;
    if (npairs < 1 || nc_x < 1 || nc_y < 1)
        return fail(SIGK_EINVAL, "need npairs, nc_x, nc_y >= 1 (got %lld, %lld, %lld)", (long long)npairs,
                    (long long)nc_x, (long long)nc_y);
    if (order > kGradMaxOrder)
        return fail(SIGK_EUNSUPPORTED, "the backward pass takes dyadic order <= %d (got %d)", kGradMaxOrder, order);
    if ((st = check_dev(inc, "inc", false)) || (st = check_dev(grad_out, "grad_out", false)) ||
        (st = check_dev(grad_inc, "grad_inc", false)) || (st = check_dev(scale_x, "scale_x", true)) ||
        (st = check_dev(scale_y, "scale_y", true)))
        return st;
    GradPlan g = make_grad_inc_plan(npairs, nc_x, nc_y, order);
    if (!g.ok) return fail(SIGK_EUNSUPPORTED, "no backward plan");
    if (!workspace || workspace_bytes < g.ws_bytes)
        return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", g.ws_bytes,
                    workspace ? workspace_bytes : 0);
    if (((uintptr_t)workspace & 255) != 0) return fail(SIGK_EINVAL, "workspace must be 256-byte aligned");
    return run_backward_inc(g, inc, npairs, nc_x, nc_y, s0, s1, s2, dtype, order, scale_x, scale_y, grad_out,
                            grad_inc, g0, g1, g2, workspace, (cudaStream_t)stream);
}

// Shared body of sigk_normalize, sigk_normalize_inc and sigk_self_norms
// (maxit = 0, no lambda output).
static int normalize_impl(const void *x, const void *inc, int64_t n, int64_t nc, int64_t d, int64_t s0, int64_t s1,
                          int64_t s2, int dtype, int order, double static_scale, double *knorm, const double *fnorm,
                          double tol, int maxit, void *lam, bool need_lam, int *iters, void *ws, size_t ws_bytes,
                          cudaStream_t stream)
{
    int st = check_common(dtype, SIGK_PREC_FP64, order);
    if (st) return st;
    if (n < 1) return fail(SIGK_EINVAL, "path count must be >= 1");
    if (nc < 1) return fail(SIGK_EINVAL, "path length must be >= 2");
    if (maxit < 0) return fail(SIGK_EINVAL, "maxit must be >= 0");
    if (!(tol >= 0)) return fail(SIGK_EINVAL, "tol must be >= 0");
    const bool from_inc = inc != nullptr;
    if (from_inc) {
        if ((st = check_dev(inc, "inc", false))) return st;
        if (!knorm || !fnorm) return fail(SIGK_EINVAL, "increment mode needs knorm and fnorm");
    } else {
        if (d < 1) return fail(SIGK_EINVAL, "dim must be >= 1");
        if ((st = check_dev(x, "x", false))) return st;
    }
    if ((st = check_dev(lam, "lam", !need_lam)) || (st = check_dev(knorm, "knorm", true)) ||
        (st = check_dev(fnorm, "fnorm", true)) || (st = check_dev(iters, "iters", true)))
        return st;
    if (fnorm && !knorm) return fail(SIGK_EINVAL, "fnorm given without knorm");
    NormPlan q = norm_plan(n, nc, d, order, from_inc);
    if (q.ws_bytes) {
        if (!ws || ws_bytes < q.ws_bytes)
            return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", q.ws_bytes, ws ? ws_bytes : 0);
        if (((uintptr_t)ws & 255) != 0) return fail(SIGK_EINVAL, "workspace must be 256-byte aligned");
    }
    unsigned char *wsb = reinterpret_cast<unsigned char *>(ws);
    double *dx = nullptr;
    if (!from_inc) { // unscaled float64 differences, dimension-major (the kernel applies the scale)
        dx = reinterpret_cast<double *>(wsb + q.dx_off);
        DeltaFn delta = get_delta_kernel(true, dtype == SIGK_F64);
        const int64_t total = n * nc * d;
        int64_t blocks = (total + 255) / 256;
        if (blocks > (int64_t)sm_count() * 8) blocks = (int64_t)sm_count() * 8;
        delta<<<(unsigned)blocks, 256, 0, stream>>>(x, n, nc + 1, d, d, 1.0, nullptr, dx);
        count_launch();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "delta kernel launch");
    }
    NormParams p{};
    p.x = x;
    p.dx = dx;
    p.tile_pitch = q.tile_pitch;
    p.n = n;
    p.nc = nc;
    p.d = d;
    p.order = order;
    p.fscale = from_inc ? 1.0 : static_scale * std::ldexp(1.0, -2 * order);
    p.inc = inc;
    p.is0 = s0;
    p.is1 = s1;
    p.is2 = s2;
    p.knorm = knorm;
    p.fnorm = fnorm;
    p.tol = tol;
    p.maxit = maxit;
    p.lam = lam;
    p.iters = iters;
    if (q.pipe) {
        cudaError_t e = cudaMemsetAsync(wsb, 0, q.bnd_bytes, stream);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(progress)");
        p.prog = reinterpret_cast<int *>(wsb + q.prog_off);
        p.err = reinterpret_cast<int *>(wsb + q.err_off);
        p.bnd = wsb + q.bnd_bytes;
        p.bnd_stride = q.bnd_stride;
        p.stage_smem = q.mode == kNormDelta && q.smem_cta > 0;
        NormFn fn = get_norm_pipe_kernel(dtype == SIGK_F64, q.mode, q.R, q.O);
        if (q.smem_cta > 48 * 1024) {
            int dev = 0, optin = 0;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
            if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
                return cuda_fail(e, "cudaDeviceGetAttribute");
            cudaFuncAttributes fa{};
            if ((e = cudaFuncGetAttributes(&fa, (const void *)fn)) != cudaSuccess)
                return cuda_fail(e, "cudaFuncGetAttributes");
            const int dyn_max = optin - (int)fa.sharedSizeBytes; // the kernel's static shared memory counts too
            if ((size_t)dyn_max < q.smem_cta)
                return fail(SIGK_ELAUNCH, "normalisation needs %zu bytes of shared memory", q.smem_cta);
            if ((e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max)) !=
                cudaSuccess)
                return cuda_fail(e, "cudaFuncSetAttribute");
        }
        const int64_t grid = n < 0x7fffffffLL ? n : 0x7fffffffLL; // one CTA per path (more paths: strided)
        fn<<<(unsigned)grid, q.nw * 32, q.smem_cta, stream>>>(p);
        count_launch();
        e = cudaGetLastError();
        return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "pipelined normalisation launch");
    }
    p.bnd = q.nbands > 1 ? ws : nullptr;
    p.bnd_stride = q.bnd_stride;
    p.stage_smem = q.smem_per_warp > 0;
    NormFn fn = get_norm_kernel(dtype == SIGK_F64, q.mode, q.R, q.O);
    return launch(fn, p, n, q.smem_per_warp * kWarpsPerBlock, stream);
}

static int run_normalize(const void *x, const void *inc, int64_t n, int64_t nc, int64_t d, int64_t s0, int64_t s1,
                         int64_t s2, int dtype, int order, double static_scale, double *knorm, const double *fnorm,
                         double tol, int maxit, void *lam, int *iters, void *ws, size_t ws_bytes,
                         cudaStream_t stream)
{
    return normalize_impl(x, inc, n, nc, d, s0, s1, s2, dtype, order, static_scale, knorm, fnorm, tol, maxit, lam,
                          true, iters, ws, ws_bytes, stream);
}

int sigk_self_norms(const void *x, int64_t n, int64_t len, int64_t dim, int dtype, int order, double static_scale,
                    double *knorm, void *workspace, size_t workspace_bytes, sigk_stream_t stream)
{
    // k(x,x) with float64 cells, written as float64; NaN -> +inf is applied by
    // the normalisation kernel, which with maxit = 0 runs no bracket iterations.
    int st = check_dev(knorm, "knorm", false);
    if (st) return st;
    if (len < 2) return fail(SIGK_EINVAL, "path length must be >= 2");
    return normalize_impl(x, nullptr, n, len - 1, dim, 0, 0, 0, dtype, order, static_scale, knorm, nullptr, 0.0, 0,
                          nullptr, false, nullptr, workspace, workspace_bytes, (cudaStream_t)stream);
}

int sigk_normalize(const void *x, int64_t n, int64_t len, int64_t dim, int dtype, int order, double static_scale,
                   double *knorm, const double *fnorm, double tol, int maxit, void *lam, int *iters, void *workspace,
                   size_t workspace_bytes, sigk_stream_t stream)
{
    if (len < 2) return fail(SIGK_EINVAL, "path length must be >= 2");
    return run_normalize(x, nullptr, n, len - 1, dim, 0, 0, 0, dtype, order, static_scale, knorm, fnorm, tol, maxit,
                         lam, iters, workspace, workspace_bytes, (cudaStream_t)stream);
}

int sigk_normalize_inc(const void *inc, int64_t n, int64_t nc, int64_t s0, int64_t s1, int64_t s2, int dtype,
                       int order, const double *knorm, const double *fnorm, double tol, int maxit, void *lam,
                       int *iters, void *workspace, size_t workspace_bytes, sigk_stream_t stream)
{
    if (!inc) return fail(SIGK_EINVAL, "inc is NULL");
    return run_normalize(nullptr, inc, n, nc, 1, s0, s1, s2, dtype, order, 1.0, const_cast<double *>(knorm), fnorm,
                         tol, maxit, lam, iters, workspace, workspace_bytes, (cudaStream_t)stream);
}

static int run_inc(int op, const void *inc, int64_t nx, int64_t ny, int64_t ncx, int64_t ncy, int64_t s0, int64_t s1,
                   int64_t s2, int64_t s3, int dtype, int order, const void *sx, const void *sy, void *out,
                   int64_t out_ld, int precision, void *ws, size_t ws_bytes, cudaStream_t stream)
{
    int st = check_common(dtype, precision, order);
    if (st) return st;
    if (nx < 1 || ny < 1 || ncx < 1 || ncy < 1) return fail(SIGK_EINVAL, "empty increment tensor");
    if ((st = check_dev(inc, "inc", false)) || (st = check_dev(out, "out", false)) ||
        (st = check_dev(sx, "scale_x", true)) || (st = check_dev(sy, "scale_y", true)))
        return st;
    Plan pl = make_plan(op, nx, ny, ncx, ncy, 1, order, tsize_of(precision), true);
    if ((st = check_ws(pl, ws, ws_bytes))) return st;
    PairParams p{};
    p.op = op;
    p.nx = nx;
    p.ny = ny;
    p.ncx = ncx;
    p.ncy = ncy;
    p.d = 1;
    p.order = order;
    p.fscale = 1.0;
    p.sx = sx;
    p.sy = sy;
    p.inc = inc;
    p.is0 = s0;
    p.is1 = s1;
    p.is2 = s2;
    p.is3 = s3;
    p.out = out;
    p.out_ld = out_ld;
    p.nitems = op == kOpPairwise ? nx : (op == kOpGram ? nx * ny : nx * (nx + 1) / 2);
    p.bnd = pl.nbands > 1 ? ws : nullptr;
    p.bnd_stride = pl.bnd_stride;
    p.stage_smem = 0;
    PairFn fn = pick_pair(precision, dtype, kPairGiven, pl.R, pl.O);
    return launch(fn, p, p.nitems, 0, stream);
}

int sigk_pairwise_inc(const void *inc, int64_t batch, int64_t nc_x, int64_t nc_y, int64_t s0, int64_t s1, int64_t s2,
                      int dtype, int order, const void *scale_x, const void *scale_y, void *out, int precision,
                      void *workspace, size_t workspace_bytes, sigk_stream_t stream)
{
    return run_inc(kOpPairwise, inc, batch, batch, nc_x, nc_y, s0, s1, s2, 0, dtype, order, scale_x, scale_y, out, 1,
                   precision, workspace, workspace_bytes, (cudaStream_t)stream);
}

int sigk_gram_inc(const void *inc, int64_t n_x, int64_t n_y, int64_t nc_x, int64_t nc_y, int64_t s0, int64_t s1,
                  int64_t s2, int64_t s3, int dtype, int order, const void *scale_x, const void *scale_y, int symmetric,
                  void *out, int64_t out_ld, int precision, void *workspace, size_t workspace_bytes,
                  sigk_stream_t stream)
{
    if (symmetric && n_x != n_y) return fail(SIGK_EINVAL, "symmetric Gram needs n_x == n_y");
    return run_inc(symmetric ? kOpGramSym : kOpGram, inc, n_x, n_y, nc_x, nc_y, s0, s1, s2, s3, dtype, order,
                   scale_x, scale_y, out, out_ld, precision, workspace, workspace_bytes, (cudaStream_t)stream);
}

} // extern "C"

// ---------------------------------------------------------------------------
// No-allocation variant of sigk_gram.
//
// Some callers cannot call cudaMalloc: a host program that links only this
// library and works inside a device-memory budget fixed up front, or a caller
// inside a framework whose allocator it may not touch.  For them the scratch
// that sigk_gram takes from the caller (the scaled path differences the
// streaming kernel reads) lives in the fixed array below instead.  The array
// is part of the library's device image, so every GPU that loads the library
// holds these 8 MiB until the process exits.
namespace sigk {
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
} // namespace
} // namespace sigk

static __device__ __align__(256) unsigned char g_sigk_noalloc_scratch[sigk::kNoAllocScratchBytes];

namespace sigk {
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kMaxDevices] = {};

// The device address of the scratch array on the current device.  In host
// code the array's name is only a host-side stand-in, so the address is taken
// once per device, with that device current, and cached.
int noalloc_scratch(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(SIGK_EUNSUPPORTED, "device index %d >= %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_sigk_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
        g_noalloc_ptr[dev] = ptr;
    }
    *out = g_noalloc_ptr[dev];
    return SIGK_OK;
}
} // namespace
} // namespace sigk

extern "C" int sigk_gram_noalloc(const void *x, const void *y, int64_t n_x, int64_t n_y, int64_t len_x,
                                 int64_t len_y, int64_t dim, int dtype, int order, double static_scale,
                                 const void *scale_x, const void *scale_y, void *out, int precision,
                                 sigk_stream_t stream)
{
    const size_t need =
        sigk_workspace_size(SIGK_OP_GRAM, n_x, n_y, len_x, len_y, dim, order, dtype, precision);
    if (need > kNoAllocScratchBytes)
        return fail(SIGK_EINVAL,
                    "sigk_gram_noalloc: this Gram needs %zu bytes of scratch; the no-allocation entry point has "
                    "%zu bytes (8 MiB); use sigk_gram with a caller workspace",
                    need, kNoAllocScratchBytes);
    void *scratch = nullptr;
    int st = noalloc_scratch(&scratch);
    if (st != SIGK_OK) return st;
    return run_pairs(kOpGram, x, y, n_x, n_y, len_x, len_y, dim, dtype, order, static_scale, scale_x, scale_y, out,
                     n_y, precision, scratch, kNoAllocScratchBytes, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Uneven batched pairwise (paths of different lengths, a dyadic order per pair)
namespace sigk {
namespace {
constexpr size_t kRaggedStageBytesPerWarp = 16 * 1024;

struct RaggedPlan {
    size_t counter_off, error_off, progress_off, pool_off, dx_off, dy_off, ws_bytes;
};

RaggedPlan ragged_plan(int64_t npairs, int64_t x_points, int64_t y_points, int64_t dim, int64_t nitems,
                       int64_t bnd_elems, size_t tsize)
{
    RaggedPlan r{};
    r.counter_off = 0;
    r.error_off = 8;
    r.progress_off = 256;
    r.pool_off = align256(r.progress_off + (size_t)nitems * sizeof(int));
    r.dx_off = align256(r.pool_off + (size_t)bnd_elems * tsize);
    r.dy_off = align256(r.dx_off + (size_t)(x_points - npairs) * (size_t)dim * tsize);
    r.ws_bytes = align256(r.dy_off + (size_t)(y_points - npairs) * (size_t)dim * tsize);
    return r;
}
} // namespace
} // namespace sigk

extern "C" size_t sigk_ragged_workspace_size(int64_t npairs, int64_t x_points, int64_t y_points, int64_t dim,
                                             int64_t nitems, int64_t bnd_elems, int precision)
{
    if (npairs < 1 || dim < 1 || nitems < npairs || bnd_elems < 0 || x_points < npairs || y_points < npairs) return 0;
    return ragged_plan(npairs, x_points, y_points, dim, nitems, bnd_elems, tsize_of(precision)).ws_bytes;
}

namespace sigk {
namespace {
// Tensor-core layout of an uneven batch in the workspace, after the ragged
// plan's counters and boundary pool: GEMM error word, A and B operand images
// (hi, lo), the increment matrix.
struct RaggedTcLayout {
    int kp;
    size_t err_off, a_off, a_bytes, b_off, b_bytes, inc_off, ws_bytes;
};

// With fp64 cells the same plan holds float64 row images [row][dim] and a
// float64 increment matrix (no hi / lo split).
RaggedTcLayout ragged_mat64_layout(size_t base, int64_t dim, const sigk_ragged_tc_plan &pl)
{
    RaggedTcLayout t{};
    t.kp = (int)dim;
    t.err_off = align256(base);
    t.a_off = t.err_off + 256;
    t.a_bytes = align256((size_t)pl.a_rows * dim * sizeof(double));
    t.b_off = t.a_off + t.a_bytes;
    t.b_bytes = align256((size_t)pl.b_rows * dim * sizeof(double));
    t.inc_off = t.b_off + t.b_bytes;
    t.ws_bytes = t.inc_off + align256((size_t)pl.inc_elems * sizeof(double));
    return t;
}

RaggedTcLayout ragged_tc_layout(size_t base, int64_t dim, const sigk_ragged_tc_plan &pl)
{
    RaggedTcLayout t{};
    t.kp = (int)((dim + 7) / 8 * 8);
    t.err_off = align256(base);
    t.a_off = t.err_off + 256;
    t.a_bytes = align256((size_t)pl.a_rows * t.kp * sizeof(float));
    t.b_off = t.a_off + 2 * t.a_bytes;
    t.b_bytes = align256((size_t)pl.b_rows * t.kp * sizeof(float));
    t.inc_off = t.b_off + 2 * t.b_bytes;
    t.ws_bytes = t.inc_off + align256((size_t)pl.inc_elems * sizeof(float));
    return t;
}

int run_ragged(const void *x_pack, const int64_t *x_off, const int64_t *x_len, int64_t x_points, const void *y_pack,
               const int64_t *y_off, const int64_t *y_len, int64_t y_points, const int *order,
               const int64_t *item_pair, const int *item_band, int64_t nitems, const int *pair_rows,
               const int *pair_bands, const int64_t *pair_bnd_off, int64_t bnd_elems, int64_t npairs, int64_t dim,
               int dtype, double static_scale, const void *scale_x, const void *scale_y, void *out, int precision,
               const sigk_ragged_tc_plan *tc, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    int st = check_common(dtype, precision, 0);
    if (st) return st;
    if (npairs < 1) return fail(SIGK_EINVAL, "npairs must be >= 1");
    if (dim < 1) return fail(SIGK_EINVAL, "dim must be >= 1");
    if (nitems < npairs) return fail(SIGK_EINVAL, "nitems must be >= npairs (one item per band)");
    if (nitems > 0x7fffffffLL) return fail(SIGK_EINVAL, "too many band items");
    if (bnd_elems < 0) return fail(SIGK_EINVAL, "bnd_elems must be >= 0");
    if (x_points < 2 * npairs || y_points < 2 * npairs)
        return fail(SIGK_EINVAL, "x_points / y_points must count every packed point (>= 2 per path)");
    if ((st = check_dev(x_pack, "x_pack", false)) || (st = check_dev(x_off, "x_off", false)) ||
        (st = check_dev(x_len, "x_len", false)) || (st = check_dev(y_pack, "y_pack", false)) ||
        (st = check_dev(y_off, "y_off", false)) || (st = check_dev(y_len, "y_len", false)) ||
        (st = check_dev(order, "order", false)) || (st = check_dev(item_pair, "item_pair", false)) ||
        (st = check_dev(item_band, "item_band", false)) || (st = check_dev(pair_rows, "pair_rows", false)) ||
        (st = check_dev(pair_bands, "pair_bands", false)) || (st = check_dev(pair_bnd_off, "pair_bnd_off", false)) ||
        (st = check_dev(out, "out", false)) || (st = check_dev(scale_x, "scale_x", true)) ||
        (st = check_dev(scale_y, "scale_y", true)))
        return st;
    const bool mat64 = tc && precision == SIGK_PREC_FP64; // float64 increments on the CUDA cores from the plan
    if (tc) {
        if (!is_tc(precision) && !mat64)
            return fail(SIGK_EINVAL, "a plan needs precision SIGK_PREC_TC32, _TC64 or _FP64");
        if (!mat64 && dim > 32)
            return fail(SIGK_EUNSUPPORTED, "tensor-core increments support dim <= 32 (got %lld)", (long long)dim);
        if (tc->tile_n != 0 && tc->tile_n != 128 && tc->tile_n != kTcBN)
            return fail(SIGK_EINVAL, "plan.tile_n must be 0, 128 or 256 (got %lld)", (long long)tc->tile_n);
        if (mat64 && tc->tile_n == 128)
            return fail(SIGK_EINVAL, "128-column tiles apply to tensor-core precisions only");
        if (tc->a_rows < kTcM || tc->b_rows < (tc->tile_n ? tc->tile_n : kTcBN) || tc->inc_elems < 4 ||
            tc->ntiles < 1 || (tc->a_rows & 7) || (tc->b_rows & 7))
            return fail(SIGK_EINVAL, "tensor-core plan sizes are inconsistent");
        if ((st = check_dev(tc->a_row0, "plan.a_row0", false)) || (st = check_dev(tc->b_row0, "plan.b_row0", false)) ||
            (st = check_dev(tc->inc_off, "plan.inc_off", false)) || (st = check_dev(tc->tiles, "plan.tiles", false)))
            return st;
    }
    const size_t ts = tsize_of(precision);
    const bool f64 = cell_prec(precision) == SIGK_PREC_FP64, in64 = dtype == SIGK_F64;
    RaggedPlan pl = ragged_plan(npairs, tc ? 2 * npairs : x_points, tc ? 2 * npairs : y_points, dim, nitems,
                                bnd_elems, ts);
    RaggedTcLayout tl{};
    size_t need = pl.ws_bytes;
    if (tc) {
        tl = mat64 ? ragged_mat64_layout(pl.dx_off, dim, *tc) : ragged_tc_layout(pl.dx_off, dim, *tc);
        need = tl.ws_bytes;
    }
    if (!workspace || workspace_bytes < need)
        return fail(SIGK_ENOMEM, "workspace of %zu bytes needed (got %zu)", need, workspace ? workspace_bytes : 0);
    if (((uintptr_t)workspace & 255) != 0) return fail(SIGK_EINVAL, "workspace must be 256-byte aligned");
    unsigned char *wsb = reinterpret_cast<unsigned char *>(workspace);
    // work counter, error flag and per-item progress start at zero (and the GEMM's error word)
    cudaError_t e = cudaMemsetAsync(wsb, 0, pl.pool_off, stream);
    if (e == cudaSuccess && tc) e = cudaMemsetAsync(wsb + tl.err_off, 0, 256, stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(counters)");
    const int nsm = sm_count();

    RaggedParams p{};
    if (!tc) {
        // scaled, dimension-major differences of both packs: static_scale * 4^-order * scale_x on x, scale_y on y.
        // grid: y over paths (strided beyond 65535), x over one path's (len - 1) * dim values
        RaggedDeltaFn delta = get_ragged_delta_kernel(f64, in64);
        const dim3 dgrid(32, (unsigned)(npairs < 65535 ? npairs : 65535));
        delta<<<dgrid, 256, 0, stream>>>(x_pack, x_off, x_len, order, static_scale, scale_x, npairs, dim,
                                         wsb + pl.dx_off);
        count_launch();
        delta<<<dgrid, 256, 0, stream>>>(y_pack, y_off, y_len, nullptr, 1.0, scale_y, npairs, dim, wsb + pl.dy_off);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "ragged delta launch");
        p.dx_pack = wsb + pl.dx_off;
        p.dy_pack = wsb + pl.dy_off;
    } else if (mat64) {
        double *a_img = reinterpret_cast<double *>(wsb + tl.a_off), *b_img = reinterpret_cast<double *>(wsb + tl.b_off);
        double *inc = reinterpret_cast<double *>(wsb + tl.inc_off);
        unsigned *gerr = reinterpret_cast<unsigned *>(wsb + tl.err_off);
        RaggedImage64Fn image = get_ragged_image64_kernel(in64);
        const dim3 igrid(8, (unsigned)(npairs < 65535 ? npairs : 65535));
        for (int side = 0; side < 2; ++side) {
            TcRaggedImageParams ip{};
            ip.x_pack = x_pack;
            ip.y_pack = y_pack;
            ip.x_off = x_off;
            ip.x_len = x_len;
            ip.y_off = y_off;
            ip.y_len = y_len;
            ip.order = order;
            ip.f = static_scale;
            ip.sx = scale_x;
            ip.sy = scale_y;
            ip.row0 = side == 0 ? tc->a_row0 : tc->b_row0;
            ip.rows_alloc = side == 0 ? tc->a_rows : tc->b_rows;
            ip.npairs = npairs;
            ip.d = dim;
            ip.side = side;
            image<<<igrid, 256, 0, stream>>>(ip, side == 0 ? a_img : b_img);
            count_launch();
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "ragged float64 image launch");
        RaggedDgemmParams gp{};
        gp.a = a_img;
        gp.b = b_img;
        gp.a_rows = tc->a_rows;
        gp.b_rows = tc->b_rows;
        gp.d = dim;
        gp.tiles = tc->tiles;
        gp.ntiles = tc->ntiles;
        gp.out = inc;
        gp.out_elems = tc->inc_elems;
        gp.err = gerr;
        RaggedDgemmFn rpipe = env_flag("SIGK_NO_DGEMM_PIPE") ? nullptr : get_ragged_dgemm_pipe_kernel(dim);
        int64_t blocks = tc->ntiles * (rpipe ? 2 : 8); // half-tiles / pieces
        if (blocks > (int64_t)nsm * 24) blocks = (int64_t)nsm * 24;
        (rpipe ? rpipe : get_ragged_dgemm_kernel())<<<(unsigned)blocks, 256, 0, stream>>>(gp);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "ragged float64 increment GEMM launch");
        p.inc = inc;
        p.inc_off = tc->inc_off;
        p.inc_elems = tc->inc_elems;
        p.tc_err = gerr;
    } else {
        float *a_hi = reinterpret_cast<float *>(wsb + tl.a_off), *a_lo = reinterpret_cast<float *>(wsb + tl.a_off + tl.a_bytes);
        float *b_hi = reinterpret_cast<float *>(wsb + tl.b_off), *b_lo = reinterpret_cast<float *>(wsb + tl.b_off + tl.b_bytes);
        float *inc = reinterpret_cast<float *>(wsb + tl.inc_off);
        unsigned *gerr = reinterpret_cast<unsigned *>(wsb + tl.err_off);
        TcRaggedImageFn image = get_tc_ragged_image_kernel(in64);
        const dim3 igrid(8, (unsigned)(npairs < 65535 ? npairs : 65535));
        for (int side = 0; side < 2; ++side) {
            TcRaggedImageParams ip{};
            ip.x_pack = x_pack;
            ip.y_pack = y_pack;
            ip.x_off = x_off;
            ip.x_len = x_len;
            ip.y_off = y_off;
            ip.y_len = y_len;
            ip.order = order;
            ip.f = static_scale;
            ip.sx = scale_x;
            ip.sy = scale_y;
            ip.row0 = side == 0 ? tc->a_row0 : tc->b_row0;
            ip.rows_alloc = side == 0 ? tc->a_rows : tc->b_rows;
            ip.npairs = npairs;
            ip.d = dim;
            ip.kp = tl.kp;
            ip.side = side;
            ip.hi = side == 0 ? a_hi : b_hi;
            ip.lo = side == 0 ? a_lo : b_lo;
            image<<<igrid, 256, 0, stream>>>(ip);
            count_launch();
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "ragged operand image launch");
        TcGemmParams gp{};
        gp.a_hi = a_hi;
        gp.a_lo = a_lo;
        gp.b_hi = b_hi;
        gp.b_lo = b_lo;
        gp.mtiles = tc->ntiles;
        gp.ntiles = 1;
        gp.kp = tl.kp;
        gp.mode = kTcTable;
        gp.out = inc;
        gp.err = gerr;
        gp.table = tc->tiles;
        gp.ntable = tc->ntiles;
        gp.a_rows = tc->a_rows;
        gp.b_rows = tc->b_rows;
        gp.out_elems = tc->inc_elems;
        if ((st = tc_gemm(gp, stream, tc->tile_n == 128 ? 128 : kTcBN))) return st;
        p.inc = inc;
        p.inc_off = tc->inc_off;
        p.inc_elems = tc->inc_elems;
        p.tc_err = gerr;
    }
    p.x_off = x_off;
    p.x_len = x_len;
    p.y_off = y_off;
    p.y_len = y_len;
    p.order = order;
    p.item_pair = item_pair;
    p.item_band = item_band;
    p.nitems = nitems;
    p.pair_rows = pair_rows;
    p.pair_bands = pair_bands;
    p.pair_bnd_off = pair_bnd_off;
    p.bnd_elems = bnd_elems;
    p.npairs = npairs;
    p.d = dim;
    p.out = out;
    p.counter = reinterpret_cast<unsigned long long *>(wsb + pl.counter_off);
    p.error = reinterpret_cast<int *>(wsb + pl.error_off);
    p.progress = reinterpret_cast<int *>(wsb + pl.progress_off);
    p.pool = wsb + pl.pool_off;
    p.stage_elems_per_warp = tc ? 0 : (int)(kRaggedStageBytesPerWarp / ts);
    p.poll_limit = wait_limit();
    RaggedFn fn = get_ragged_kernel(f64, in64, tc != nullptr, mat64);
    const size_t smem = tc ? 0 : kRaggedStageBytesPerWarp * kWarpsPerBlock;
    int nb = 0;
    if ((st = blocks_per_sm((const void *)fn, smem, &nb))) return st;
    // persistent grid: never more blocks than can be resident at once (band waits rely on it)
    int64_t blocks = (int64_t)nsm * nb;
    const int64_t want = (nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > want) blocks = want;
    fn<<<(unsigned)blocks, kWarpsPerBlock * 32, smem, stream>>>(p);
    count_launch();
    e = cudaGetLastError();
    return e == cudaSuccess ? SIGK_OK : cuda_fail(e, "ragged kernel launch");
}
} // namespace
} // namespace sigk

extern "C" int sigk_pairwise_ragged(const void *x_pack, const int64_t *x_off, const int64_t *x_len, int64_t x_points,
                                    const void *y_pack, const int64_t *y_off, const int64_t *y_len, int64_t y_points,
                                    const int *order, const int64_t *item_pair, const int *item_band, int64_t nitems,
                                    const int *pair_rows, const int *pair_bands, const int64_t *pair_bnd_off,
                                    int64_t bnd_elems, int64_t npairs, int64_t dim, int dtype, double static_scale,
                                    const void *scale_x, const void *scale_y, void *out, int precision,
                                    void *workspace, size_t workspace_bytes, sigk_stream_t stream)
{
    if (is_tc(precision)) precision = cell_prec(precision); // no plan: CUDA-core increments, same cells
    return run_ragged(x_pack, x_off, x_len, x_points, y_pack, y_off, y_len, y_points, order, item_pair, item_band,
                      nitems, pair_rows, pair_bands, pair_bnd_off, bnd_elems, npairs, dim, dtype, static_scale,
                      scale_x, scale_y, out, precision, nullptr, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int sigk_ragged_status(const void *workspace, sigk_stream_t stream)
{
    if (!workspace) return fail(SIGK_EINVAL, "workspace is NULL");
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    int word = 0;
    e = cudaMemcpy(&word, reinterpret_cast<const unsigned char *>(workspace) + 8, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy of the error word");
    if (word & kErrWaitTimeout)
        return fail(SIGK_ETIMEDOUT, "a band wait of the last uneven-batch launch ran out (or its increment GEMM gave "
                                    "up a wait); the affected pairs are NaN");
    if (word & kErrInvalidItem)
        return fail(SIGK_EINVAL, "an item of the last uneven-batch launch broke the plan rules; its pair is NaN");
    return SIGK_OK;
}

extern "C" size_t sigk_ragged_tc_workspace_size(int64_t npairs, int64_t dim, int64_t nitems, int64_t bnd_elems,
                                                int precision, const sigk_ragged_tc_plan *plan)
{
    if (!plan || npairs < 1 || dim < 1 || (dim > 32 && precision != SIGK_PREC_FP64) || nitems < npairs ||
        bnd_elems < 0 || plan->a_rows < 0 ||
        plan->b_rows < 0 || plan->inc_elems < 0)
        return 0;
    RaggedPlan pl = ragged_plan(npairs, 2 * npairs, 2 * npairs, dim, nitems, bnd_elems, tsize_of(precision));
    if (precision == SIGK_PREC_FP64) return ragged_mat64_layout(pl.dx_off, dim, *plan).ws_bytes;
    return ragged_tc_layout(pl.dx_off, dim, *plan).ws_bytes;
}

extern "C" int sigk_pairwise_ragged_tc(const void *x_pack, const int64_t *x_off, const int64_t *x_len,
                                       int64_t x_points, const void *y_pack, const int64_t *y_off,
                                       const int64_t *y_len, int64_t y_points, const int *order,
                                       const int64_t *item_pair, const int *item_band, int64_t nitems,
                                       const int *pair_rows, const int *pair_bands, const int64_t *pair_bnd_off,
                                       int64_t bnd_elems, int64_t npairs, int64_t dim, int dtype,
                                       double static_scale, const void *scale_x, const void *scale_y, void *out,
                                       int precision, const sigk_ragged_tc_plan *plan, void *workspace,
                                       size_t workspace_bytes, sigk_stream_t stream)
{
    if (!plan) return fail(SIGK_EINVAL, "plan is NULL");
    return run_ragged(x_pack, x_off, x_len, x_points, y_pack, y_off, y_len, y_points, order, item_pair, item_band,
                      nitems, pair_rows, pair_bands, pair_bnd_off, bnd_elems, npairs, dim, dtype, static_scale,
                      scale_x, scale_y, out, precision, plan, workspace, workspace_bytes, (cudaStream_t)stream);
}
