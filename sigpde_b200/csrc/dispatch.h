// dispatch.h -- kernel-variant getters shared by the host code and the
// translation units that instantiate the kernels (one per file so that nvcc
// compiles them in parallel).
#pragma once

#include <stdint.h>

namespace sigk {

struct PairParams;
struct NormParams;
struct StreamParams;
struct RaggedParams;
struct StreamIncParams;
struct TcImageParams;
struct TcGemmParams;
struct TcRaggedImageParams;
struct DgemmIncParams;
struct StaticIncParams;
struct GradParams;
struct RaggedDgemmParams;
struct GradContractParams;
struct FusedTcParams;
}
struct CUtensorMap_st; // cuda.h
namespace sigk {

using PairFn = void (*)(PairParams);
using NormFn = void (*)(NormParams);
using StreamFn = void (*)(StreamParams);
using RaggedFn = void (*)(RaggedParams);
using RaggedDeltaFn = void (*)(const void *, const int64_t *, const int64_t *, const int *, double, const void *,
                                int64_t, int64_t, void *);
using StreamIncFn = void (*)(StreamIncParams);
using TcImageFn = void (*)(TcImageParams);
using TcRaggedImageFn = void (*)(TcRaggedImageParams);
using DgemmIncFn = void (*)(DgemmIncParams);
using StaticIncFn = void (*)(StaticIncParams);
using TcGemmFn = void (*)(TcGemmParams, CUtensorMap_st);
using DeltaFn = void (*)(const void *, int64_t, int64_t, int64_t, int64_t, double, const void *, void *);

// f64cells: float64 cells (SIGK_PREC_FP64) vs float32; in64: float64 inputs;
// R in {2,4,8,16} rows per lane; O = min(order, 4).
// mode: kPairDelta (path differences), kPairGiven (caller's increments), kPairMat (increment matrix)
PairFn get_pair_kernel_f64(bool in64, int mode, int R, int O);
PairFn get_pair_kernel_f32(bool in64, int mode, int R, int O);
// mode: kNormDelta, kNormGiven or kNormTile (sigk_kernels.cuh)
NormFn get_norm_kernel(bool in64, int mode, int R, int O);
// one CTA per path, its bands as a warp pipeline (norm_pipe.cuh)
NormFn get_norm_pipe_kernel(bool in64, int mode, int R, int O);
// D: dimension padded to a power of two in {2,...,32}; returns null unless
// the lane's register tile (coarse rows per lane) * D <= 32.
StreamFn get_stream_reg_kernel(bool f64cells, int R, int O, int D);
StreamFn get_stream_reg_kernel_f64(int R, int O, int D);
StreamFn get_stream_reg_kernel_f32(int R, int O, int D);
// float32 cells, two pairs per lane on paired float32 instructions (same shapes)
StreamFn get_stream_reg_kernel_f32x2(int R, int O, int D);
// float64 cells, two Gram entries of one x path per lane (kOpGram only)
StreamFn get_stream_reg_kernel_f64x2(int R, int O, int D);
StreamFn get_stream_smem_kernel(bool f64cells, int R, int O);
DeltaFn get_delta_kernel(bool f64cells, bool in64);
// mat: increments from a precomputed matrix (tensor-core modes) instead of differences
// mat64: the increment matrix holds float64 (fp64 cells with a plan) instead of float32
RaggedFn get_ragged_kernel(bool f64cells, bool in64, bool mat, bool mat64 = false);
// float64 increments of an uneven batch (dgemm_inc.cuh)
using RaggedImage64Fn = void (*)(TcRaggedImageParams, double *);
RaggedImage64Fn get_ragged_image64_kernel(bool in64);
using RaggedDgemmFn = void (*)(RaggedDgemmParams);
RaggedDgemmFn get_ragged_dgemm_kernel();
// pipelined variant (half-tiles sharing their A rows) for d <= 32, null above
RaggedDgemmFn get_ragged_dgemm_pipe_kernel(int64_t d);
RaggedDeltaFn get_ragged_delta_kernel(bool f64cells, bool in64);
// Tensor-core increments (tc.cuh): operand images, the TF32x3 GEMM (N tile
// kTcBN) and the streaming wavefront that reads its output.
constexpr int kTcBN = 256;
TcImageFn get_tc_image_kernel(bool in64);
TcGemmFn get_tc_gemm_kernel(int bn = kTcBN); // 128 x bn tiles, bn in {128, 256}
TcRaggedImageFn get_tc_ragged_image_kernel(bool in64);
// float64 increment matrix on the CUDA cores (dgemm_inc.cuh)
DgemmIncFn get_dgemm_inc_kernel();
// pipelined variant for d <= 32 (null above), and its dynamic shared memory
DgemmIncFn get_dgemm_inc_pipe_kernel(int64_t d);
size_t dgemm_inc_pipe_smem(int64_t d);
// float64 increment matrix of the RBF / L1-RBF static kernel from the path points (static_inc.cuh);
// null for dim > 32
// out64: float64 matrix (float64 cells), else float32 (float32 cells)
StaticIncFn get_static_inc_kernel(int kind, int64_t dim, bool out64);
// backward pass (grad.cuh): forward-with-derivatives and adjoint wavefronts for R rows a lane,
// order O (R >= 2^O); null members where the combination is not built
struct GradFns {
    void (*fwd)(GradParams);
    void (*bwd)(GradParams);
};
GradFns get_grad_kernels(int R, int O);
struct GradAuxFns {
    void (*pair_inc)(const double *, const double *, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, double *);
    void (*gx)(GradContractParams);
    void (*gy)(GradContractParams);
    void (*reduce)(const double *, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, double *);
    void (*points)(const double *, int64_t, int64_t, int64_t, double, const void *, int, void *);
    void (*rows)(const double *, int64_t, int64_t, int64_t, int64_t, double *);
    void (*gy_gram)(GradContractParams);
    void (*inc_blocks)(const void *, int, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t,
                       const void *, const void *, double *, void *, int);
};
GradAuxFns get_grad_aux_kernels();
// mat64: the increment matrix holds float64 (dgemm_inc_kernel) instead of float32 (tensor cores)
// W: lanes a pair pipeline (32, or 16 for pairs of at most 16 R rows with R <= 8)
StreamIncFn get_stream_inc_kernel(bool f64cells, int R, int O, bool mat64, int W = 32);
// Fused tensor-core Gram (fused_tc.cuh): tcgen05 increments handed to the wavefront through shared
// memory; R rows a lane at order O (R >= 2^O, R >> O <= 4), null where not built
using FusedTcFn = void (*)(FusedTcParams);
FusedTcFn get_fused_tc_kernel(int R, int O, int ring); // ring: 16 or 8 steps between boundaries

} // namespace sigk
