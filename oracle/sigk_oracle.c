/*
 * sigk_oracle.c -- FP64 CPU restatement of the SigPDE signature-kernel hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the CUDA product is
 * checked against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product library never links or calls it.
 *
 * What is restated (paths are relative to the stojl/SigPDE project root):
 *   - the Goursat stencil          sigpde/cuda_device_functions.py:3-5
 *   - the per-pair cell loop       sigpde/cuda_pairwise_kernels.py:17-39
 *       (rows i in [1,lx-1], columns j in [1,ly-1], coarse increment at
 *        ((i-1)>>order, (j-1)>>order), boundary K = 1 on row 0 / column 0,
 *        result = K[lx-1][ly-1])
 *   - the scaled variant           sigpde/cuda_pairwise_kernels.py:41-85
 *       (inc * scale_x * scale_y)
 *   - the LinearKernel increments  sigpde/torch/kernel.py:13-21 with
 *                                  sigpde/torch/static_kernels.py:3-11
 *       (4-term second difference of the static Gram, divided by 4^order)
 *   - the Chandrupatla lambda loop sigpde/cuda_pairwise_kernels.py:88-165
 *       with the argument order of sigpde/torch/kernel.py:180-195
 *   - the gradient of a solve with respect to its increments (the adjoint of
 *     the scheme; the reference has none): sko_grad_solve, checked against
 *     central differences of sko_solve by the tests
 *
 * Arithmetic follows the reference expression order exactly and must be
 * compiled without FMA contraction (-ffp-contract=off), so that float64
 * inputs reproduce the reference's float64 results bit for bit.
 *
 * `store_f32` != 0 rounds every stored cell to float32, which models the
 * reference's GPU semantics for float32 inputs (float64 arithmetic because of
 * the double literals in pde_step, float32 scratch storage).
 *
 * Parity of this restatement is pinned against outputs of the reference run
 * under NUMBA_ENABLE_CUDASIM=1 (tests/golden/gen_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* sigpde/cuda_device_functions.py:3-5 */
static inline double pde_step(double k00, double k01, double k10, double inc)
{
    const double inc2 = inc * inc;
    return (k01 + k10) * (1. + 0.5 * inc + (1. / 12) * inc2) - k00 * (1. - (1. / 12) * inc2);
}

static inline double store(double v, int store_f32) { return store_f32 ? (double)(float)v : v; }

/*
 * One Goursat solve on the dyadically refined grid.
 * inc: (ncx, ncy) row-major coarse increments (already divided by 4^order).
 * Row-by-row order gives the same values as the reference's anti-diagonal
 * order: every cell reads the same three neighbours either way.
 * Follows sigpde/cuda_pairwise_kernels.py:17-39 (scale == 1) and :41-85.
 */
double sko_solve(const double *inc, int64_t ncx, int64_t ncy, int order, double scale, int store_f32,
                 double *row_buf /* 2*(ly) doubles or NULL */)
{
    const int64_t lx = (ncx << order) + 1; /* sigpde/utils.py:6-7 */
    const int64_t ly = (ncy << order) + 1;
    double *buf = row_buf;
    int own = 0;
    if (!buf) {
        buf = (double *)malloc(sizeof(double) * 2 * (size_t)ly);
        own = 1;
    }
    double *prev = buf, *cur = buf + ly;
    for (int64_t j = 0; j < ly; ++j) prev[j] = 1.0;
    for (int64_t i = 1; i < lx; ++i) {
        cur[0] = 1.0;
        const double *irow = inc + ((i - 1) >> order) * ncy;
        for (int64_t j = 1; j < ly; ++j) {
            double c = irow[(j - 1) >> order];
            if (scale != 1.0) c = c * scale;
            cur[j] = store(pde_step(prev[j - 1], prev[j], cur[j - 1], c), store_f32);
        }
        double *t = prev; prev = cur; cur = t;
    }
    double r = (lx == 1 || ly == 1) ? 1.0 : prev[ly - 1];
    if (own) free(buf);
    return r;
}

/*
 * LinearKernel increments for one pair (x: (Lx,d), y: (Ly,d), row-major):
 *   ip[p][q] = scale * <x_p, y_q>                    static_kernels.py:7-8
 *   inc[i][j] = (ip[i+1][j+1] + ip[i][j] - ip[i+1][j] - ip[i][j+1]) / 4^order
 *                                                     kernel.py:13-16
 * The 4-term expression is evaluated left to right as in the reference.
 */
void sko_increments_linear(const double *x, const double *y, int64_t Lx, int64_t Ly, int64_t d, int order,
                           double static_scale, double *inc)
{
    double *ip = (double *)malloc(sizeof(double) * (size_t)(Lx * Ly));
    for (int64_t p = 0; p < Lx; ++p)
        for (int64_t q = 0; q < Ly; ++q) {
            double s = 0.0;
            for (int64_t k = 0; k < d; ++k) s += x[p * d + k] * y[q * d + k];
            ip[p * Ly + q] = static_scale * s;
        }
    const double denom = (double)(1LL << (2 * order));
    for (int64_t i = 0; i + 1 < Lx; ++i)
        for (int64_t j = 0; j + 1 < Ly; ++j) {
            double v = ip[(i + 1) * Ly + (j + 1)] + ip[i * Ly + j] - ip[(i + 1) * Ly + j] - ip[i * Ly + (j + 1)];
            inc[i * (Ly - 1) + j] = v / denom;
        }
    free(ip);
}

/*
 * Batched solve over precomputed increments.
 * incs: (npairs, ncx, ncy); sx, sy: per-pair scales or NULL (scaled kernels
 * multiply inc by scale_x * scale_y, cuda_pairwise_kernels.py:61,69).
 */
void sko_solve_batch(const double *incs, int64_t npairs, int64_t ncx, int64_t ncy, int order, const double *sx,
                     const double *sy, int store_f32, double *out)
{
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)((ncy << order) + 1));
#pragma omp for schedule(dynamic, 1)
        for (int64_t b = 0; b < npairs; ++b) {
            double s = 1.0;
            if (sx || sy) s = (sy ? sy[b] : 1.0) * (sx ? sx[b] : 1.0);
            out[b] = sko_solve(incs + b * ncx * ncy, ncx, ncy, order, s, store_f32, buf);
        }
        free(buf);
    }
}

/*
 * Pairwise LinearKernel signature kernel (SigPDE.pairwise, kernel.py:31-65):
 * x: (B,Lx,d), y: (B,Ly,d); out: (B,).
 */
void sko_pairwise_linear(const double *x, const double *y, int64_t B, int64_t Lx, int64_t Ly, int64_t d, int order,
                         double static_scale, const double *sx, const double *sy, int store_f32, double *out)
{
    const int64_t ncx = Lx - 1, ncy = Ly - 1;
#pragma omp parallel
    {
        double *inc = (double *)malloc(sizeof(double) * (size_t)(ncx * ncy > 0 ? ncx * ncy : 1));
        double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)((ncy << order) + 1));
#pragma omp for schedule(dynamic, 1)
        for (int64_t b = 0; b < B; ++b) {
            sko_increments_linear(x + b * Lx * d, y + b * Ly * d, Lx, Ly, d, order, static_scale, inc);
            double s = 1.0;
            if (sx || sy) s = (sy ? sy[b] : 1.0) * (sx ? sx[b] : 1.0);
            out[b] = sko_solve(inc, ncx, ncy, order, s, store_f32, buf);
        }
        free(buf);
        free(inc);
    }
}

/*
 * Gram LinearKernel signature kernel (SigPDE._gram, kernel.py:75-126):
 * x: (Nx,Lx,d), y: (Ny,Ly,d); out: (Nx,Ny) row-major.  Scaled entries use
 * scale_x[i] * scale_y[j] (cuda_gram_kernels.py:52).
 * `pairs`/`npairs` optionally restrict the work to a list of flat indices
 * i*Ny+j (for sampled checks); when pairs == NULL every entry is computed.
 */
void sko_gram_linear(const double *x, const double *y, int64_t Nx, int64_t Ny, int64_t Lx, int64_t Ly, int64_t d,
                     int order, double static_scale, const double *sx, const double *sy, int store_f32,
                     const int64_t *pairs, int64_t npairs, double *out)
{
    const int64_t ncx = Lx - 1, ncy = Ly - 1;
    const int64_t total = pairs ? npairs : Nx * Ny;
#pragma omp parallel
    {
        double *inc = (double *)malloc(sizeof(double) * (size_t)(ncx * ncy > 0 ? ncx * ncy : 1));
        double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)((ncy << order) + 1));
#pragma omp for schedule(dynamic, 1)
        for (int64_t t = 0; t < total; ++t) {
            const int64_t f = pairs ? pairs[t] : t;
            const int64_t i = f / Ny, j = f % Ny;
            sko_increments_linear(x + i * Lx * d, y + j * Ly * d, Lx, Ly, d, order, static_scale, inc);
            double s = 1.0;
            if (sx || sy) s = (sx ? sx[i] : 1.0) * (sy ? sy[j] : 1.0);
            out[pairs ? t : f] = sko_solve(inc, ncx, ncy, order, s, store_f32, buf);
        }
        free(buf);
        free(inc);
    }
}

/*
 * Chandrupatla root-find for the robust normalisation of one path.
 * Restates sigpde/cuda_pairwise_kernels.py:88-165 as called from
 * sigpde/torch/kernel.py:180-195:
 *   the kernel parameter `norms` receives fk = f(k(x,x)) and `f_norms`
 *   receives k = k(x,x), so the bracket is lambda in [0,1] for
 *   g(lambda) = k(lambda x, lambda x) - f(k),  g(0) = 1 - fk,  g(1) = k - fk.
 * Each iteration re-solves the PDE with inc * xt^2.  A NaN solve maps to +inf
 * (:144).  Division is IEEE (inf/NaN propagate) as on the GPU.
 * Returns the best end point; *iters receives the iteration count used.
 */
double sko_chandrupatla(const double *inc, int64_t nc, int order, double k, double fk, double tol, int maxit,
                        int store_f32, int *iters)
{
    double a = 0.0, c = 0.0, b = 1.0;
    double fa = 1.0 - fk;
    double fb = k - fk;
    double fc = fa;
    double t = 0.5;
    double out = 0.0;
    int it = 0;
    double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)((nc << order) + 1));
    for (it = 0; it < maxit; ++it) {
        const double xt = a + t * (b - a);
        const double sol = sko_solve(inc, nc, nc, order, xt * xt, store_f32, buf);
        const double ft = isnan(sol) ? INFINITY : store(sol - fk, store_f32);
        if (ft * fa >= 0) {
            c = a;
            fc = fa;
        } else {
            c = b;
            b = a;
            fc = fb;
            fb = fa;
        }
        a = xt;
        fa = ft;
        if (fabs(fa) < fabs(fb)) {
            out = a;
            if (fabs(fa) < tol) { ++it; break; }
        } else {
            out = b;
            if (fabs(fb) < tol) { ++it; break; }
        }
        const double xi = (a - b) / (c - b);
        const double phi = (fa - fb) / (fc - fb);
        if (phi * phi < xi && (1 - phi) * (1 - phi) < 1 - xi)
            t = fa / (fb - fa) * fc / (fb - fc) + (c - a) / (b - a) * fa / (fc - fa) * fb / (fc - fb);
        else
            t = 0.5;
        if (!(0 < t && t < 1)) t = 0.5;
    }
    free(buf);
    if (iters) *iters = it;
    return out;
}

/*
 * Batched lambda solve: incs (B, nc, nc) self-increments, k (B,), fk (B,).
 * Applies the post-processing of kernel.py:195 (lambda = 0 where k < 1).
 */
void sko_chandrupatla_batch(const double *incs, int64_t B, int64_t nc, int order, const double *k, const double *fk,
                            double tol, int maxit, int store_f32, double *lam, int *iters)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < B; ++b) {
        double l = sko_chandrupatla(incs + b * nc * nc, nc, order, k[b], fk[b], tol, maxit, store_f32,
                                    iters ? iters + b : NULL);
        lam[b] = (k[b] < 1) ? 0.0 : l;
    }
}

/*
 * Gradient of one solve with respect to its coarse increments: the adjoint of
 * the scheme above (the reference has no backward pass; this restates the
 * calculus of pde_step, sigpde/cuda_device_functions.py:3-5).
 *   c = inc * scale,  A(c) = 1 + c/2 + c^2/12,  B(c) = 1 - c^2/12,
 *   K[p][q] = (K[p][q-1] + K[p-1][q]) A(c_pq) - K[p-1][q-1] B(c_pq).
 * Lambda = w * dK[lx-1][ly-1] / dK over the nodes, in reverse row-major order:
 *   Lambda[p][q] = A(c_p,q+1) Lambda[p][q+1] + A(c_p+1,q) Lambda[p+1][q]
 *                  - B(c_p+1,q+1) Lambda[p+1][q+1]        (absent terms are 0)
 * with Lambda[lx-1][ly-1] = w, and each cell adds
 *   Lambda[p][q] * ((K[p][q-1] + K[p-1][q]) A'(c) - K[p-1][q-1] B'(c)),
 *   A'(c) = 1/2 + c/6, B'(c) = -c/6,
 * to G at its coarse cell.  G = w * dK / dc (ncx x ncy); returns K[lx-1][ly-1].
 */
static inline double coef_a(double c) { return 1. + 0.5 * c + (1. / 12) * (c * c); }
static inline double coef_b(double c) { return 1. - (1. / 12) * (c * c); }

double sko_grad_solve(const double *inc, int64_t ncx, int64_t ncy, int order, double scale, double w, double *G)
{
    const int64_t lx = (ncx << order) + 1, ly = (ncy << order) + 1;
    double *K = (double *)malloc(sizeof(double) * (size_t)(lx * ly));
    double *Lm = (double *)calloc((size_t)(lx * ly), sizeof(double));
#define CELL(p, q) (inc[(((p) - 1) >> order) * ncy + (((q) - 1) >> order)] * scale)
    for (int64_t q = 0; q < ly; ++q) K[q] = 1.0;
    for (int64_t p = 1; p < lx; ++p) {
        K[p * ly] = 1.0;
        for (int64_t q = 1; q < ly; ++q) {
            const double c = CELL(p, q);
            K[p * ly + q] = (K[p * ly + q - 1] + K[(p - 1) * ly + q]) * coef_a(c) - K[(p - 1) * ly + q - 1] * coef_b(c);
        }
    }
    memset(G, 0, sizeof(double) * (size_t)(ncx * ncy));
    for (int64_t p = lx - 1; p >= 1; --p)
        for (int64_t q = ly - 1; q >= 1; --q) {
            double lam = (p == lx - 1 && q == ly - 1) ? w : 0.0;
            if (q + 1 < ly) lam += coef_a(CELL(p, q + 1)) * Lm[p * ly + q + 1];
            if (p + 1 < lx) lam += coef_a(CELL(p + 1, q)) * Lm[(p + 1) * ly + q];
            if (p + 1 < lx && q + 1 < ly) lam -= coef_b(CELL(p + 1, q + 1)) * Lm[(p + 1) * ly + q + 1];
            Lm[p * ly + q] = lam;
            const double c = CELL(p, q);
            const double dk = (K[p * ly + q - 1] + K[(p - 1) * ly + q]) * (0.5 + c / 6.) - K[(p - 1) * ly + q - 1] * (-c / 6.);
            G[((p - 1) >> order) * ncy + ((q - 1) >> order)] += lam * dk;
        }
#undef CELL
    const double r = K[lx * ly - 1];
    free(K);
    free(Lm);
    return r;
}

/* sko_grad_solve over a batch of increment blocks (npairs, ncx, ncy) with per-pair scale and weight. */
void sko_grad_solve_batch(const double *incs, int64_t npairs, int64_t ncx, int64_t ncy, int order,
                          const double *scale, const double *w, double *G, double *out)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < npairs; ++b)
        out[b] = sko_grad_solve(incs + b * ncx * ncy, ncx, ncy, order, scale ? scale[b] : 1.0, w ? w[b] : 1.0,
                                G + b * ncx * ncy);
}

int sko_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void sko_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
