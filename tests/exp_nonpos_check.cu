// Checks sigk::exp_nonpos (static_inc.cuh) against CUDA's exp on a dense sweep
// of [-707.5, 0] plus arguments a few ulps above 0; prints the largest
// relative difference and the largest difference in units of the last place.
// Built and run by tests/test_exp_gpu.py.
#include <cstdio>
#include <cmath>
#include <vector>
#include "static_inc.cuh"

__global__ void sweep(int n, double lo, double *rel, double *ulp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = i < n - 8 ? lo * (double)i / (n - 9) : 1e-16 * (i - (n - 8));
    const double e = exp(a), o = sigk::exp_nonpos(a);
    rel[i] = fabs(o - e) / e;
    ulp[i] = fabs(o - e) / (nextafter(e, 2.0 * e + 1.0) - e);
}

int main()
{
    const int n = 1 << 22;
    double *rel, *ulp;
    if (cudaMalloc(&rel, n * sizeof(double)) != cudaSuccess || cudaMalloc(&ulp, n * sizeof(double)) != cudaSuccess)
        return 2;
    sweep<<<(n + 255) / 256, 256>>>(n, -707.5, rel, ulp);
    std::vector<double> hr(n), hu(n);
    if (cudaMemcpy(hr.data(), rel, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return 3;
    if (cudaMemcpy(hu.data(), ulp, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return 3;
    double mr = 0, mu = 0;
    for (int i = 0; i < n; ++i) {
        mr = fmax(mr, hr[i]);
        mu = fmax(mu, hu[i]);
    }
    printf("max_rel %.6e max_ulp %.3f\n", mr, mu);
    return 0;
}
