// Device check of nr_sqrt (hlld_ai_b200/csrc/srmhd_phys.cuh), the Newton
// square root of the mixed form's FP64 p* residual and Kastaun master
// function, against CUDA's correctly rounded sqrt on the same inputs.
//
// Inputs: n positive doubles with exponents spread over [1e-300, 1e300] and
// random mantissas (a fixed-seed LCG on the host), the two ends of the
// documented domain (2^-1000 and the double below 2^1000), 0 and a NaN.
// Output: one line "max_ulp <k> n=<n> zero_ok=<0|1> nan_ok=<0|1>"; exit
// status 1 if any result of the domain is more than `bound` ulp (default 2)
// from sqrt(x) or not finite, if 0 does not give 0, or the NaN no NaN.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "srmhd_phys.cuh"

__global__ void sqrt_kernel(const double *x, double *nr, double *ref, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        nr[i] = hlld::nr_sqrt(x[i]);
        ref[i] = sqrt(x[i]);
    }
}

int main(int argc, char **argv) {
    const long long bound = argc > 1 ? atoll(argv[1]) : 2;
    const double ends[] = {0x1p-1000, nextafter(0x1p1000, 0.0)};
    const int nends = (int)(sizeof(ends) / sizeof(ends[0]));
    const int nr = (1 << 20) + nends;  // inputs of the domain
    const int n = nr + 2;              // then 0 and a NaN
    std::vector<double> h(n), a(n), b(n);
    uint64_t s = 88172645463325252ull;
    h[nr] = 0.0;
    h[nr + 1] = NAN;
    for (int k = 0; k < nends; ++k) h[nr - nends + k] = ends[k];
    for (int i = 0; i < nr - nends; ++i) {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        const double u = (double)(s >> 11) / 9007199254740992.0;  // [0, 1)
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        const double m = 1.0 + (double)(s >> 11) / 9007199254740992.0;  // [1, 2)
        h[i] = m * pow(10.0, -300.0 + 600.0 * u);
    }
    double *dx, *dn, *dr;
    if (cudaMalloc(&dx, n * 8) || cudaMalloc(&dn, n * 8) || cudaMalloc(&dr, n * 8)) return 2;
    cudaMemcpy(dx, h.data(), n * 8, cudaMemcpyHostToDevice);
    sqrt_kernel<<<(n + 255) / 256, 256>>>(dx, dn, dr, n);
    if (cudaDeviceSynchronize() != cudaSuccess) return 2;
    cudaMemcpy(a.data(), dn, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(b.data(), dr, n * 8, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dn);
    cudaFree(dr);
    long long worst = 0;
    bool bad = false;
    for (int i = 0; i < nr; ++i) {
        if (!std::isfinite(a[i])) { bad = true; continue; }
        int64_t ia, ib;
        memcpy(&ia, &a[i], 8);
        memcpy(&ib, &b[i], 8);
        const long long du = llabs((long long)(ia - ib));
        if (du > worst) worst = du;
    }
    const bool zero_ok = a[nr] == 0.0;
    const bool nan_ok = std::isnan(a[nr + 1]);
    printf("max_ulp %lld n=%d zero_ok=%d nan_ok=%d\n", worst, nr, zero_ok ? 1 : 0, nan_ok ? 1 : 0);
    return (bad || worst > bound || !zero_ok || !nan_ok) ? 1 : 0;
}
