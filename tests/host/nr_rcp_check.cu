// Device check of nr_rcp (hlld_ai_b200/csrc/srmhd_phys.cuh), the Newton
// reciprocal of the mixed form's FP64 p* solve, against CUDA's correctly
// rounded division 1.0 / d on the same inputs.
//
// Inputs: n doubles of both signs with exponents spread over [1e-300, 1e300]
// and random mantissas (a fixed-seed LCG on the host), the two ends of the
// documented domain 2^-1000 <= |d| < 2^1000 (both signs), and a NaN, whose
// result must be a NaN.  Output: one line "max_ulp <k> n=<n> nan_ok=<0|1>";
// exit status 1 if any result of the domain is more than `bound` ulp
// (default 2) from 1.0 / d or not finite, or the NaN does not give a NaN.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "srmhd_phys.cuh"

__global__ void rcp_kernel(const double *d, double *nr, double *ref, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        nr[i] = hlld::nr_rcp(d[i]);
        ref[i] = 1.0 / d[i];
    }
}

int main(int argc, char **argv) {
    const long long bound = argc > 1 ? atoll(argv[1]) : 2;
    const double ends[] = {0x1p-1000, -0x1p-1000, nextafter(0x1p1000, 0.0),
                           -nextafter(0x1p1000, 0.0)};
    const int nends = (int)(sizeof(ends) / sizeof(ends[0]));
    const int nr = (1 << 20) + nends;  // inputs of the domain
    const int n = nr + 1;              // and a NaN
    std::vector<double> h(n), a(n), b(n);
    uint64_t s = 88172645463325252ull;
    h[nr] = NAN;
    for (int k = 0; k < nends; ++k) h[nr - nends + k] = ends[k];
    for (int i = 0; i < nr - nends; ++i) {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        const double u = (double)(s >> 11) / 9007199254740992.0;  // [0, 1)
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        const double m = 1.0 + (double)(s >> 11) / 9007199254740992.0;  // [1, 2)
        const double e = -300.0 + 600.0 * u;
        h[i] = ((i & 1) ? -1.0 : 1.0) * m * pow(10.0, e);
    }
    double *dd, *dn, *dr;
    if (cudaMalloc(&dd, n * 8) || cudaMalloc(&dn, n * 8) || cudaMalloc(&dr, n * 8)) return 2;
    cudaMemcpy(dd, h.data(), n * 8, cudaMemcpyHostToDevice);
    rcp_kernel<<<(n + 255) / 256, 256>>>(dd, dn, dr, n);
    if (cudaDeviceSynchronize() != cudaSuccess) return 2;
    cudaMemcpy(a.data(), dn, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(b.data(), dr, n * 8, cudaMemcpyDeviceToHost);
    cudaFree(dd);
    cudaFree(dn);
    cudaFree(dr);
    long long worst = 0;
    bool bad = false;
    const bool nan_ok = std::isnan(a[nr]) && std::isnan(b[nr]);
    for (int i = 0; i < nr; ++i) {
        if (!std::isfinite(a[i])) { bad = true; continue; }
        int64_t ia, ib;
        memcpy(&ia, &a[i], 8);
        memcpy(&ib, &b[i], 8);
        const long long du = llabs((long long)(ia - ib));
        if (du > worst) worst = du;
    }
    printf("max_ulp %lld n=%d nan_ok=%d\n", worst, nr, nan_ok ? 1 : 0);
    return (bad || worst > bound || !nan_ok) ? 1 : 0;
}
