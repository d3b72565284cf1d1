// Host check of the hand-written reverse mode of the face solvers
// (hlld_ai_b200/csrc/face_vjp.cuh) against forward-mode dual numbers.
//
// The device physics headers compile as plain C++ (the CUDA headers define
// __device__ away for a host compiler).  For random face states -- sub- and
// ultra-relativistic velocities, densities and pressures over two decades,
// B_n = 0 on every seventh case -- the vector-Jacobian product of the HLLE
// and HLLD fluxes with a random flux adjoint is compared with the same
// contraction of a Dual<18> evaluation of the forward solver (nine
// primitives per side; HLLD at the solved p* through the implicit-function
// theorem, its HLLE fallback where the forward one failed).
//
// Arguments: bound (default 1e-9), cases (4000), seed (11).  Output: one
// line "worst <hlle> <hlld_fallback> <hlld> failed=<n> cases=<m>" with the
// largest component error relative to the largest reference component of
// each case; exit status 1 if any exceeds the bound.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "face_vjp.cuh"

using namespace hlld;

int main(int argc, char **argv) {
    const double bound = argc > 1 ? atof(argv[1]) : 1e-9;
    const int cases = argc > 2 ? atoi(argv[2]) : 4000;
    std::mt19937_64 rng(argc > 3 ? atoi(argv[3]) : 11);
    std::uniform_real_distribution<double> U(0, 1);
    const double gamma = 5.0 / 3.0;
    double worst[3] = {0, 0, 0};
    int nfail = 0;
    for (int t = 0; t < cases; ++t) {
        double PL[NPRIM], PR[NPRIM];
        for (int s = 0; s < 2; ++s) {
            double *P = s ? PR : PL;
            P[P_RHO] = pow(10, -1 + 2 * U(rng));
            P[P_P] = pow(10, -1 + 2 * U(rng));
            const double sp = 0.95 * U(rng), th = M_PI * U(rng), ph = 2 * M_PI * U(rng);
            P[P_VX] = sp * sin(th) * cos(ph);
            P[P_VY] = sp * sin(th) * sin(ph);
            P[P_VZ] = sp * cos(th);
            P[P_BY] = -3 + 6 * U(rng);
            P[P_BZ] = -3 + 6 * U(rng);
        }
        PL[P_BX] = PR[P_BX] = (t % 7 == 0) ? 0.0 : -2 + 4 * U(rng);
        for (int s = 0; s < 2; ++s) {
            double *P = s ? PR : PL;
            P[P_EPS] = eos_eps(P[P_P], P[P_RHO], gamma);
        }
        FaceOut<double> o;
        hlld_face<0, double>(PL, PR, gamma, false, o);
        const bool failed = (o.flags & RF_FAILED) != 0;
        nfail += failed;
        const double given[2] = {o.pstar, failed ? 1.0 : 0.0};
        double lam[NCONS];
        for (int k = 0; k < NCONS; ++k) lam[k] = -1 + 2 * U(rng);
        using D = Dual<18>;
        D DL[NPRIM], DR[NPRIM];
        for (int k = 0; k < NPRIM; ++k) {
            DL[k] = D::var(PL[k], k);
            DR[k] = D::var(PR[k], 9 + k);
        }
        for (int solver = 0; solver < 2; ++solver) {
            FaceOut<D> od;
            if (solver == 1) hlld_face<0, D, D, D, true>(DL, DR, D(gamma), false, od, given);
            else hlle_face<0, D>(DL, DR, D(gamma), false, false, od);
            double ref[18], scale = 1e-300;
            for (int j = 0; j < 18; ++j) {
                double s = 0;
                for (int k = 0; k < NCONS; ++k) s += lam[k] * od.F[k].d[j];
                ref[j] = s;
                scale = fmax(scale, fabs(s));
            }
            double aL[NPRIM] = {}, aR[NPRIM] = {};
            if (solver == 1) vjp::hlld_face_vjp<0>(PL, PR, gamma, o.pstar, failed, lam, aL, aR);
            else vjp::hlle_face_vjp<0>(PL, PR, gamma, lam, aL, aR);
            const int w = solver == 0 ? 0 : (failed ? 1 : 2);
            for (int j = 0; j < 18; ++j) {
                const double got = j < 9 ? aL[j] : aR[j - 9];
                worst[w] = fmax(worst[w], fabs(got - ref[j]) / scale);
            }
        }
    }
    printf("worst %.3e %.3e %.3e failed=%d cases=%d\n", worst[0], worst[1], worst[2], nfail, cases);
    return (worst[0] > bound || worst[1] > bound || worst[2] > bound) ? 1 : 0;
}
