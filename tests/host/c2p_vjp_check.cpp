// Host check of the reverse-mode C2P (hlld_ai_b200/csrc/c2p_vjp.cuh)
// against the dual-number tangent of the same map (cons_to_prim_tangent with
// Dual<8>, srmhd_phys.cuh).
//
// Random primitive states -- densities and pressures over three decades,
// speeds up to 0.99, fields up to |B| = 10 and B = 0 -- are mapped to
// conserved variables; every fifth case scales the momentum up by 1-30 % (so
// that some states take Kastaun's S-rescale branch) and every seventh lowers
// the density below the atmosphere.  The root mu is solved by cons_to_prim
// itself; a random primitive adjoint is then pulled back both ways.
//
// Arguments: bound (default 1e-9), cases (4000), seed (3).  Output: one line
// "worst <err> rescaled=<n> atmo=<m> cases=<k>" with the largest component
// error relative to the largest reference component of each case; exit
// status 1 if it exceeds the bound.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "c2p_vjp.cuh"

using namespace hlld;

int main(int argc, char **argv) {
    const double bound = argc > 1 ? atof(argv[1]) : 1e-9;
    const int cases = argc > 2 ? atoi(argv[2]) : 4000;
    std::mt19937_64 rng(argc > 3 ? atoi(argv[3]) : 3);
    std::uniform_real_distribution<double> U(0, 1);
    const double gamma = 5.0 / 3.0, atmo_rho = 1e-10, atmo_eps = 1e-10;
    double worst = 0;
    int nres = 0, natmo = 0;
    for (int t = 0; t < cases; ++t) {
        double P[NPRIM];
        P[P_RHO] = (t % 7 == 3) ? 1e-11 : pow(10, -2 + 3 * U(rng));
        P[P_P] = pow(10, -2 + 3 * U(rng));
        const double sp = 0.99 * U(rng), th = M_PI * U(rng), ph = 2 * M_PI * U(rng);
        P[P_VX] = sp * sin(th) * cos(ph);
        P[P_VY] = sp * sin(th) * sin(ph);
        P[P_VZ] = sp * cos(th);
        const double bs = (t % 11 == 0) ? 0.0 : 10 * U(rng);
        P[P_BX] = bs * (2 * U(rng) - 1);
        P[P_BY] = bs * (2 * U(rng) - 1);
        P[P_BZ] = bs * (2 * U(rng) - 1);
        P[P_EPS] = eos_eps(P[P_P], P[P_RHO], gamma);
        double C[NCONS];
        prim_to_cons(P, C);
        if (t % 5 == 0) {
            const double s = 1.0 + 0.3 * U(rng);
            C[C_SX] *= s;
            C[C_SY] *= s;
            C[C_SZ] *= s;
        }
        double Pout[NPRIM], mu = 0;
        const uint8_t st = cons_to_prim<double>(C, gamma, atmo_rho, atmo_eps, Pout, &mu);
        natmo += (st & ST_ATMO) != 0;
        const double S = sqrt(C[C_SX] * C[C_SX] + C[C_SY] * C[C_SY] + C[C_SZ] * C[C_SZ]);
        nres += S > C[C_D] + fmax(C[C_TAU], 0.0);
        double lP[NPRIM];
        for (int k = 0; k < NPRIM; ++k) lP[k] = 2 * U(rng) - 1;
        using D8 = Dual<NCONS>;
        D8 Cd[NCONS], Pd[NPRIM];
        for (int k = 0; k < NCONS; ++k) Cd[k] = D8::var(C[k], k);
        cons_to_prim_tangent<D8>(Cd, gamma, atmo_rho, atmo_eps, mu, Pd);
        double ref[NCONS], scale = 1e-300;
        for (int k = 0; k < NCONS; ++k) {
            double s = 0;
            for (int m = 0; m < NPRIM; ++m) s += lP[m] * Pd[m].d[k];
            ref[k] = s;
            scale = fmax(scale, fabs(s));
        }
        double lC[NCONS];
        vjp::c2p_vjp(C, gamma, atmo_rho, mu, lP, lC);
        double e = 0;
        for (int k = 0; k < NCONS; ++k) e = fmax(e, fabs(lC[k] - ref[k]) / scale);
        if (e > bound && e > worst)
            printf("case %d err %.3e status %d mu %.6g\n", t, e, (int)st, mu);
        worst = fmax(worst, e);
    }
    printf("worst %.3e rescaled=%d atmo=%d cases=%d\n", worst, nres, natmo, cases);
    return worst > bound ? 1 : 0;
}
