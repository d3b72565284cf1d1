// Discrete adjoint of the FP64 2D step (SSP-RK2/3 + CT), included by the
// FP64 variant after kernels_impl.cuh (same namespace, R = double).
//
// The adjoint of one step maps lambda of the step's output state (the
// evolved cell variables, the staggered field and the primitives) to
// lambda of its input, with the step's time step held fixed.  It is the
// exact transpose of the forward step's Jacobian with every discrete
// decision frozen at its forward outcome: limiter branches and the PCM
// positivity fallback of the reconstruction, HLLD region selection and the
// HLLD -> HLLE fallback, the upwind signs (and deadband) of the corner EMF,
// clamps and floors.  The two root solves are differentiated by the
// implicit-function theorem: the HLLD total pressure p* (residual
// hlld.py:586-602) and the Kastaun root mu of the C2P master function
// (c2p.py:129-158), both in dual arithmetic from the solved root.
//
// Reverse of stage s (driver2d.py:183-192 combine + sync):
//   a. primitive ghost fill (fold the ghost lambdas onto their sources)
//   b. C2P of the physical cells (reverse mode at the recorded root, IFT on
//      mu: c2p_vjp.cuh)
//   c. cell-centred B -> faces
//   d. conserved and face ghost fills
//   e. RK combine and flux divergence / CT curl -> lambda of the fluxes and
//      corner EMFs, and of U0 / U_s
//   f. corner EMF (ct.py:119-177) -> transverse-B fluxes, cell E -> v, B
//   g. the two sweeps: per face the Riemann solver in reverse mode at the
//      forward p* (face_vjp.cuh), then the primitive conversion and the
//      reconstruction (Dual over the stencil) in reverse, gathered onto
//      cells without atomics.
#pragma once

#include "c2p_vjp.cuh"
#include "face_vjp.cuh"

namespace hlld {
namespace HLLD_NS {

// blocks of kThreads per SM the adjoint sweep is compiled for (its register
// cap: 65536 / (kThreads * min blocks), at most 255)
#ifndef HLLD_ADJ_SWEEP_MIN_BLOCKS
#define HLLD_ADJ_SWEEP_MIN_BLOCKS 2
#endif

constexpr int kAdjDirs = 15;  // rho, p, vx, vy, vz, B_t, Bz per side + B_n
constexpr int kMaxNW = 8;     // widest reconstruction window (MP7)

struct AdjSweepParams {
    Grid g;
    const double *rho, *p, *vx, *vy, *vz, *bz;
    const double *Bxf, *Byf;
    const double *lamF[NFLUX];
    const double *pstar_in;    // the forward sweep's p* and fallback per face
    const uint8_t *fail_in;
    double *lamS[kMaxNW * 7];  // [slot * 7 + var] per face
    double *lamBn;
};

// Adjoint of one face of sweep_kernel<AXIS, LIM, SOLVER> (FP64).
template <int AXIS, int LIM, int SOLVER>
__global__ void __launch_bounds__(kThreads, HLLD_ADJ_SWEEP_MIN_BLOCKS) adj_sweep_kernel(const AdjSweepParams p) {
    constexpr int S = Stencil<LIM>::S;
    constexpr int NW = 2 * S + 2;
    const Grid &g = p.g;
    const int cols = AXIS == 0 ? g.nyt : g.nyt + 1;
    const int rows = AXIS == 0 ? g.nxt + 1 : g.nxt;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows * cols) return;
    const int row = (int)(e / cols), col = (int)(e - (int64_t)row * cols);
    const int f = AXIS == 0 ? row : col;
    const int tr = AXIS == 0 ? col : row;
    const int n = AXIS == 0 ? g.nxt : g.nyt;
    const int64_t cstride = AXIS == 0 ? g.nyt : 1;
    const int64_t cbase = AXIS == 0 ? (int64_t)tr : (int64_t)tr * g.nyt;
    auto bt_at = [&](int c) -> double {
        return AXIS == 0 ? 0.5 * (p.Byf[(int64_t)c * (g.nyt + 1) + tr] + p.Byf[(int64_t)c * (g.nyt + 1) + tr + 1])
                         : 0.5 * (p.Bxf[(int64_t)tr * g.nyt + c] + p.Bxf[(int64_t)(tr + 1) * g.nyt + c]);
    };
    const bool edge = (f == 0 || f == n);
    // window: cells f-1-S .. f+S (clamped; clamped entries are never read)
    int cw[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        int c = f - 1 - S + k;
        cw[k] = c < 0 ? 0 : (c > n - 1 ? n - 1 : c);
    }
    // on an outermost face the edge cell sits in slot S + 1 (f = 0) or S (f = n)
    // work variables of window slot k (reconstruction.py:269): rho, p, W v,
    // B_t, Bz; velocities and W kept for the conversion's reverse
    auto load_slot = [&](int k, double *qk, double *vk, double &W) {
        const int64_t ci = cbase + cw[k] * cstride;
        vk[0] = p.vx[ci];
        vk[1] = p.vy[ci];
        vk[2] = p.vz[ci];
        double v2 = vk[0] * vk[0] + vk[1] * vk[1] + vk[2] * vk[2];
        W = 1.0 / sqrt(clamp_lo(1.0 - v2, 1e-14));
        qk[0] = p.rho[ci];
        qk[1] = p.p[ci];
        qk[2] = W * vk[0];
        qk[3] = W * vk[1];
        qk[4] = W * vk[2];
        qk[5] = bt_at(cw[k]);
        qk[6] = p.bz[ci];
    };
    const double bn = AXIS == 0 ? p.Bxf[(int64_t)f * g.nyt + tr] : p.Byf[(int64_t)tr * (g.nyt + 1) + f];
    constexpr int IBT = AXIS == 0 ? P_BY : P_BX;
    constexpr int IBN = AXIS == 0 ? P_BX : P_BY;
    // forward face states.  Only what the reverse of the conversion needs is
    // kept through the Riemann solver's reverse (the face's W v, its
    // 1/sqrt(1 + (W v)^2) and the floor flags); the window is loaded again
    // afterwards for the reconstruction's reverse.
    double PL[NPRIM], PR[NPRIM], fac[2], zq[2][3];
    bool floor_rho[2], floor_p[2];
    bool bad = false;
    {
        double q[7][NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            double qk[7], vk[3], W;
            load_slot(k, qk, vk, W);
#pragma unroll
            for (int v = 0; v < 7; ++v) q[v][k] = qk[v];
        }
        double L[7], Rt[7];
        if (edge) {
#pragma unroll
            for (int v = 0; v < 7; ++v) {
                const double x = f == 0 ? q[v][S + 1] : q[v][S];  // constant slots: registers
                L[v] = x + 0.5 * 0.0;
                Rt[v] = x - 0.5 * 0.0;
            }
        } else {
#pragma unroll
            for (int v = 0; v < 7; ++v) {
                L[v] = cell_edge<LIM, true, S>(q[v], f - 1, n);
                Rt[v] = cell_edge<LIM, false, S + 1>(q[v], f, n);
            }
            if (LIM != HLLD_LIM_PCM) {
                bad = (L[0] <= 1e-12) || (Rt[0] <= 1e-12) || (L[1] <= 1e-14) || (Rt[1] <= 1e-14);
                if (bad) {
#pragma unroll
                    for (int v = 0; v < 7; ++v) {
                        L[v] = q[v][S] + 0.5 * 0.0;
                        Rt[v] = q[v][S + 1] - 0.5 * 0.0;
                    }
                }
            }
        }
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const double *qq = side == 0 ? L : Rt;
            double *P = side == 0 ? PL : PR;
            double z2 = qq[2] * qq[2] + qq[3] * qq[3] + qq[4] * qq[4];
            fac[side] = 1.0 / sqrt(1.0 + z2);
            P[P_VX] = qq[2] * fac[side];
            P[P_VY] = qq[3] * fac[side];
            P[P_VZ] = qq[4] * fac[side];
            P[P_RHO] = clamp_lo(qq[0], 1e-12);
            P[P_P] = clamp_lo(qq[1], 1e-14);
            P[P_EPS] = eos_eps(P[P_P], P[P_RHO], g.gamma);
            P[IBN] = bn;
            P[IBT] = qq[5];
            P[P_BZ] = qq[6];
            zq[side][0] = qq[2];
            zq[side][1] = qq[3];
            zq[side][2] = qq[4];
            floor_rho[side] = qq[0] < 1e-12;
            floor_p[side] = qq[1] < 1e-14;
        }
    }
    double given[2] = {0.0, 0.0};
    if (SOLVER == HLLD_SOLVER_HLLD) {
        given[0] = p.pstar_in[e];
        given[1] = p.fail_in[e] ? 1.0 : 0.0;
    }
    // the Riemann solver in reverse (face_vjp.cuh): flux adjoint -> the nine
    // primitives of each face state, then eps = eps(p, rho) and the shared
    // normal field
    double lam[kAdjDirs];
    {
        double lF[NCONS] = {0, 0, 0, 0, 0, 0, 0, 0};
        lF[C_D] = p.lamF[F_D][e];
        lF[C_SX] = p.lamF[F_SX][e];
        lF[C_SY] = p.lamF[F_SY][e];
        lF[C_SZ] = p.lamF[F_SZ][e];
        lF[C_TAU] = p.lamF[F_TAU][e];
        lF[C_BZ] = p.lamF[F_BZ][e];
        lF[AXIS == 0 ? C_BY : C_BX] = p.lamF[F_BT][e];
        double aL[NPRIM] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, aR[NPRIM] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (SOLVER == HLLD_SOLVER_HLLD)
            vjp::hlld_face_vjp<AXIS>(PL, PR, g.gamma, given[0], given[1] != 0.0, lF, aL, aR);
        else
            vjp::hlle_face_vjp<AXIS>(PL, PR, g.gamma, lF, aL, aR);
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const double *P = side == 0 ? PL : PR;
            const double *A = side == 0 ? aL : aR;
            double *l = lam + side * 7;
            // eps = p / (rho (gamma - 1))
            l[0] = A[P_RHO] - A[P_EPS] * P[P_EPS] / P[P_RHO];
            l[1] = A[P_P] + A[P_EPS] / (P[P_RHO] * (g.gamma - 1.0));
            l[2] = A[P_VX];
            l[3] = A[P_VY];
            l[4] = A[P_VZ];
            l[5] = A[IBT];
            l[6] = A[P_BZ];
        }
        lam[14] = aL[IBN] + aR[IBN];
    }
    p.lamBn[e] = lam[14];
    // reverse of the conversion W v -> v and the floors, per side
    double lq[2][7];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const double *l = lam + side * 7;
        lq[side][0] = floor_rho[side] ? 0.0 : l[0];
        lq[side][1] = floor_p[side] ? 0.0 : l[1];
        const double fc = fac[side], fc3 = fc * fc * fc;
        const double zl = zq[side][0] * l[2] + zq[side][1] * l[3] + zq[side][2] * l[4];
#pragma unroll
        for (int j = 0; j < 3; ++j) lq[side][2 + j] = fc * l[2 + j] - fc3 * zq[side][j] * zl;
        lq[side][5] = l[5];
        lq[side][6] = l[6];
    }
    // the window again (the store above may alias it for all the compiler
    // knows, so these are fresh loads, not values held since the start)
    double q[7][NW], vel[3][NW], Wf[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        double qk[7], vk[3];
        load_slot(k, qk, vk, Wf[k]);
#pragma unroll
        for (int v = 0; v < 7; ++v) q[v][k] = qk[v];
#pragma unroll
        for (int j = 0; j < 3; ++j) vel[j][k] = vk[j];
    }
    // reverse of the reconstruction onto the window slots
    double ls[7][NW];
#pragma unroll
    for (int v = 0; v < 7; ++v)
#pragma unroll
        for (int k = 0; k < NW; ++k) ls[v][k] = 0.0;
    if (edge) {
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            if (f == 0) ls[v][S + 1] = lq[0][v] + lq[1][v];
            else ls[v][S] = lq[0][v] + lq[1][v];
        }
    } else if (bad) {
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            ls[v][S] = lq[0][v];
            ls[v][S + 1] = lq[1][v];
        }
    } else {
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            Dual<NW> w[NW];
#pragma unroll
            for (int k = 0; k < NW; ++k) w[k] = Dual<NW>::var(q[v][k], k);
            Dual<NW> dl = cell_edge<LIM, true, S>(w, f - 1, n);
            Dual<NW> dr = cell_edge<LIM, false, S + 1>(w, f, n);
#pragma unroll
            for (int k = 0; k < NW; ++k) ls[v][k] = lq[0][v] * dl.d[k] + lq[1][v] * dr.d[k];
        }
    }
    // work variables -> primitives of each window cell: q = W v with
    // W = 1 / sqrt(max(1 - v^2, 1e-14))
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        const double W = Wf[k];
        double v2 = vel[0][k] * vel[0][k] + vel[1][k] * vel[1][k] + vel[2][k] * vel[2][k];
        const bool clamped = (1.0 - v2) < 1e-14;
        const double vq = vel[0][k] * ls[2][k] + vel[1][k] * ls[3][k] + vel[2][k] * ls[4][k];
        const double g3 = clamped ? 0.0 : W * W * W * vq;
        double out[7];
        out[0] = ls[0][k];
        out[1] = ls[1][k];
#pragma unroll
        for (int j = 0; j < 3; ++j) out[2 + j] = W * ls[2 + j][k] + g3 * vel[j][k];
        out[5] = ls[5][k];
        out[6] = ls[6][k];
#pragma unroll
        for (int v = 0; v < 7; ++v) p.lamS[k * 7 + v][e] = out[v];
    }
}

struct AdjGatherParams {
    Grid g;
    const double *lamS[kMaxNW * 7];
    const double *lamBn;
    double *lP[6];      // lambda of rho, p, vx, vy, vz, Bz (cells, accumulated)
    double *lBc;        // lambda of the cell-centred transverse B (cells, accumulated)
    double *lBn;        // lambda of the normal face field (faces, accumulated)
};

// Sum each cell's window-slot lambdas over the faces whose stencil holds it
// (face f holds cell f - 1 - S + k in slot k).
template <int AXIS, int S>
__global__ void __launch_bounds__(kThreads) adj_sweep_gather_kernel(const AdjGatherParams p) {
    constexpr int NW = 2 * S + 2;
    const Grid &g = p.g;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ncell = (int64_t)g.nxt * g.nyt;
    const int64_t nface = AXIS == 0 ? (int64_t)(g.nxt + 1) * g.nyt : (int64_t)g.nxt * (g.nyt + 1);
    // Every load is issued before the first store: the arrays may alias for
    // all the compiler knows, so a load after a store would wait for it, and
    // a chain of read-modify-writes would cost one memory latency each.
    double bn_old = 0.0, bn_add = 0.0;
    if (e < nface) {
        bn_old = p.lBn[e];
        bn_add = p.lamBn[e];
    }
    if (e < ncell) {
        const int i = (int)(e / g.nyt), j = (int)(e - (int64_t)i * g.nyt);
        const int c = AXIS == 0 ? i : j;
        const int tr = AXIS == 0 ? j : i;
        const int n = AXIS == 0 ? g.nxt : g.nyt;
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            const int f = c + 1 + S - k;
            if (f < 0 || f > n) continue;
            const int64_t fe = AXIS == 0 ? (int64_t)f * g.nyt + tr : (int64_t)tr * (g.nyt + 1) + f;
#pragma unroll
            for (int v = 0; v < 7; ++v) acc[v] += p.lamS[k * 7 + v][fe];
        }
        double old[7];
#pragma unroll
        for (int v = 0; v < 6; ++v) old[v] = p.lP[v][e];
        old[6] = p.lBc[e];
        p.lP[0][e] = old[0] + acc[0];
        p.lP[1][e] = old[1] + acc[1];
        p.lP[2][e] = old[2] + acc[2];
        p.lP[3][e] = old[3] + acc[3];
        p.lP[4][e] = old[4] + acc[4];
        p.lP[5][e] = old[5] + acc[6];
        p.lBc[e] = old[6] + acc[5];
    }
    if (e < nface) p.lBn[e] = bn_old + bn_add;
}

// ── C2P of the physical cells (c2p_cells_kernel) in reverse ──────────────

struct AdjC2PParams {
    Grid g;
    const double *U[6];
    const double *Bxf, *Byf;
    double *lP[9];     // lambda of the primitives (read, then zeroed)
    double *lU[6];     // accumulated
    double *lBcx, *lBcy;  // accumulated
    const double *mu_in;  // the forward's C2P roots, or NULL (solved here)
};

__global__ void __launch_bounds__(kThreads) adj_c2p_kernel(const AdjC2PParams p) {
    const Grid &g = p.g;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)g.nx * g.ny) return;
    const int i = g.ng + (int)(e / g.ny), j = g.ng + (int)(e % g.ny);
    const int nyt = g.nyt;
    const int64_t c = (int64_t)i * nyt + j;
    // Loads before stores throughout (the arrays may alias for all the
    // compiler knows, so a load after a store waits for it): the primitive
    // lambdas, and -- for a cell with work -- the state, the root and the
    // accumulators, then the zeroing and the sums.
    double lp[NPRIM];
    bool any = false;
#pragma unroll
    for (int k = 0; k < NPRIM; ++k) {
        lp[k] = p.lP[k][c];
        any = any || (lp[k] != 0.0);
    }
    if (!any) return;  // nothing to pull back, nothing to zero
    double Bcx = 0.5 * (p.Bxf[c] + p.Bxf[(int64_t)(i + 1) * nyt + j]);
    double Bcy = 0.5 * (p.Byf[(int64_t)i * (nyt + 1) + j] + p.Byf[(int64_t)i * (nyt + 1) + j + 1]);
    double C[NCONS] = {p.U[0][c], p.U[1][c], p.U[2][c], p.U[3][c], p.U[4][c], Bcx, Bcy, p.U[5][c]};
    double mu = p.mu_in ? p.mu_in[c] : 0.0;
    double acc[8];
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = p.lU[k][c];
    acc[6] = p.lBcx[c];
    acc[7] = p.lBcy[c];
#pragma unroll
    for (int k = 0; k < NPRIM; ++k) p.lP[k][c] = 0.0;
    if (!p.mu_in) {
        double P[NPRIM];
        cons_to_prim<double>(C, g.gamma, g.atmo_rho, 1e-10, P, &mu);
    }
    double lc[NCONS];
    vjp::c2p_vjp(C, g.gamma, g.atmo_rho, mu, lp, lc);
    p.lU[0][c] = acc[0] + lc[C_D];
    p.lU[1][c] = acc[1] + lc[C_SX];
    p.lU[2][c] = acc[2] + lc[C_SY];
    p.lU[3][c] = acc[3] + lc[C_SZ];
    p.lU[4][c] = acc[4] + lc[C_TAU];
    p.lU[5][c] = acc[5] + lc[C_BZ];
    p.lBcx[c] = acc[6] + lc[C_BX];
    p.lBcy[c] = acc[7] + lc[C_BY];
}

// cell-centred B = face averages (ct.py:44-54) in reverse: faces gather
// half of each adjacent cell's lambda
struct AdjBcParams {
    Grid g;
    double *lBcx, *lBcy;
    double *lBxf, *lByf;
};

__global__ void __launch_bounds__(kThreads) adj_bc_faces_kernel(const AdjBcParams p) {
    const Grid &g = p.g;
    const int nxt = g.nxt, nyt = g.nyt;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nfx = (int64_t)(nxt + 1) * nyt, nfy = (int64_t)nxt * (nyt + 1);
    // (loads before stores, as in the gathers above)
    double sx = 0.0, sy = 0.0, ox = 0.0, oy = 0.0;
    if (e < nfx) {
        const int i = (int)(e / nyt), j = (int)(e - (int64_t)i * nyt);
        if (i >= 1) sx += p.lBcx[(int64_t)(i - 1) * nyt + j];
        if (i < nxt) sx += p.lBcx[(int64_t)i * nyt + j];
        ox = p.lBxf[e];
    }
    if (e < nfy) {
        const int i = (int)(e / (nyt + 1)), j = (int)(e - (int64_t)i * (nyt + 1));
        if (j >= 1) sy += p.lBcy[(int64_t)i * nyt + j - 1];
        if (j < nyt) sy += p.lBcy[(int64_t)i * nyt + j];
        oy = p.lByf[e];
    }
    if (e < nfx) p.lBxf[e] = ox + 0.5 * sx;
    if (e < nfy) p.lByf[e] = oy + 0.5 * sy;
}

// ── ghost fills in reverse ───────────────────────────────────────────────

// Every entry of the never-written block adds the lambdas of the ghost
// entries filled from it (a gather, so the sum order is fixed).  The ghost
// indices of each axis are [0, a) and [b, n): at most 2 ng + 1 of them.
// Only the band within ng + 1 of the block's edges can be a source; the
// threads enumerate that band (the block minus its inner hole).
__host__ __device__ __forceinline__ int fold_band(const int ng) { return ng + 1; }
__host__ __device__ __forceinline__ int fold_hole(int in, int band) {
    return in > 2 * band ? in - 2 * band : 0;
}

template <typename E>
__global__ void __launch_bounds__(kThreads) adj_fold_kernel(const GhostParams<E> p) {
    E *v = p.v[blockIdx.y];
    const int in0 = p.b0 - p.a0, in1 = p.b1 - p.a1;
    const int B = fold_band(p.ng);
    int h0 = fold_hole(in0, B), h1 = fold_hole(in1, B);
    if (h0 == 0 || h1 == 0) h0 = h1 = 0;
    const int64_t nA = (int64_t)(in0 - h0) * in1;
    const int64_t nB = (int64_t)h0 * (in1 - h1);
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nA + nB) return;
    int rr, cc;
    if (e < nA) {
        const int q = (int)(e / in1);
        cc = (int)(e - (int64_t)q * in1);
        rr = (h0 > 0 && q >= B) ? q + h0 : q;
    } else {
        const int64_t e2 = e - nA;
        const int w = in1 - h1;
        const int q = (int)(e2 / w), k = (int)(e2 - (int64_t)q * w);
        rr = B + q;
        cc = k < B ? k : k + h1;
    }
    const int r = p.a0 + rr, c = p.a1 + cc;
    int rs[8], cs[8], nr = 1, nc = 1;
    rs[0] = r;
    cs[0] = c;
    for (int gi = 0; gi < p.n0; ++gi) {
        if (gi == p.a0) gi = p.b0;
        if (gi >= p.n0 || nr >= 8) break;
        int s = p.face0 ? bc_face_src(gi, p.n_ph0, p.ng, p.kind0) : bc_cc_src(gi, p.n_ph0, p.ng, p.kind0);
        if (s == r) rs[nr++] = gi;
    }
    for (int gi = 0; gi < p.n1; ++gi) {
        if (gi == p.a1) gi = p.b1;
        if (gi >= p.n1 || nc >= 8) break;
        int s = p.face1 ? bc_face_src(gi, p.n_ph1, p.ng, p.kind1) : bc_cc_src(gi, p.n_ph1, p.ng, p.kind1);
        if (s == c) cs[nc++] = gi;
    }
    if (nr == 1 && nc == 1) return;
    E acc = E(0);
    for (int a = 0; a < nr; ++a)
        for (int b = 0; b < nc; ++b)
            if (a || b) acc += v[(int64_t)rs[a] * p.n1 + cs[b]];
    v[(int64_t)r * p.n1 + c] += acc;
}

template <typename E>
__global__ void __launch_bounds__(kThreads) adj_zero_ghost_kernel(const GhostParams<E> p) {
    E *v = p.v[blockIdx.y];
    const int in0 = p.b0 - p.a0, in1 = p.b1 - p.a1;
    const int64_t nA = (int64_t)(p.n0 - in0) * p.n1;
    const int64_t nB = (int64_t)in0 * (p.n1 - in1);
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nA + nB) return;
    int r, c;
    if (e < nA) {
        int rr = (int)(e / p.n1);
        c = (int)(e - (int64_t)rr * p.n1);
        r = rr < p.a0 ? rr : rr + in0;
    } else {
        int64_t e2 = e - nA;
        int w = p.n1 - in1;
        int rr = (int)(e2 / w);
        int cc = (int)(e2 - (int64_t)rr * w);
        r = p.a0 + rr;
        c = cc < p.a1 ? cc : cc + in1;
    }
    v[(int64_t)r * p.n1 + c] = E(0);
}

// ── RK combine, flux divergence and CT curl in reverse ───────────────────

struct AdjUpdateParams {
    Grid g;
    double *lU[6];             // lambda of the stage output (physical cells); scaled by b
    double *lBxf, *lByf;       // lambda of the stage output faces; scaled by b
    double *lU0[6], *lBx0, *lBy0;  // accumulated a * lambda
    double *lFx[NFLUX], *lFy[NFLUX];  // written: slots D .. Bz
    double *lEz;               // written
    double a, b, w2;
};

// lambda of the fluxes (faces) and corner EMFs from the stage output lambda
// (ct_update_kernel in reverse); runs before adj_update_scale_kernel
__global__ void __launch_bounds__(kThreads) adj_divergence_kernel(const AdjUpdateParams p) {
    const Grid &g = p.g;
    const int nxt = g.nxt, nyt = g.nyt;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nfx = (int64_t)(nxt + 1) * nyt, nfy = (int64_t)nxt * (nyt + 1),
                  ncr = (int64_t)(nxt + 1) * (nyt + 1);
    auto cell_upd = [&](int i, int j) {
        return i >= g.ng && i < g.ng + g.nx && j >= g.ng && j < g.ng + g.ny;
    };
    // (every load before the first store, as in the gathers above)
    double sx[6] = {0, 0, 0, 0, 0, 0}, sy[6] = {0, 0, 0, 0, 0, 0}, sz = 0.0;
    if (e < nfx) {
        const int f = (int)(e / nyt), j = (int)(e - (int64_t)f * nyt);
        const bool hi = cell_upd(f, j), lo = cell_upd(f - 1, j);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (hi) sx[k] += p.lU[k][(int64_t)f * nyt + j];
            if (lo) sx[k] -= p.lU[k][(int64_t)(f - 1) * nyt + j];
        }
    }
    if (e < nfy) {
        const int i = (int)(e / (nyt + 1)), f = (int)(e - (int64_t)i * (nyt + 1));
        const bool hi = cell_upd(i, f), lo = cell_upd(i, f - 1);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (hi) sy[k] += p.lU[k][(int64_t)i * nyt + f];
            if (lo) sy[k] -= p.lU[k][(int64_t)i * nyt + f - 1];
        }
    }
    if (e < ncr) {
        const int i = (int)(e / (nyt + 1)), j = (int)(e - (int64_t)i * (nyt + 1));
        // updated faces: Bxf(i, j) for i in [ng, ng+nx], j in [ng, ng+ny);
        // Byf(i, j) for i in [ng, ng+nx), j in [ng, ng+ny]
        auto bx_upd = [&](int fi, int fj) {
            return fi >= g.ng && fi <= g.ng + g.nx && fj >= g.ng && fj < g.ng + g.ny;
        };
        auto by_upd = [&](int fi, int fj) {
            return fi >= g.ng && fi < g.ng + g.nx && fj >= g.ng && fj <= g.ng + g.ny;
        };
        // Bxf(i, j) += w2 (Ez(i, j) - Ez(i, j+1)) / dy
        if (j < nyt && bx_upd(i, j)) sz += p.lBxf[(int64_t)i * nyt + j] / g.dy;
        if (j >= 1 && bx_upd(i, j - 1)) sz -= p.lBxf[(int64_t)i * nyt + j - 1] / g.dy;
        // Byf(i, j) += w2 (Ez(i+1, j) - Ez(i, j)) / dx
        if (i < nxt && by_upd(i, j)) sz -= p.lByf[(int64_t)i * (nyt + 1) + j] / g.dx;
        if (i >= 1 && by_upd(i - 1, j)) sz += p.lByf[(int64_t)(i - 1) * (nyt + 1) + j] / g.dx;
    }
    if (e < nfx) {
#pragma unroll
        for (int k = 0; k < 6; ++k) p.lFx[k][e] = p.w2 * sx[k] / g.dx;
    }
    if (e < nfy) {
#pragma unroll
        for (int k = 0; k < 6; ++k) p.lFy[k][e] = p.w2 * sy[k] / g.dy;
    }
    if (e < ncr) p.lEz[e] = p.w2 * sz;
}

// lambda(U0) += a lambda, lambda(U_s) = b lambda on the updated entries
__global__ void __launch_bounds__(kThreads) adj_update_scale_kernel(const AdjUpdateParams p) {
    const Grid &g = p.g;
    const int nyt = g.nyt;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)(g.nx + 1) * (g.ny + 1)) return;
    const int ii = (int)(e / (g.ny + 1)), jj = (int)(e - (int64_t)ii * (g.ny + 1));
    const int i = g.ng + ii, j = g.ng + jj;
    // (every load before the first store, as in the gathers above)
    const bool cell = ii < g.nx && jj < g.ny, fxl = jj < g.ny, fyl = ii < g.nx;
    const int64_t c = (int64_t)i * nyt + j, fx = c, fy = (int64_t)i * (nyt + 1) + j;
    double l[6], l0[6], bx = 0.0, bx0 = 0.0, by = 0.0, by0 = 0.0;
    if (cell) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            l[k] = p.lU[k][c];
            l0[k] = p.lU0[k][c];
        }
    }
    if (fxl) {
        bx = p.lBxf[fx];
        bx0 = p.lBx0[fx];
    }
    if (fyl) {
        by = p.lByf[fy];
        by0 = p.lBy0[fy];
    }
    if (cell) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            p.lU0[k][c] = l0[k] + p.a * l[k];
            p.lU[k][c] = p.b * l[k];
        }
    }
    if (fxl) {
        p.lBx0[fx] = bx0 + p.a * bx;
        p.lBxf[fx] = p.b * bx;
    }
    if (fyl) {
        p.lBy0[fy] = by0 + p.a * by;
        p.lByf[fy] = p.b * by;
    }
}

// ── corner EMF in reverse ────────────────────────────────────────────────

struct AdjEmfParams {
    Grid g;
    const double *vx, *vy, *Bxf, *Byf;
    const double *FxD, *FyD;
    const hlld_step_diag_t *diag;  // the stage's sweep counters (max |F_D|: deadband scale)
    int upwind;
    const double *lEz;
    double *lFxBt, *lFyBt;  // written
    double *lvx, *lvy, *lBcx, *lBcy;  // accumulated
};

struct EmfCoef {
    double yf, yfm, xf, xfm, NE, NW, SE, SW;
};

// d Ez(i, j) / d (its eight inputs), upwind signs frozen (ct_emf_kernel)
__device__ __forceinline__ EmfCoef emf_coef(const AdjEmfParams &p, int i, int j) {
    EmfCoef c;
    if (!p.upwind) {
        c.yf = c.yfm = c.xf = c.xfm = 0.25;
        c.NE = c.NW = c.SE = c.SW = 0.0;
        return c;
    }
    const int nyt = p.g.nyt;
    const double sx = __longlong_as_double((long long)p.diag->sweep[0].fd_max_bits);
    const double sy = __longlong_as_double((long long)p.diag->sweep[1].fd_max_bits);
    const double Sx = upwind_sign(p.FxD[(int64_t)i * nyt + j], sx);
    const double Sxm = upwind_sign(p.FxD[(int64_t)i * nyt + j - 1], sx);
    const double Sy = upwind_sign(p.FyD[(int64_t)i * (nyt + 1) + j], sy);
    const double Sym = upwind_sign(p.FyD[(int64_t)(i - 1) * (nyt + 1) + j], sy);
    c.yf = 0.25 + 0.125 * ((1.0 - Sx) + (1.0 - Sxm));
    c.yfm = 0.25 + 0.125 * ((1.0 + Sx) + (1.0 + Sxm));
    c.xf = 0.25 + 0.125 * ((1.0 - Sy) + (1.0 - Sym));
    c.xfm = 0.25 + 0.125 * ((1.0 + Sy) + (1.0 + Sym));
    c.NE = -0.125 * ((1.0 - Sx) + (1.0 - Sy));
    c.NW = -0.125 * ((1.0 + Sx) + (1.0 - Sym));
    c.SE = -0.125 * ((1.0 - Sxm) + (1.0 + Sy));
    c.SW = -0.125 * ((1.0 + Sxm) + (1.0 + Sym));
    return c;
}

__device__ __forceinline__ bool emf_live(const Grid &g, int i, int j) {
    return i >= 1 && i <= g.nxt - 1 && j >= 1 && j <= g.nyt - 1;
}

__global__ void __launch_bounds__(kThreads) adj_emf_kernel(const AdjEmfParams p) {
    const Grid &g = p.g;
    const int nxt = g.nxt, nyt = g.nyt;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nfx = (int64_t)(nxt + 1) * nyt, nfy = (int64_t)nxt * (nyt + 1),
                  nc = (int64_t)nxt * nyt;
    auto lez = [&](int i, int j) { return p.lEz[(int64_t)i * (nyt + 1) + j]; };
    // (every load before the first store, as in the gathers above)
    // x faces: Ezxf = -FxBt(i, j) at corner (i, j), Ezxfm at corner (i, j + 1)
    double sx = 0.0, sy = 0.0;
    if (e < nfx) {
        const int i = (int)(e / nyt), j = (int)(e - (int64_t)i * nyt);
        if (emf_live(g, i, j)) sx += lez(i, j) * emf_coef(p, i, j).xf;
        if (emf_live(g, i, j + 1)) sx += lez(i, j + 1) * emf_coef(p, i, j + 1).xfm;
    }
    // y faces: Ezyf = FyBt(i, j) at corner (i, j), Ezyfm at corner (i + 1, j)
    if (e < nfy) {
        const int i = (int)(e / (nyt + 1)), j = (int)(e - (int64_t)i * (nyt + 1));
        if (emf_live(g, i, j)) sy += lez(i, j) * emf_coef(p, i, j).yf;
        if (emf_live(g, i + 1, j)) sy += lez(i + 1, j) * emf_coef(p, i + 1, j).yfm;
    }
    // cells: E(i, j) is NE of corner (i, j), NW of (i+1, j), SE of (i, j+1),
    // SW of (i+1, j+1); E = Bcx vy - Bcy vx (cell_emf)
    double lE = 0.0, Bcx = 0.0, Bcy = 0.0, vx = 0.0, vy = 0.0;
    double o_vy = 0.0, o_vx = 0.0, o_bx = 0.0, o_by = 0.0;
    if (e < nc && p.upwind) {
        const int i = (int)(e / nyt), j = (int)(e - (int64_t)i * nyt);
        if (emf_live(g, i, j)) lE += lez(i, j) * emf_coef(p, i, j).NE;
        if (emf_live(g, i + 1, j)) lE += lez(i + 1, j) * emf_coef(p, i + 1, j).NW;
        if (emf_live(g, i, j + 1)) lE += lez(i, j + 1) * emf_coef(p, i, j + 1).SE;
        if (emf_live(g, i + 1, j + 1)) lE += lez(i + 1, j + 1) * emf_coef(p, i + 1, j + 1).SW;
        if (lE != 0.0) {
            Bcx = 0.5 * (p.Bxf[(int64_t)i * nyt + j] + p.Bxf[(int64_t)(i + 1) * nyt + j]);
            Bcy = 0.5 * (p.Byf[(int64_t)i * (nyt + 1) + j] + p.Byf[(int64_t)i * (nyt + 1) + j + 1]);
            vx = p.vx[e];
            vy = p.vy[e];
            o_vy = p.lvy[e];
            o_vx = p.lvx[e];
            o_bx = p.lBcx[e];
            o_by = p.lBcy[e];
        }
    }
    if (e < nfx) p.lFxBt[e] = -sx;
    if (e < nfy) p.lFyBt[e] = sy;
    if (lE != 0.0) {
        p.lvy[e] = o_vy + Bcx * lE;
        p.lvx[e] = o_vx - Bcy * lE;
        p.lBcx[e] = o_bx + vy * lE;
        p.lBcy[e] = o_by - vx * lE;
    }
}

struct AdjAddParams {
    double *dst[6];
    const double *src[6];
    int64_t n;
};

__global__ void __launch_bounds__(kThreads) add_arrays_kernel(const AdjAddParams p) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < p.n) p.dst[blockIdx.y][e] += p.src[blockIdx.y][e];
}

// primitive_to_conserved (hlld.py:185-217) in reverse, per element:
// lam_prim = (d cons / d prim)^T lam_cons (all nine primitives, eps
// included as the independent input it is there)
struct P2CVjpParams {
    int64_t n;
    const double *prim[NPRIM];
    const double *lc[NCONS];  // may hold NULL entries (zero lambda)
    double *lp[NPRIM];
};

__global__ void __launch_bounds__(kThreads) p2c_vjp_kernel(const P2CVjpParams p) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= p.n) return;
    using D9 = Dual<NPRIM>;
    D9 P[NPRIM], C[NCONS];
#pragma unroll
    for (int k = 0; k < NPRIM; ++k) P[k] = D9::var(p.prim[k][e], k);
    prim_to_cons<D9>(P, C);
    double lc[NCONS];
#pragma unroll
    for (int k = 0; k < NCONS; ++k) lc[k] = p.lc[k] ? p.lc[k][e] : 0.0;
#pragma unroll
    for (int j = 0; j < NPRIM; ++j) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NCONS; ++k) s += lc[k] * C[k].d[j];
        p.lp[j][e] = s;
    }
}

// ── host side ────────────────────────────────────────────────────────────

static inline unsigned grid1d(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

static Grid make_grid(const hlld_grid2d_t *g) {
    Grid G;
    G.nx = g->nx;
    G.ny = g->ny;
    G.ng = g->ng;
    G.nxt = g->nx + 2 * g->ng;
    G.nyt = g->ny + 2 * g->ng;
    G.dx = g->dx;
    G.dy = g->dy;
    G.gamma = g->gamma;
    G.atmo_rho = g->atmo_rho;
    G.bc_x = g->bc_x;
    G.bc_y = g->bc_y;
    return G;
}

struct AdjState {   // one saved stage state
    double *U[6], *Bxf, *Byf, *P[9];
};

// What the forward step records for its reverse: the inputs of stages 1
// and 2, and per stage the F_D of both sweeps (CT upwind signs), the sweep
// counters (their max |F_D| sets the deadband) and each face's p* and
// HLLE fallback.
struct AdjTape {
    AdjState X[2];
    double *FxD[3], *FyD[3];
    double *psx[3], *psy[3];
    uint8_t *fx[3], *fy[3];
    double *mu[3];           // C2P roots of each stage's sync (the inputs of the next stage)
    hlld_step_diag_t *diag;  // [3]
};

// Work arrays of the reverse (and of the recording forward step).
struct AdjScratch {
    Scratch2D fw;
    double *lU0[6], *lBx0, *lBy0, *lBcx, *lBcy;
    double *lFx[NFLUX], *lFy[NFLUX], *lEz;
    double *lamS[kMaxNW * 7], *lamBn;
};

static size_t adj_align(size_t b) { return (b + 255) & ~(size_t)255; }

struct Carver {
    char *base;
    size_t off = 0;
    double *d(size_t n) {
        double *p = base ? (double *)(base + off) : nullptr;
        off += adj_align(n * 8);
        return p;
    }
    uint8_t *b(size_t n) {
        uint8_t *p = base ? (uint8_t *)(base + off) : nullptr;
        off += adj_align(n);
        return p;
    }
};

static size_t tape_layout(const hlld_grid2d_t *g, char *base, AdjTape *t) {
    const size_t nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    const size_t nfx = (nxt + 1) * nyt, nfy = nxt * (nyt + 1), nc = nxt * nyt;
    Carver c{base};
    AdjTape s{};
    for (int x = 0; x < 2; ++x) {
        for (int k = 0; k < 6; ++k) s.X[x].U[k] = c.d(nc);
        s.X[x].Bxf = c.d(nfx);
        s.X[x].Byf = c.d(nfy);
        for (int k = 0; k < 9; ++k) s.X[x].P[k] = c.d(nc);
    }
    for (int st = 0; st < 3; ++st) {
        s.FxD[st] = c.d(nfx);
        s.FyD[st] = c.d(nfy);
        s.psx[st] = c.d(nfx);
        s.psy[st] = c.d(nfy);
        s.fx[st] = c.b(nfx);
        s.fy[st] = c.b(nfy);
        s.mu[st] = c.d(nc);
    }
    s.diag = base ? (hlld_step_diag_t *)(base + c.off) : nullptr;
    c.off += adj_align(3 * sizeof(hlld_step_diag_t));
    if (t) *t = s;
    return c.off;
}

static size_t scratch_layout(const hlld_grid2d_t *g, char *base, AdjScratch *sc) {
    const size_t nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    const size_t nfx = (nxt + 1) * nyt, nfy = nxt * (nyt + 1), ncr = (nxt + 1) * (nyt + 1),
                 nc = nxt * nyt, nfmax = nfx > nfy ? nfx : nfy;
    const int nw = 2 * (g->limiter == HLLD_LIM_MP7 ? 3
                        : (g->limiter == HLLD_LIM_WENO5Z || g->limiter == HLLD_LIM_MP5) ? 2 : 1) + 2;
    Carver c{base};
    AdjScratch s{};
    for (int k = 0; k < 7; ++k) s.fw.Fx[k] = c.d(nfx);
    for (int k = 0; k < 7; ++k) s.fw.Fy[k] = c.d(nfy);
    s.fw.Ez = c.d(ncr);
    for (int k = 0; k < 6; ++k) s.fw.U0[k] = c.d(nc);
    s.fw.Bx0 = c.d(nfx);
    s.fw.By0 = c.d(nfy);
    s.fw.diag = nullptr;
    for (int k = 0; k < 6; ++k) s.lU0[k] = c.d(nc);
    s.lBx0 = c.d(nfx);
    s.lBy0 = c.d(nfy);
    s.lBcx = c.d(nc);
    s.lBcy = c.d(nc);
    for (int k = 0; k < NFLUX; ++k) s.lFx[k] = c.d(nfx);
    for (int k = 0; k < NFLUX; ++k) s.lFy[k] = c.d(nfy);
    s.lEz = c.d(ncr);
    // window-slot lambdas: only the limiter's window width is stored
    for (int k = 0; k < kMaxNW * 7; ++k) s.lamS[k] = (k < nw * 7) ? c.d(nfmax) : nullptr;
    s.lamBn = c.d(nfmax);
    if (sc) *sc = s;
    return c.off;
}

size_t adjoint_tape_bytes(const hlld_grid2d_t *g) { return tape_layout(g, nullptr, nullptr); }
size_t adjoint_reverse_scratch_bytes(const hlld_grid2d_t *g) { return scratch_layout(g, nullptr, nullptr); }

void launch_prim_to_cons_vjp(int64_t n, const void *const *prim, const void *const *lam_cons,
                             void *const *lam_prim, cudaStream_t st) {
    P2CVjpParams pp = {};
    pp.n = n;
    for (int k = 0; k < NPRIM; ++k) {
        pp.prim[k] = (const double *)prim[k];
        pp.lp[k] = (double *)lam_prim[k];
    }
    for (int k = 0; k < NCONS; ++k) pp.lc[k] = (const double *)lam_cons[k];
    p2c_vjp_kernel<<<grid1d(n), kThreads, 0, st>>>(pp);
}


static GhostParams<double> ghost_params_cc(const Grid &G, double *const *arrs, int narr) {
    GhostParams<double> gp = {};
    for (int k = 0; k < narr; ++k) gp.v[k] = arrs[k];
    gp.n0 = G.nxt;
    gp.n1 = G.nyt;
    gp.a0 = G.ng;
    gp.b0 = G.ng + G.nx;
    gp.a1 = G.ng;
    gp.b1 = G.ng + G.ny;
    gp.n_ph0 = G.nx;
    gp.n_ph1 = G.ny;
    gp.ng = G.ng;
    gp.kind0 = G.bc_x;
    gp.kind1 = G.bc_y;
    return gp;
}

static void adj_fold(const GhostParams<double> &gp, int narr, cudaStream_t st) {
    const int in0 = gp.b0 - gp.a0, in1 = gp.b1 - gp.a1;
    const int64_t in = (int64_t)in0 * in1;
    const int64_t out = (int64_t)gp.n0 * gp.n1 - in;
    const int B = fold_band(gp.ng);
    int h0 = fold_hole(in0, B), h1 = fold_hole(in1, B);
    if (h0 == 0 || h1 == 0) h0 = h1 = 0;
    const int64_t band = in - (int64_t)h0 * h1;
    adj_fold_kernel<double><<<dim3(grid1d(band), narr), kThreads, 0, st>>>(gp);
    adj_zero_ghost_kernel<double><<<dim3(grid1d(out), narr), kThreads, 0, st>>>(gp);
}

// reverse of launch_sync_state (face ghosts, cell ghosts, C2P, primitive
// ghosts) at state X: lambda(P) -> lambda(U, faces); also moves the pending
// cell-centred-B lambdas onto the faces
static void adj_sync(const Grid &G, const AdjState &X, double *const *lU, double *lBxf, double *lByf,
                     double *const *lP, const AdjScratch &sc, cudaStream_t st,
                     const double *mu = nullptr) {
    // a. primitive ghosts
    adj_fold(ghost_params_cc(G, lP, 9), 9, st);
    // b. C2P of the physical cells
    AdjC2PParams cp = {};
    cp.g = G;
    for (int k = 0; k < 6; ++k) cp.U[k] = X.U[k];
    cp.Bxf = X.Bxf;
    cp.Byf = X.Byf;
    for (int k = 0; k < 9; ++k) cp.lP[k] = lP[k];
    for (int k = 0; k < 6; ++k) cp.lU[k] = lU[k];
    cp.lBcx = sc.lBcx;
    cp.lBcy = sc.lBcy;
    cp.mu_in = mu;
    adj_c2p_kernel<<<grid1d((int64_t)G.nx * G.ny), kThreads, 0, st>>>(cp);
    // c. cell-centred B -> faces
    AdjBcParams bp = {G, sc.lBcx, sc.lBcy, lBxf, lByf};
    const int64_t nfmax = (int64_t)(G.nxt + 1) * (G.nyt + 1);
    adj_bc_faces_kernel<<<grid1d(nfmax), kThreads, 0, st>>>(bp);
    cudaMemsetAsync(sc.lBcx, 0, sizeof(double) * G.nxt * G.nyt, st);
    cudaMemsetAsync(sc.lBcy, 0, sizeof(double) * G.nxt * G.nyt, st);
    // d. conserved and face ghosts (launch_sync_state / launch_ghost_faces)
    adj_fold(ghost_params_cc(G, lU, 6), 6, st);
    GhostParams<double> fx = ghost_params_cc(G, &lBxf, 1);
    fx.n0 = G.nxt + 1;
    fx.b0 = G.ng + G.nx + (G.bc_x == HLLD_BC_OUTFLOW ? 1 : 0);
    fx.face0 = 1;
    adj_fold(fx, 1, st);
    GhostParams<double> fy = ghost_params_cc(G, &lByf, 1);
    fy.n1 = G.nyt + 1;
    fy.b1 = G.ng + G.ny + (G.bc_y == HLLD_BC_OUTFLOW ? 1 : 0);
    fy.face1 = 1;
    adj_fold(fy, 1, st);
}

template <int AXIS, int LIM>
static void launch_adj_sweep_lim(int solver, const AdjSweepParams &ap, cudaStream_t st) {
    const int64_t nf = AXIS == 0 ? (int64_t)(ap.g.nxt + 1) * ap.g.nyt : (int64_t)ap.g.nxt * (ap.g.nyt + 1);
    if (solver == HLLD_SOLVER_HLLD)
        adj_sweep_kernel<AXIS, LIM, HLLD_SOLVER_HLLD><<<grid1d(nf), kThreads, 0, st>>>(ap);
    else
        adj_sweep_kernel<AXIS, LIM, HLLD_SOLVER_HLLE><<<grid1d(nf), kThreads, 0, st>>>(ap);
}

template <int AXIS>
static void launch_adj_sweep(int limiter, int solver, const AdjSweepParams &ap,
                             const AdjGatherParams &gp, cudaStream_t st) {
    int S = 1;
    switch (limiter) {
    case HLLD_LIM_PCM: launch_adj_sweep_lim<AXIS, HLLD_LIM_PCM>(solver, ap, st); break;
    case HLLD_LIM_MC: launch_adj_sweep_lim<AXIS, HLLD_LIM_MC>(solver, ap, st); break;
    case HLLD_LIM_MINMOD: launch_adj_sweep_lim<AXIS, HLLD_LIM_MINMOD>(solver, ap, st); break;
    case HLLD_LIM_WENO5Z: launch_adj_sweep_lim<AXIS, HLLD_LIM_WENO5Z>(solver, ap, st); S = 2; break;
    case HLLD_LIM_MP5: launch_adj_sweep_lim<AXIS, HLLD_LIM_MP5>(solver, ap, st); S = 2; break;
    default: launch_adj_sweep_lim<AXIS, HLLD_LIM_MP7>(solver, ap, st); S = 3; break;
    }
    const int64_t nc = (int64_t)gp.g.nxt * gp.g.nyt;
    const int64_t nf = AXIS == 0 ? (int64_t)(gp.g.nxt + 1) * gp.g.nyt : (int64_t)gp.g.nxt * (gp.g.nyt + 1);
    const int64_t nthr = nc > nf ? nc : nf;
    if (S == 1) adj_sweep_gather_kernel<AXIS, 1><<<grid1d(nthr), kThreads, 0, st>>>(gp);
    else if (S == 2) adj_sweep_gather_kernel<AXIS, 2><<<grid1d(nthr), kThreads, 0, st>>>(gp);
    else adj_sweep_gather_kernel<AXIS, 3><<<grid1d(nthr), kThreads, 0, st>>>(gp);
}

static hlld_state2d_t as_state(const AdjState &X) {
    hlld_state2d_t s{};
    for (int k = 0; k < 6; ++k) s.cons[k] = X.U[k];
    s.Bxf = X.Bxf;
    s.Byf = X.Byf;
    for (int k = 0; k < 9; ++k) s.prims[k] = X.P[k];
    return s;
}

static AdjState from_state(const hlld_state2d_t *s) {
    AdjState X;
    for (int k = 0; k < 6; ++k) X.U[k] = (double *)s->cons[k];
    X.Bxf = (double *)s->Bxf;
    X.Byf = (double *)s->Byf;
    for (int k = 0; k < 9; ++k) X.P[k] = (double *)s->prims[k];
    return X;
}

static void copy_state(const Grid &G, const AdjState &src, const AdjState &dst, cudaStream_t st) {
    const size_t nc = sizeof(double) * G.nxt * G.nyt;
    for (int k = 0; k < 6; ++k) cudaMemcpyAsync(dst.U[k], src.U[k], nc, cudaMemcpyDeviceToDevice, st);
    for (int k = 0; k < 9; ++k) cudaMemcpyAsync(dst.P[k], src.P[k], nc, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(dst.Bxf, src.Bxf, sizeof(double) * (G.nxt + 1) * G.nyt, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(dst.Byf, src.Byf, sizeof(double) * G.nxt * (G.nyt + 1), cudaMemcpyDeviceToDevice, st);
}

// One forward step (the same kernels and order as launch_rk_step_ct) that
// advances s in place and records the tape.
void launch_adjoint_record(const hlld_grid2d_t *g, const hlld_state2d_t *s, double dt, int scheme,
                           void *tape, void *scratch, cudaStream_t st) {
    Grid G = make_grid(g);
    AdjTape tp;
    tape_layout(g, (char *)tape, &tp);
    AdjScratch sc;
    scratch_layout(g, (char *)scratch, &sc);
    const int nst = scheme == 3 ? 3 : 2;
    const size_t nfx = (size_t)(G.nxt + 1) * G.nyt, nfy = (size_t)G.nxt * (G.nyt + 1);
    cudaMemsetAsync(tp.diag, 0, 3 * sizeof(hlld_step_diag_t), st);
    const AdjState S = from_state(s);
    for (int stage = 0; stage < nst; ++stage) {
        hlld_step_diag_t *dg = tp.diag + stage;
        ::hlld::v_fp64::launch_sweep2d(g, s, 0, sc.fw.Fx, &dg->sweep[0], st, tp.psx[stage], tp.fx[stage]);
        ::hlld::v_fp64::launch_sweep2d(g, s, 1, sc.fw.Fy, &dg->sweep[1], st, tp.psy[stage], tp.fy[stage]);
        cudaMemcpyAsync(tp.FxD[stage], sc.fw.Fx[F_D], sizeof(double) * nfx, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(tp.FyD[stage], sc.fw.Fy[F_D], sizeof(double) * nfy, cudaMemcpyDeviceToDevice, st);
        ::hlld::v_fp64::launch_ct_update2d(g, s, sc.fw, dg, stage, scheme, dt, nullptr, st);
        ::hlld::v_fp64::launch_sync_state(g, s, nullptr, dg, st, tp.mu[stage]);
        if (stage + 1 < nst) copy_state(G, S, tp.X[stage], st);
    }
}

// The reverse of one recorded step: s_in / s_out are the step's input and
// output; lam: on entry lambda of the output (cons, faces, prims), on return
// lambda of the input (prims lambda zero).
void launch_adjoint_reverse(const hlld_grid2d_t *g, const hlld_state2d_t *s_in,
                            const hlld_state2d_t *s_out, double dt, int scheme, const void *tape,
                            const hlld_state2d_t *lam, void *scratch, cudaStream_t st) {
    Grid G = make_grid(g);
    AdjTape tp;
    tape_layout(g, (char *)tape, &tp);
    AdjScratch sc;
    scratch_layout(g, (char *)scratch, &sc);
    const int nst = scheme == 3 ? 3 : 2;
    const size_t nc = (size_t)G.nxt * G.nyt, nfx = (size_t)(G.nxt + 1) * G.nyt,
                 nfy = (size_t)G.nxt * (G.nyt + 1);
    const AdjState X0 = from_state(s_in);
    const AdjState Xs[3] = {X0, tp.X[0], tp.X[1]};
    double *lU[6], *lP[9];
    for (int k = 0; k < 6; ++k) lU[k] = (double *)lam->cons[k];
    for (int k = 0; k < 9; ++k) lP[k] = (double *)lam->prims[k];
    double *lBxf = (double *)lam->Bxf, *lByf = (double *)lam->Byf;
    for (int k = 0; k < 6; ++k) cudaMemsetAsync(sc.lU0[k], 0, sizeof(double) * nc, st);
    cudaMemsetAsync(sc.lBx0, 0, sizeof(double) * nfx, st);
    cudaMemsetAsync(sc.lBy0, 0, sizeof(double) * nfy, st);
    cudaMemsetAsync(sc.lBcx, 0, sizeof(double) * nc, st);
    cudaMemsetAsync(sc.lBcy, 0, sizeof(double) * nc, st);
    // driver2d.py:104-105
    static const double kW3[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
    static const double kW2[2][3] = {{1.0, 0.0, 1.0}, {0.5, 0.5, 0.5}};
    const AdjState Xlast = from_state(s_out);
    const int64_t nmax = (int64_t)(G.nxt + 1) * (G.nyt + 1);
    for (int stage = nst - 1; stage >= 0; --stage) {
        const AdjState &Xin = Xs[stage];
        const AdjState &Xout = stage == nst - 1 ? Xlast : Xs[stage + 1];
        const double *w = scheme == 3 ? kW3[stage] : kW2[stage];
        // a-d: lambda(P_{s+1}) -> lambda(U_{s+1}, faces_{s+1})
        adj_sync(G, Xout, lU, lBxf, lByf, lP, sc, st, tp.mu[stage]);
        // e: RK combine, divergence and CT curl
        AdjUpdateParams up = {};
        up.g = G;
        for (int k = 0; k < 6; ++k) {
            up.lU[k] = lU[k];
            up.lU0[k] = sc.lU0[k];
        }
        up.lBxf = lBxf;
        up.lByf = lByf;
        up.lBx0 = sc.lBx0;
        up.lBy0 = sc.lBy0;
        for (int k = 0; k < NFLUX; ++k) {
            up.lFx[k] = sc.lFx[k];
            up.lFy[k] = sc.lFy[k];
        }
        up.lEz = sc.lEz;
        up.a = w[0];
        up.b = w[1];
        up.w2 = w[2] * dt;
        adj_divergence_kernel<<<grid1d(nmax), kThreads, 0, st>>>(up);
        adj_update_scale_kernel<<<grid1d((int64_t)(G.nx + 1) * (G.ny + 1)), kThreads, 0, st>>>(up);
        // f: corner EMF at X_s
        AdjEmfParams ep = {};
        ep.g = G;
        ep.vx = Xin.P[P_VX];
        ep.vy = Xin.P[P_VY];
        ep.Bxf = Xin.Bxf;
        ep.Byf = Xin.Byf;
        ep.FxD = tp.FxD[stage];
        ep.FyD = tp.FyD[stage];
        ep.diag = tp.diag + stage;
        ep.upwind = g->upwind;
        ep.lEz = sc.lEz;
        ep.lFxBt = sc.lFx[F_BT];
        ep.lFyBt = sc.lFy[F_BT];
        ep.lvx = lP[P_VX];
        ep.lvy = lP[P_VY];
        ep.lBcx = sc.lBcx;
        ep.lBcy = sc.lBcy;
        adj_emf_kernel<<<grid1d(nmax), kThreads, 0, st>>>(ep);
        // g: the two sweeps at X_s
        for (int axis = 0; axis < 2; ++axis) {
            AdjSweepParams ap = {};
            ap.g = G;
            ap.rho = Xin.P[P_RHO];
            ap.p = Xin.P[P_P];
            ap.vx = Xin.P[P_VX];
            ap.vy = Xin.P[P_VY];
            ap.vz = Xin.P[P_VZ];
            ap.bz = Xin.P[P_BZ];
            ap.Bxf = Xin.Bxf;
            ap.Byf = Xin.Byf;
            for (int k = 0; k < NFLUX; ++k) ap.lamF[k] = axis == 0 ? sc.lFx[k] : sc.lFy[k];
            ap.pstar_in = axis == 0 ? tp.psx[stage] : tp.psy[stage];
            ap.fail_in = axis == 0 ? tp.fx[stage] : tp.fy[stage];
            for (int k = 0; k < kMaxNW * 7; ++k) ap.lamS[k] = sc.lamS[k];
            ap.lamBn = sc.lamBn;
            AdjGatherParams gp = {};
            gp.g = G;
            for (int k = 0; k < kMaxNW * 7; ++k) gp.lamS[k] = sc.lamS[k];
            gp.lamBn = sc.lamBn;
            gp.lP[0] = lP[P_RHO];
            gp.lP[1] = lP[P_P];
            gp.lP[2] = lP[P_VX];
            gp.lP[3] = lP[P_VY];
            gp.lP[4] = lP[P_VZ];
            gp.lP[5] = lP[P_BZ];
            gp.lBc = axis == 0 ? sc.lBcy : sc.lBcx;
            gp.lBn = axis == 0 ? lBxf : lByf;
            if (axis == 0) launch_adj_sweep<0>(g->limiter, g->solver, ap, gp, st);
            else launch_adj_sweep<1>(g->limiter, g->solver, ap, gp, st);
        }
    }
    // lambda(X_0) = the b-terms already in lam + the a-terms, then the
    // primitives of X_0 (the previous step's sync) in reverse
    AdjAddParams ad = {};
    for (int k = 0; k < 6; ++k) {
        ad.dst[k] = lU[k];
        ad.src[k] = sc.lU0[k];
    }
    ad.n = (int64_t)nc;
    add_arrays_kernel<<<dim3(grid1d(ad.n), 6), kThreads, 0, st>>>(ad);
    AdjAddParams af = {};
    af.dst[0] = lBxf;
    af.src[0] = sc.lBx0;
    af.n = (int64_t)nfx;
    add_arrays_kernel<<<dim3(grid1d(af.n), 1), kThreads, 0, st>>>(af);
    af.dst[0] = lByf;
    af.src[0] = sc.lBy0;
    af.n = (int64_t)nfy;
    add_arrays_kernel<<<dim3(grid1d(af.n), 1), kThreads, 0, st>>>(af);
    adj_sync(G, X0, lU, lBxf, lByf, lP, sc, st);
}

// Self-contained form: the scratch holds the reverse's work arrays, a tape
// and a working copy of s_in, which the recording step advances.
static size_t state_layout(const hlld_grid2d_t *g, char *base, AdjState *X) {
    const size_t nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    Carver c{base};
    AdjState s{};
    for (int k = 0; k < 6; ++k) s.U[k] = c.d(nxt * nyt);
    s.Bxf = c.d((nxt + 1) * nyt);
    s.Byf = c.d(nxt * (nyt + 1));
    for (int k = 0; k < 9; ++k) s.P[k] = c.d(nxt * nyt);
    if (X) *X = s;
    return c.off;
}

size_t adjoint_scratch_bytes(const hlld_grid2d_t *g) {
    return scratch_layout(g, nullptr, nullptr) + tape_layout(g, nullptr, nullptr) +
           state_layout(g, nullptr, nullptr);
}

void launch_adjoint_rk_step_ct(const hlld_grid2d_t *g, const hlld_state2d_t *s_in,
                               const hlld_state2d_t *s_out, double dt, int scheme,
                               const hlld_state2d_t *lam, void *scratch, cudaStream_t st) {
    Grid G = make_grid(g);
    char *tape = (char *)scratch + scratch_layout(g, nullptr, nullptr);
    char *work = tape + tape_layout(g, nullptr, nullptr);
    AdjState W;
    state_layout(g, work, &W);
    copy_state(G, from_state(s_in), W, st);
    hlld_state2d_t ws = as_state(W);
    launch_adjoint_record(g, &ws, dt, scheme, tape, scratch, st);
    launch_adjoint_reverse(g, s_in, s_out, dt, scheme, tape, lam, scratch, st);
}

}  // namespace HLLD_NS
}  // namespace hlld
