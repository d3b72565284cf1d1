// Kernels of the SRMHD step, compiled once per arithmetic variant: this
// header is included by a translation unit that defines HLLD_NS (the
// variant's namespace) and is built with or without FMA contraction.
//
// Kernels:
//   riemann_faces_kernel  flux_fn plugin on flattened faces (hlld.py:1005, :1202)
//   c2p_kernel            conservative_to_primitive (c2p.py:313-363)
//   p2c_kernel            primitive_to_conserved (hlld.py:185-217)
//   sweep_kernel          one directional sweep of the 2D step, fused:
//                         reconstruction + normal-B override + Riemann
//                         solver + max|F_D| (sweep.py:30-119, reconstruction.py:272-338)
//   ct_emf_kernel         Gardiner-Stone corner EMF (ct.py:44-177)
//   ct_update_kernel      flux divergence + CT face update + RK combine
//                         (sweep.py:122-135, ct.py:180-185, state.py:77-103)
//   ghost_kernel          separable ghost fill (grid.py:93-143, :229-255)
//   c2p_cells_kernel      cell-centred B + C2P of physical cells (driver2d.py:196-218)
//   speed_kernel/dt_kernel compute_dt_2d (driver2d.py:52-82)
#pragma once

#ifndef HLLD_NS
#error "define HLLD_NS before including kernels_impl.cuh"
#endif

#include "srmhd_phys.cuh"
#include "variants.h"

// Real type of the 2D step's primitives, reconstruction, face fluxes, corner
// EMF and flux divergence (double, or float for the mixed and FP32 forms), and
// of the HLL-state C2P that seeds the HLLD p* bracket.
#ifndef HLLD_REAL
#define HLLD_REAL double
#endif
#ifndef HLLD_BRACKET_REAL
#define HLLD_BRACKET_REAL HLLD_REAL
#endif
// Real type of the conserved state, the staggered field, the RK stage-0 copy,
// the RK accumulation, the cell C2P and the HLLD p* iteration: double, or
// float in the all-FP32 form.
#ifndef HLLD_STATE_REAL
#define HLLD_STATE_REAL double
#endif

namespace hlld {
namespace HLLD_NS {

using R = HLLD_REAL;
using RB = HLLD_BRACKET_REAL;
using RS = HLLD_STATE_REAL;
constexpr int kThreads = 128;
// HLLD_SWEEP_PARK = 1: the sweep's faces keep the values that only the HLLD
// star states read again in shared memory during the p* solve (hlld_face's
// PARK_STRIDE); float faces only (the FP64 slot would not fit the 48 KB of
// static shared memory beside the tile)
#ifndef HLLD_SWEEP_PARK
#define HLLD_SWEEP_PARK 1
#endif
constexpr int kSweepPark = (HLLD_SWEEP_PARK && sizeof(R) == sizeof(float)) ? kThreads : 0;
// minimum resident blocks per SM requested for the sweep kernel (caps its
// registers at 65536 / (kThreads * this)); 0 picks per form: 5 with the
// parked face state (96 registers), else 4 (128).  Measured on B200 (rotor
// 2048^2, mixed step): 4 unparked 5.70 ms, 4 parked 5.45 ms, 5 parked
// 5.34 ms; FP64 step: 4 13.26 ms, 5 14.43 ms.
#ifndef HLLD_SWEEP_MIN_BLOCKS
#define HLLD_SWEEP_MIN_BLOCKS 0
#endif
constexpr int kSweepMinBlocks =
    HLLD_SWEEP_MIN_BLOCKS > 0 ? HLLD_SWEEP_MIN_BLOCKS : (kSweepPark > 0 ? 5 : 4);
// minimum resident blocks per SM requested for the cell C2P kernel: 8 (64
// registers, a few spills) against the compiler's 96 registers at 5 blocks
// measured on B200 (rotor 2048^2): mixed step 5.35 -> 5.22 ms, FP64 step
// 13.30 -> 13.04 ms (6 blocks: 5.28 and 13.15 ms)
#ifndef HLLD_C2P_MIN_BLOCKS
#define HLLD_C2P_MIN_BLOCKS 8
#endif
constexpr int kC2PMinBlocks = HLLD_C2P_MIN_BLOCKS;
// The 2D sweeps and the tube kernel solve no p* on faces without normal
// field (their HLLE fallback output does not depend on it), except in the
// exact form, which keeps the reference's solver counters.
constexpr bool kSkipBnZero = !HLLD_EXACT_ARITH;

// ── small utilities ──────────────────────────────────────────────────────

// non-negative doubles order like their bit patterns; a NaN (sign cleared)
// sorts above +inf, so atomicMax on the bits propagates it like torch's max
__device__ __forceinline__ unsigned long long abs_bits(double x) {
    return (unsigned long long)__double_as_longlong(fabs(x));
}

struct Counts {
    unsigned long long v[9];  // slots [0, NS) are summed, [NS, NS + NM) maxed
};

// Block-reduce NS sum slots and NM max slots; thread 0 adds the sums to
// dst[0..NS) and max-combines the maxima into dmax[0..NM).  Every thread of
// the block must call it.
template <int NS, int NM>
__device__ __forceinline__ void block_accumulate(Counts c, unsigned long long *dst,
                                                 unsigned long long *const *dmax) {
    __shared__ unsigned long long sm[kThreads / 32][NS + NM];
#pragma unroll
    for (int k = 0; k < NS + NM; ++k) {
        unsigned long long x = c.v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long y = __shfl_down_sync(0xffffffffu, x, o);
            x = (k >= NS) ? (x > y ? x : y) : x + y;
        }
        c.v[k] = x;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NS + NM; ++k) sm[w][k] = c.v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s[NS + NM];
#pragma unroll
        for (int k = 0; k < NS + NM; ++k) s[k] = sm[0][k];
        for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww)
#pragma unroll
            for (int k = 0; k < NS + NM; ++k)
                s[k] = (k >= NS) ? (s[k] > sm[ww][k] ? s[k] : sm[ww][k]) : s[k] + sm[ww][k];
#pragma unroll
        for (int k = 0; k < NS; ++k)
            if (s[k]) atomicAdd(dst + k, s[k]);
#pragma unroll
        for (int k = 0; k < NM; ++k)
            if (s[NS + k]) atomicMax(dmax[k], s[NS + k]);
    }
}

__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long x) {
    __shared__ unsigned long long sm[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long y = __shfl_down_sync(0xffffffffu, x, o);
        x = x > y ? x : y;
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = x;
    __syncthreads();
    unsigned long long r = 0;
    if (threadIdx.x == 0) {
        r = sm[0];
        for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww) r = r > sm[ww] ? r : sm[ww];
    }
    return r;
}

// ── reconstruction (reconstruction.py) ───────────────────────────────────

template <typename T> __device__ __forceinline__ T minmod(T a, T b) {
    return (a * b > T(0)) ? ((fabs(a) < fabs(b)) ? a : b) : T(0);
}
template <typename T> __device__ __forceinline__ T mc_lim(T a, T b) {
    T c = T(0.5) * (a + b);
    return (a * b > T(0)) ? tsign(c) * tmin(T(2) * fabs(a), tmin(T(2) * fabs(b), fabs(c))) : T(0);
}
// reconstruction.py:111-128
template <typename T> __device__ __forceinline__ T weno5z(T vm2, T vm1, T v0, T vp1, T vp2) {
    T p0 = (T(2) * vm2 - T(7) * vm1 + T(11) * v0) / T(6);
    T p1 = (-vm1 + T(5) * v0 + T(2) * vp1) / T(6);
    T p2 = (T(2) * v0 + T(5) * vp1 - vp2) / T(6);
    const T c1 = T(13.0 / 12.0), c2 = T(0.25);
    T t = vm2 - T(2) * vm1 + v0, u = vm2 - T(4) * vm1 + T(3) * v0;
    T b0 = c1 * (t * t) + c2 * (u * u);
    t = vm1 - T(2) * v0 + vp1;
    u = vm1 - vp1;
    T b1 = c1 * (t * t) + c2 * (u * u);
    t = v0 - T(2) * vp1 + vp2;
    u = T(3) * v0 - T(4) * vp1 + vp2;
    T b2 = c1 * (t * t) + c2 * (u * u);
    T tau5 = fabs(b0 - b2);
    const T eps = K<T>::weno_eps;
    T r0 = tau5 / (b0 + eps), r1 = tau5 / (b1 + eps), r2 = tau5 / (b2 + eps);
    if constexpr (sizeof(T) == 4) {
        // FP32: r^2 overflows once r > 1.8e19 (a smooth stencil next to a
        // jump has beta = 0); the weights are normalised, so divide every
        // 1 + r^2 by the largest (1 + r^2) scale first
        T s = tmax(T(1), tmax(r0, tmax(r1, r2)));
        T is = T(1) / s, i2 = is * is;
        T q0 = r0 * is, q1 = r1 * is, q2 = r2 * is;
        T a0 = T(0.1) * (i2 + q0 * q0);
        T a1 = T(0.6) * (i2 + q1 * q1);
        T a2 = T(0.3) * (i2 + q2 * q2);
        return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
    }
    T a0 = T(0.1) * (T(1) + r0 * r0);
    T a1 = T(0.6) * (T(1) + r1 * r1);
    T a2 = T(0.3) * (T(1) + r2 * r2);
    return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}
// reconstruction.py:136-162
template <typename T>
__device__ __forceinline__ T mp_limit(T vl, T vm2, T vm1, T v0, T vp1, T vp2) {
    const T alpha = T(4);
    T vmp = v0 + minmod(vp1 - v0, alpha * (v0 - vm1));
    bool need = (vl - v0) * (vl - vmp) > K<T>::mp_eps;
    if (!need) return vl;
    T d_m1 = vm2 - T(2) * vm1 + v0;
    T d_0 = vm1 - T(2) * v0 + vp1;
    T d_p1 = v0 - T(2) * vp1 + vp2;
    T dm4_p = minmod(minmod(T(4) * d_0 - d_p1, T(4) * d_p1 - d_0), minmod(d_0, d_p1));
    T dm4_m = minmod(minmod(T(4) * d_m1 - d_0, T(4) * d_0 - d_m1), minmod(d_m1, d_0));
    T v_ul = v0 + alpha * (v0 - vm1);
    T v_av = T(0.5) * (v0 + vp1);
    T v_md = v_av - T(0.5) * dm4_p;
    T v_lc = v0 + T(0.5) * (v0 - vm1) + T(4.0 / 3.0) * dm4_m;
    T vmin = tmax(tmin(tmin(v0, vp1), v_md), tmin(tmin(v0, v_ul), v_lc));
    T vmax = tmin(tmax(tmax(v0, vp1), v_md), tmax(tmax(v0, v_ul), v_lc));
    return vl + minmod(vmin - vl, vmax - vl);
}
template <typename T> __device__ __forceinline__ T mp5(T vm2, T vm1, T v0, T vp1, T vp2) {
    T vl = (T(2) * vm2 - T(13) * vm1 + T(47) * v0 + T(27) * vp1 - T(3) * vp2) / T(60);
    return mp_limit(vl, vm2, vm1, v0, vp1, vp2);
}
template <typename T>
__device__ __forceinline__ T mp7(T vm3, T vm2, T vm1, T v0, T vp1, T vp2, T vp3) {
    T vl = (T(-3) * vm3 + T(25) * vm2 - T(101) * vm1 + T(319) * v0 + T(214) * vp1 - T(38) * vp2 +
            T(4) * vp3) /
           T(420);
    return mp_limit(vl, vm2, vm1, v0, vp1, vp2);
}

template <int LIM> struct Stencil { static constexpr int S = 1; };
template <> struct Stencil<HLLD_LIM_PCM> { static constexpr int S = 1; };
template <> struct Stencil<HLLD_LIM_WENO5Z> { static constexpr int S = 2; };
template <> struct Stencil<HLLD_LIM_MP5> { static constexpr int S = 2; };
template <> struct Stencil<HLLD_LIM_MP7> { static constexpr int S = 3; };

// Edge value of cell c (window index M, i.e. cell c = base + M) toward
// the right (RIGHT = true: value at c+1/2) or the left (c-1/2), for one line
// of n cells; reconstruction.py:182-264.
template <int LIM, bool RIGHT, int M, typename T>
__device__ __forceinline__ T cell_edge(const T *w, int c, int n) {
    if (LIM == HLLD_LIM_PCM) return RIGHT ? w[M] + T(0.5) * T(0) : w[M] - T(0.5) * T(0);
    constexpr int HW = (LIM == HLLD_LIM_WENO5Z || LIM == HLLD_LIM_MP5) ? 2 : (LIM == HLLD_LIM_MP7 ? 3 : 0);
    if (HW > 0 && n > 2 * HW && c >= HW && c < n - HW) {
        if (LIM == HLLD_LIM_WENO5Z) {
            return RIGHT ? weno5z(w[M - 2], w[M - 1], w[M], w[M + 1], w[M + 2])
                         : weno5z(w[M + 2], w[M + 1], w[M], w[M - 1], w[M - 2]);
        } else if (LIM == HLLD_LIM_MP5) {
            return RIGHT ? mp5(w[M - 2], w[M - 1], w[M], w[M + 1], w[M + 2])
                         : mp5(w[M + 2], w[M + 1], w[M], w[M - 1], w[M - 2]);
        } else {
            if constexpr (HW == 3)
                return RIGHT ? mp7(w[M - 3], w[M - 2], w[M - 1], w[M], w[M + 1], w[M + 2], w[M + 3])
                             : mp7(w[M + 3], w[M + 2], w[M + 1], w[M], w[M - 1], w[M - 2], w[M - 3]);
        }
    }
    T slope = T(0);
    if (c >= 1 && c <= n - 2) {
        T a = w[M] - w[M - 1];
        T b = w[M + 1] - w[M];
        slope = (LIM == HLLD_LIM_MINMOD) ? minmod(a, b) : mc_lim(a, b);
    }
    return RIGHT ? w[M] + T(0.5) * slope : w[M] - T(0.5) * slope;
}

// ── per-element kernels (flattened plugin API) ───────────────────────────

struct FacesParams {
    int64_t n;
    const double *sL[9];
    const double *sR[9];
    double *F[8];
    double *U[8];
    double *pstar;
    int32_t *err;
    int32_t *iters;
    uint8_t *flags;
    hlld_flux_diag_t *diag;
    double gamma;
};

template <int IDIR, int SOLVER>
__global__ void __launch_bounds__(kThreads) riemann_faces_kernel(const FacesParams p) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    Counts c = {};
    bool live = e < p.n;
    if (live) {
        double PL[NPRIM], PR[NPRIM];
#pragma unroll
        for (int k = 0; k < NPRIM; ++k) {
            PL[k] = p.sL[k][e];
            PR[k] = p.sR[k][e];
        }
        FaceOut<double> o;
        bool want_u = p.U[0] != nullptr;
        if (SOLVER == HLLD_SOLVER_HLLD)
            hlld_face<IDIR, double>(PL, PR, p.gamma, want_u, o);
        else if (SOLVER == HLLD_SOLVER_HLLC)
            hllc_face<IDIR, double>(PL, PR, p.gamma, want_u, o);
        else
            hlle_face<IDIR, double>(PL, PR, p.gamma, want_u, true, o);
#pragma unroll
        for (int k = 0; k < NCONS; ++k) p.F[k][e] = o.F[k];
        if (want_u)
#pragma unroll
            for (int k = 0; k < NCONS; ++k) p.U[k][e] = o.U[k];
        p.pstar[e] = o.pstar;
        if (p.err) p.err[e] = o.err;
        if (p.iters) p.iters[e] = o.iters;
        if (p.flags) p.flags[e] = o.flags;
        c.v[0] = 1;
        c.v[1] = o.err > 0;
        c.v[2] = (o.flags & RF_WAVE_ORDER_BAD) != 0;
        c.v[3] = (o.flags & RF_BN_ZERO) != 0;
        c.v[4] = (o.flags & RF_FAILED) != 0;
        c.v[5] = (o.err == 0) ? (unsigned long long)o.iters : 0ull;
        c.v[6] = o.err == 0;
        c.v[7] = (unsigned long long)o.iters;
        c.v[8] = abs_bits(o.F[C_D]);
    }
    if (p.diag) {
        unsigned long long *mx[2] = {&p.diag->max_iters, &p.diag->fd_max_bits};
        block_accumulate<7, 2>(c, &p.diag->n_faces, mx);
    }
}

struct CellsParams {
    int64_t n;
    const double *in[9];
    double *out[9];
    uint8_t *status;
    double gamma, atmo_rho, atmo_eps;
};

__global__ void __launch_bounds__(kThreads) c2p_kernel(const CellsParams p) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= p.n) return;
    double C[NCONS], P[NPRIM];
#pragma unroll
    for (int k = 0; k < NCONS; ++k) C[k] = p.in[k][e];
    uint8_t st = cons_to_prim<double>(C, p.gamma, p.atmo_rho, p.atmo_eps, P);
#pragma unroll
    for (int k = 0; k < NPRIM; ++k) p.out[k][e] = P[k];
    if (p.status) p.status[e] = st;
}

__global__ void __launch_bounds__(kThreads) p2c_kernel(const CellsParams p) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= p.n) return;
    double P[NPRIM], C[NCONS];
#pragma unroll
    for (int k = 0; k < NPRIM; ++k) P[k] = p.in[k][e];
    prim_to_cons<double>(P, C);
#pragma unroll
    for (int k = 0; k < NCONS; ++k) p.out[k][e] = C[k];
}

// ── 2D step kernels ──────────────────────────────────────────────────────

struct Grid {
    int nx, ny, ng, nxt, nyt;
    double dx, dy, gamma, atmo_rho;
    int bc_x, bc_y;
    int emf_hll;  // face EMF from the HLL average (HLLD_EMF_HLL), else the solver's flux
};

// face flux slots of a sweep: the six evolved fluxes plus the transverse-B
// flux that becomes the face EMF (ct.py:63-88)
enum { F_D = 0, F_SX, F_SY, F_SZ, F_TAU, F_BZ, F_BT, NFLUX };

struct SweepParams {
    Grid g;
    const R *rho, *p, *vx, *vy, *vz, *bz;
    const RS *Bxf, *Byf;
    R *F[NFLUX];
    hlld_flux_diag_t *diag;
    // optional per-face record for the adjoint: p* and the HLLE fallback
    double *pstar_out;
    uint8_t *fail_out;
};

// A directional sweep, one face per thread, on tiles of faces staged in
// shared memory.  AXIS 0: faces (nxt+1, nyt), face f is the lower-x face of
// cell (f, j); AXIS 1: faces (nxt, nyt+1).
//
// A CTA of 128 threads owns a tile of 4 x 32 faces: 4 rows along x by 32
// along y, so a warp's 32 faces are consecutive in y and its loads and
// stores are coalesced.  First the CTA fills the tile's stencil -- for the x
// sweep (4 + 2S + 1) x 32 cells, for the y sweep 4 x (32 + 2S + 1) -- with
// the seven reconstructed variables of every cell (rho, p, W vx, W vy, W vz,
// the cell-centred transverse B, Bz; reconstruction.py:269 with vel_var Wv,
// ct.py:44-54), each computed once instead of once per face that reads it;
// then every thread reads its face's window from shared memory.  The
// arithmetic per cell and per face is the per-face gather's, so the results
// are the same bit for bit.
constexpr int kTileAlong = 4;   // face rows along x per tile
constexpr int kTileLanes = 32;  // face columns along y per tile

template <int AXIS, int S> struct SweepTile {
    static constexpr int ROWS = AXIS == 0 ? kTileAlong + 2 * S + 1 : kTileAlong;
    static constexpr int COLS = AXIS == 0 ? kTileLanes : kTileLanes + 2 * S + 1;
};

template <int AXIS, int LIM, int SOLVER, bool EMF_HLL>
__global__ void __launch_bounds__(kThreads, kSweepMinBlocks) sweep_kernel(const SweepParams p) {
    using T = R;
    constexpr int S = Stencil<LIM>::S;
    constexpr int NW = 2 * S + 2;
    constexpr int TR = SweepTile<AXIS, S>::ROWS, TC = SweepTile<AXIS, S>::COLS;
    __shared__ T tile[7][TR][TC];
    __shared__ T park[kSweepPark > 0 ? kParkWords : 1][kThreads];
    const Grid &g = p.g;
    const int cols = AXIS == 0 ? g.nyt : g.nyt + 1;
    const int rows = AXIS == 0 ? g.nxt + 1 : g.nxt;
    const int n = AXIS == 0 ? g.nxt : g.nyt;  // cells along the sweep axis
    const int tiles_y = (cols + kTileLanes - 1) / kTileLanes;
    const int row0 = (int)(blockIdx.x / tiles_y) * kTileAlong;  // first face row (x)
    const int col0 = (int)(blockIdx.x % tiles_y) * kTileLanes;  // first face column (y)
    // the window of the tile's first face starts at cell c0 along the sweep
    // axis; cells outside [0, n) are clamped (the edge rules never read them)
    const int c0 = (AXIS == 0 ? row0 : col0) - 1 - S;
    // transverse in-plane B at cell (i, j), averaged from its faces (ct.py:44-54)
    auto bt_at = [&](int i, int j) -> T {
        return AXIS == 0
                   ? T(RS(0.5) * (p.Byf[(int64_t)i * (g.nyt + 1) + j] + p.Byf[(int64_t)i * (g.nyt + 1) + j + 1]))
                   : T(RS(0.5) * (p.Bxf[(int64_t)i * g.nyt + j] + p.Bxf[(int64_t)(i + 1) * g.nyt + j]));
    };
    for (int q = threadIdx.x; q < TR * TC; q += blockDim.x) {
        const int r = q / TC, cc = q - r * TC;
        int i = AXIS == 0 ? c0 + r : row0 + r;
        int j = AXIS == 0 ? col0 + cc : c0 + cc;
        if (AXIS == 0) {
            i = i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
            if (j > g.nyt - 1) continue;
        } else {
            j = j < 0 ? 0 : (j > n - 1 ? n - 1 : j);
            if (i > g.nxt - 1) continue;
        }
        const int64_t ci = (int64_t)i * g.nyt + j;
        T vx = p.vx[ci], vy = p.vy[ci], vz = p.vz[ci];
        T v2 = vx * vx + vy * vy + vz * vz;
        T W = T(1) / sqrt(clamp_lo(T(1) - v2, T(1e-14)));
        tile[0][r][cc] = p.rho[ci];
        tile[1][r][cc] = p.p[ci];
        tile[2][r][cc] = W * vx;
        tile[3][r][cc] = W * vy;
        tile[4][r][cc] = W * vz;
        tile[5][r][cc] = bt_at(i, j);
        tile[6][r][cc] = p.bz[ci];
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int row = row0 + w, col = col0 + l;
    Counts cnt = {};
    const bool live = row < rows && col < cols;
    if (live) {
        const int f = AXIS == 0 ? row : col;   // face index along the sweep axis
        const int tr = AXIS == 0 ? col : row;  // transverse index
        // tile entry of window cell k (cell f - 1 - S + k) of this face
        auto at = [&](int v, int k) -> T { return AXIS == 0 ? tile[v][w + k][l] : tile[v][w][l + k]; };
        T L[7], Rt[7];
        if (f == 0 || f == n) {
            // outermost faces: the edge cell (0 or n - 1) has zero slope in
            // every scheme
            const int k = f == 0 ? S + 1 : S;
#pragma unroll
            for (int v = 0; v < 7; ++v) {
                const T q = at(v, k);
                L[v] = q + T(0.5) * T(0);
                Rt[v] = q - T(0.5) * T(0);
            }
        } else {
            T pcmL[7], pcmR[7];
#pragma unroll
            for (int v = 0; v < 7; ++v) {
                T wv[NW];
#pragma unroll
                for (int k = 0; k < NW; ++k) wv[k] = at(v, k);
                L[v] = cell_edge<LIM, true, S>(wv, f - 1, n);
                Rt[v] = cell_edge<LIM, false, S + 1>(wv, f, n);
                pcmL[v] = wv[S];
                pcmR[v] = wv[S + 1];
            }
            if (LIM != HLLD_LIM_PCM) {
                // positivity fallback to PCM (reconstruction.py:315-326)
                bool bad = (L[0] <= T(1e-12)) || (Rt[0] <= T(1e-12)) || (L[1] <= T(1e-14)) ||
                           (Rt[1] <= T(1e-14));
                if (bad) {
#pragma unroll
                    for (int v = 0; v < 7; ++v) {
                        L[v] = pcmL[v] + T(0.5) * T(0);
                        Rt[v] = pcmR[v] - T(0.5) * T(0);
                    }
                }
            }
        }
        // Wv -> v, floors, EOS-consistent eps (reconstruction.py:328-336); the
        // normal field is the face value (sweep.py:82-89)
        const T bn = T(AXIS == 0 ? p.Bxf[(int64_t)f * g.nyt + tr] : p.Byf[(int64_t)tr * (g.nyt + 1) + f]);
        T PL[NPRIM], PR[NPRIM];
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            T *q = side == 0 ? L : Rt;
            T *P = side == 0 ? PL : PR;
            T z2 = q[2] * q[2] + q[3] * q[3] + q[4] * q[4];
            T fac = T(1) / sqrt(T(1) + z2);
            P[P_VX] = q[2] * fac;
            P[P_VY] = q[3] * fac;
            P[P_VZ] = q[4] * fac;
            P[P_RHO] = clamp_lo(q[0], T(1e-12));
            P[P_P] = clamp_lo(q[1], T(1e-14));
            P[P_EPS] = eos_eps(P[P_P], P[P_RHO], (T)g.gamma);
            P[P_BX] = AXIS == 0 ? bn : q[5];
            P[P_BY] = AXIS == 0 ? q[5] : bn;
            P[P_BZ] = q[6];
        }
        FaceOut<T> o;
        if (SOLVER == HLLD_SOLVER_HLLD)
            hlld_face<AXIS, T, RB, RS, false, kSkipBnZero, true, kSweepPark>(
                PL, PR, (T)g.gamma, false, o, nullptr, p.pstar_out != nullptr,
                &park[0][threadIdx.x]);
        else if (SOLVER == HLLD_SOLVER_HLLC)
            hllc_face<AXIS, T>(PL, PR, (T)g.gamma, false, o);
        else
            hlle_face<AXIS, T>(PL, PR, (T)g.gamma, false, false, o);
        if (EMF_HLL) {
            // emf_mode "hll" (ct.py:63-96, sweep.py:106-119): the transverse-B
            // flux, which only feeds the face EMF, is the HLL average of the
            // face states' fluxes instead of the solver's
            Phys<T> ph;
            srmhd_fluxes<AXIS>(PL, PR, (T)g.gamma, ph);
            constexpr int KB = AXIS == 0 ? C_BY : C_BX;
            o.F[KB] = hf(ph.L.f[KB], ph.R.f[KB], ph.L.u[KB], ph.R.u[KB], ph.cmin, ph.cmax);
        }
        const int64_t fi = (int64_t)row * cols + col;
        p.F[F_D][fi] = o.F[C_D];
        p.F[F_SX][fi] = o.F[C_SX];
        p.F[F_SY][fi] = o.F[C_SY];
        p.F[F_SZ][fi] = o.F[C_SZ];
        p.F[F_TAU][fi] = o.F[C_TAU];
        p.F[F_BZ][fi] = o.F[C_BZ];
        p.F[F_BT][fi] = AXIS == 0 ? o.F[C_BY] : o.F[C_BX];
        if (p.pstar_out) {
            p.pstar_out[fi] = (double)o.pstar;
            p.fail_out[fi] = (o.flags & RF_FAILED) ? 1 : 0;
        }
        cnt.v[0] = 1;
        cnt.v[1] = o.err > 0;
        cnt.v[2] = (o.flags & RF_WAVE_ORDER_BAD) != 0;
        cnt.v[3] = (o.flags & RF_BN_ZERO) != 0;
        cnt.v[4] = (o.flags & RF_FAILED) != 0;
        cnt.v[5] = (o.err == 0) ? (unsigned long long)o.iters : 0ull;
        cnt.v[6] = o.err == 0;
        cnt.v[7] = (unsigned long long)o.iters;
        // max |F_D| over the sweep, for the CT deadband (ct.py:114)
        cnt.v[8] = abs_bits((double)o.F[C_D]);
    }
    unsigned long long *mx[2] = {&p.diag->max_iters, &p.diag->fd_max_bits};
    block_accumulate<7, 2>(cnt, &p.diag->n_faces, mx);
}

// ct.py:96-116 with the sweep-global scale
template <typename T> __device__ __forceinline__ T upwind_sign(T F, T scale) {
    return (fabs(F) > T(1e-9) * scale) ? tsign(F) : T(0);
}

struct CtParams {
    Grid g;
    const R *vx, *vy;
    const RS *Bxf, *Byf;
    const R *FxD, *FyD, *FxBt, *FyBt;
    const hlld_step_diag_t *diag;
    int upwind;
    R *Ez;
};

// cell-centred E^z = v^y B^x - v^x B^y from face-averaged B (ct.py:44-60)
__device__ __forceinline__ R cell_emf(const CtParams &p, int i, int j) {
    const int nyt = p.g.nyt;
    R Bcx = R(RS(0.5) * (p.Bxf[(int64_t)i * nyt + j] + p.Bxf[(int64_t)(i + 1) * nyt + j]));
    R Bcy = R(RS(0.5) * (p.Byf[(int64_t)i * (nyt + 1) + j] + p.Byf[(int64_t)i * (nyt + 1) + j + 1]));
    int64_t c = (int64_t)i * nyt + j;
    return Bcx * p.vy[c] - Bcy * p.vx[c];
}

__global__ void __launch_bounds__(kThreads) ct_emf_kernel(const CtParams p) {
    using T = R;
    const int nxt = p.g.nxt, nyt = p.g.nyt;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)(nxt + 1) * (nyt + 1)) return;
    const int i = (int)(e / (nyt + 1)), j = (int)(e - (int64_t)i * (nyt + 1));
    T val = T(0);
    if (i >= 1 && i <= nxt - 1 && j >= 1 && j <= nyt - 1) {
        // Efy (nxt, nyt+1) = +F^y(Bx); Efx (nxt+1, nyt) = -F^x(By)
        T Ezyf = p.FyBt[(int64_t)i * (nyt + 1) + j];
        T Ezyfm = p.FyBt[(int64_t)(i - 1) * (nyt + 1) + j];
        T Ezxf = -p.FxBt[(int64_t)i * nyt + j];
        T Ezxfm = -p.FxBt[(int64_t)i * nyt + j - 1];
        T EzNE = cell_emf(p, i, j);
        T EzNW = cell_emf(p, i - 1, j);
        T EzSE = cell_emf(p, i, j - 1);
        T EzSW = cell_emf(p, i - 1, j - 1);
        T Eavg = T(0.25) * ((Ezyf + Ezyfm) + (Ezxf + Ezxfm));
        if (p.upwind) {
            T sx = T(__longlong_as_double((long long)p.diag->sweep[0].fd_max_bits));
            T sy = T(__longlong_as_double((long long)p.diag->sweep[1].fd_max_bits));
            T Sx = upwind_sign(p.FxD[(int64_t)i * nyt + j], sx);
            T Sxm = upwind_sign(p.FxD[(int64_t)i * nyt + j - 1], sx);
            T dEdyN = (T(1) - Sx) * (EzNE - Ezyf) + (T(1) + Sx) * (EzNW - Ezyfm);
            T dEdyS = (T(1) - Sxm) * (Ezyf - EzSE) + (T(1) + Sxm) * (Ezyfm - EzSW);
            T dEdy = T(0.125) * (dEdyS - dEdyN);
            T Sy = upwind_sign(p.FyD[(int64_t)i * (nyt + 1) + j], sy);
            T Sym = upwind_sign(p.FyD[(int64_t)(i - 1) * (nyt + 1) + j], sy);
            T dEdxE = (T(1) - Sy) * (EzNE - Ezxf) + (T(1) + Sy) * (EzSE - Ezxfm);
            T dEdxW = (T(1) - Sym) * (Ezxf - EzNW) + (T(1) + Sym) * (Ezxfm - EzSW);
            T dEdx = T(0.125) * (dEdxW - dEdxE);
            val = Eavg + (dEdy + dEdx);
        } else {
            val = Eavg;
        }
    }
    p.Ez[e] = val;
}

struct UpdateParams {
    Grid g;
    RS *U[6];
    RS *U0[6];
    RS *Bxf, *Byf, *Bx0, *By0;
    const R *Fx[6];
    const R *Fy[6];
    const R *Ez;
    const double *dt_dev;
    double dt_host;
    double a, b, c;
    int first_stage;
};

// flux divergence (in R) + CT face update + RK combine (in RS) on the
// physical block and its upper faces; a thread owns cell (i, j), face
// Bxf(i, j) and face Byf(i, j)
__global__ void __launch_bounds__(kThreads) ct_update_kernel(const UpdateParams p) {
    const Grid &g = p.g;
    const int nyt = g.nyt;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)(g.nx + 1) * (g.ny + 1)) return;
    const int ii = (int)(e / (g.ny + 1)), jj = (int)(e - (int64_t)ii * (g.ny + 1));
    const int i = g.ng + ii, j = g.ng + jj;
    const double dt = p.dt_dev ? *p.dt_dev : p.dt_host;
    const RS w2 = RS(p.c * dt);
    const RS a = RS(p.a), b = RS(p.b);
    const R rdx = R(g.dx), rdy = R(g.dy);
    if (ii < g.nx && jj < g.ny) {
        const int64_t c = (int64_t)i * nyt + j;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            R rx = -(p.Fx[k][(int64_t)(i + 1) * nyt + j] - p.Fx[k][c]) / rdx;
            R ry = -(p.Fy[k][(int64_t)i * (nyt + 1) + j + 1] - p.Fy[k][(int64_t)i * (nyt + 1) + j]) / rdy;
            RS L = (RS)(rx + ry);
            RS u = p.U[k][c];
            RS u0;
            if (p.first_stage) {
                u0 = u;
                p.U0[k][c] = u;
            } else {
                u0 = p.U0[k][c];
            }
            RS v = a * u0;
            v = v + b * u;
            v = v + w2 * L;
            p.U[k][c] = v;
        }
    }
    if (jj < g.ny) {
        const int64_t fx = (int64_t)i * nyt + j;
        RS dB = ((RS)p.Ez[(int64_t)i * (nyt + 1) + j] - (RS)p.Ez[(int64_t)i * (nyt + 1) + j + 1]) / RS(g.dy);
        RS u = p.Bxf[fx];
        RS u0;
        if (p.first_stage) {
            u0 = u;
            p.Bx0[fx] = u;
        } else {
            u0 = p.Bx0[fx];
        }
        RS v = a * u0;
        v = v + b * u;
        v = v + w2 * dB;
        p.Bxf[fx] = v;
    }
    if (ii < g.nx) {
        const int64_t fy = (int64_t)i * (nyt + 1) + j;
        RS dB = ((RS)p.Ez[(int64_t)(i + 1) * (nyt + 1) + j] - (RS)p.Ez[(int64_t)i * (nyt + 1) + j]) / RS(g.dx);
        RS u = p.Byf[fy];
        RS u0;
        if (p.first_stage) {
            u0 = u;
            p.By0[fy] = u;
        } else {
            u0 = p.By0[fy];
        }
        RS v = a * u0;
        v = v + b * u;
        v = v + w2 * dB;
        p.Byf[fy] = v;
    }
}

// ── ghost fill (grid.py:93-143) ──────────────────────────────────────────

// source index of a cell-centred array along one axis (grid.py:93-113)
__device__ __forceinline__ int bc_cc_src(int idx, int n, int ng, int kind) {
    if (idx >= ng && idx < ng + n) return idx;
    if (kind == HLLD_BC_OUTFLOW) return idx < ng ? ng : ng + n - 1;
    return idx < ng ? idx + n : idx - n;
}
// source index of a face array along its normal axis (grid.py:116-143)
__device__ __forceinline__ int bc_face_src(int idx, int n, int ng, int kind) {
    if (kind == HLLD_BC_OUTFLOW) {
        if (idx < ng) return ng;
        if (idx > ng + n) return ng + n;
        return idx;
    }
    if (idx == ng + n) return ng;  // the periodic seam collapses onto face ng
    if (idx < ng) return idx + n;
    if (idx > ng + n) return idx - n;
    return idx;
}

template <typename E> struct GhostParams {
    E *v[9];       // blockIdx.y selects the array
    int n0, n1;    // array shape
    int a0, b0, a1, b1;  // block never written (its entries are every source)
    int n_ph0, n_ph1, ng;
    int kind0, kind1;
    int face0, face1;    // axis is the face-normal axis of this array
};

// Fills every entry outside [a0,b0) x [a1,b1) from its separable source;
// all sources lie inside that block, so the fill is race free in place.
template <typename E>
__global__ void __launch_bounds__(kThreads) ghost_kernel(const GhostParams<E> p) {
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
    int sr = p.face0 ? bc_face_src(r, p.n_ph0, p.ng, p.kind0) : bc_cc_src(r, p.n_ph0, p.ng, p.kind0);
    int sc = p.face1 ? bc_face_src(c, p.n_ph1, p.ng, p.kind1) : bc_cc_src(c, p.n_ph1, p.ng, p.kind1);
    v[(int64_t)r * p.n1 + c] = v[(int64_t)sr * p.n1 + sc];
}

struct C2PCellsParams {
    Grid g;
    const RS *U[6];
    const RS *Bxf, *Byf;
    R *P[9];
    uint8_t *status;
    hlld_step_diag_t *diag;
    double *mu_out;  // optional per-cell record of the C2P root (for the adjoint)
    double *mu_warm; // optional per-cell previous root, read as the start and updated
};

// Kastaun's root mu = 1 / (h W) of a cell's primitives (h = 1 + eps + p / rho),
// or 0 -- no start, the bracketed solve -- where they are not physical
template <typename T>
__device__ __forceinline__ T kastaun_mu_of_prims(const R *const *P, int64_t c) {
    const T rho = P[P_RHO][c], press = P[P_P][c], eps = P[P_EPS][c];
    const T vx = P[P_VX][c], vy = P[P_VY][c], vz = P[P_VZ][c];
    const T v2 = vx * vx + vy * vy + vz * vz;
    const T h = T(1) + eps + press / rho;
    return (v2 < T(1) && rho > T(0) && h > T(0)) ? sqrt(T(1) - v2) / h : T(0);
}

// cell-centred B (ct.py:44-54) + C2P (c2p.py:313-363) of the physical cells,
// in RS; primitives stored as R.  FROM_PRIMS: each root search starts
// from the root of the cell's current primitives, which the kernel then
// overwrites (a template flag: a runtime one made the other launches 5 %
// slower)
template <bool FROM_PRIMS>
__global__ void __launch_bounds__(kThreads, kC2PMinBlocks) c2p_cells_kernel(const C2PCellsParams p) {
    const Grid &g = p.g;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    Counts cnt = {};
    if (e < (int64_t)g.nx * g.ny) {
        const int i = g.ng + (int)(e / g.ny), j = g.ng + (int)(e % g.ny);
        const int nyt = g.nyt;
        const int64_t c = (int64_t)i * nyt + j;
        RS Bcx = RS(0.5) * (p.Bxf[c] + p.Bxf[(int64_t)(i + 1) * nyt + j]);
        RS Bcy = RS(0.5) * (p.Byf[(int64_t)i * (nyt + 1) + j] + p.Byf[(int64_t)i * (nyt + 1) + j + 1]);
        RS C[NCONS] = {p.U[0][c], p.U[1][c], p.U[2][c], p.U[3][c], p.U[4][c], Bcx, Bcy, p.U[5][c]};
        RS P[NPRIM];
        RS mu = RS(0);
        RS mu0 = RS(0);
        if constexpr (FROM_PRIMS) mu0 = kastaun_mu_of_prims<RS>(p.P, c);
        else if (p.mu_warm) mu0 = (RS)p.mu_warm[c];
        uint8_t st = cons_to_prim<RS>(C, RS(g.gamma), RS(g.atmo_rho), RS(1e-10), P,
                                      (p.mu_out || p.mu_warm) ? &mu : nullptr, mu0);
        if (p.mu_out) p.mu_out[c] = (double)mu;
        if (p.mu_warm) p.mu_warm[c] = (double)mu;
#pragma unroll
        for (int k = 0; k < NPRIM; ++k) p.P[k][c] = (R)P[k];
        if (p.status) p.status[c] = st;
        cnt.v[0] = !(st & ST_CONVERGED);
        cnt.v[1] = (st & ST_BISECTED) != 0;
        cnt.v[2] = (st & ST_ATMO) != 0;
        cnt.v[3] = !(st & ST_BRACKET_OK);
    }
    if (p.diag) block_accumulate<4, 0>(cnt, &p.diag->c2p_not_converged, nullptr);
}

struct SpeedParams {
    Grid g;
    const R *P[9];
    unsigned long long *out;  // [2]
};

// max(|v_d| + c_f) over the physical cells (driver2d.py:61-80), in double
__global__ void __launch_bounds__(kThreads) speed_kernel(const SpeedParams p) {
    const Grid &g = p.g;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long mx = 0, my = 0;
    if (e < (int64_t)g.nx * g.ny) {
        const int i = g.ng + (int)(e / g.ny), j = g.ng + (int)(e % g.ny);
        const int64_t c = (int64_t)i * g.nyt + j;
        double rho = p.P[P_RHO][c], eps = p.P[P_EPS][c];
        double vx = p.P[P_VX][c], vy = p.P[P_VY][c], vz = p.P[P_VZ][c];
        double Bx = p.P[P_BX][c], By = p.P[P_BY][c], Bz = p.P[P_BZ][c];
        double pr, cs2;
        eos_press_cs2(eps, rho, g.gamma, pr, cs2);
        double v2 = vx * vx + vy * vy + vz * vz;
        double W = 1.0 / sqrt(clamp_lo(1.0 - v2, 1e-10));
        double B2 = Bx * Bx + By * By + Bz * Bz;
        double vdotB = vx * Bx + vy * By + vz * Bz;
        double b2 = (B2 + vdotB * vdotB) / (W * W);
        double h = 1.0 + eps + pr / rho;
        double v02 = cs2 + (b2 / (rho * h + b2)) * (1.0 - cs2);
        double cf = sqrt(clamp_hi(clamp_lo(v02, 0.0), 1.0));
        mx = abs_bits(fabs(vx) + cf);
        my = abs_bits(fabs(vy) + cf);
    }
    unsigned long long bx = block_max_u64(mx);
    __syncthreads();
    unsigned long long by = block_max_u64(my);
    if (threadIdx.x == 0) {
        if (bx) atomicMax(p.out, bx);
        if (by) atomicMax(p.out + 1, by);
    }
}

// dt = cfl / (sx/dx + sy/dy), with torch's `cfl / tensor` = reciprocal * cfl
__global__ void dt_kernel(const unsigned long long *speeds, double dx, double dy, double cfl,
                          double *dt) {
    double mx = __longlong_as_double((long long)speeds[0]);
    double my = __longlong_as_double((long long)speeds[1]);
    if (isnan(mx) || isnan(my)) {
        *dt = mx + my;
        return;
    }
    double sx = clamp_lo(mx, 1e-14), sy = clamp_lo(my, 1e-14);
    *dt = (1.0 / (sx / dx + sy / dy)) * cfl;
}

// driver2d.py:104-105 in device memory
__constant__ double kRK3d[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
__constant__ double kRK2d[2][3] = {{1.0, 0.0, 1.0}, {0.5, 0.5, 0.5}};

// ── batched 1D tubes (one persistent launch) ─────────────────────────────
//
// Each tube is driver2d.py:110-156 rk_step on a ny = 1 grid (whose y sweep
// contributes exactly zero), advanced to tend with its own dt
// (driver.py:77-127 compute_dt).  A CTA takes whole tubes from an atomic
// counter (in the caller's order, e.g. longest first) and time-steps each
// one with block barriers between the face, update, boundary and C2P
// phases; a tube's arrays live in the concatenated cell / face arrays.

struct TubesParams {
    int ntubes, ng, max_steps, scheme;
    int light;      // driver flavors: max speed taken as 1 (dt = cfl dx)
    int resume;     // cons already valid: skip the prim -> cons at launch
    const int32_t *ncells;
    const int64_t *cell_off;  // first cell (ghosts included) of each tube
    const double *dx;
    const int32_t *order;
    double cfl, tend, gamma, atmo_rho;
    RS *U[8];   // conserved, all eight components
    RS *U0[8];
    R *P[9];        // primitives
    R *F[8];        // face fluxes (slot C_BX unused: F[Bx] = 0)
    double *t_out;
    int32_t *steps_out;
    unsigned int *next;
    int smem_faces;  // faces whose seven fluxes fit the CTA's dynamic shared memory
};

// HLLD_TUBE_PARK = 1 (float faces): the tube kernel's faces keep the values
// only the HLLD star states read again in a shared-memory slot during the
// p* solve (hlld_face's PARK_STRIDE, here the kernel's 512-thread maximum),
// at the front of the CTA's dynamic shared memory, before the fluxes
#ifndef HLLD_TUBE_PARK
#define HLLD_TUBE_PARK 1
#endif
constexpr int kTubeMaxThreads = 512;
constexpr int kTubePark = (HLLD_TUBE_PARK && sizeof(R) == sizeof(float)) ? kTubeMaxThreads : 0;
constexpr int kTubeParkBytes = kTubePark > 0 ? kParkWords * kTubeMaxThreads * (int)sizeof(R) : 0;

// The seven flux slots of a tube face (F[Bx] = 0 is never stored): slot of
// conserved component k
__device__ __forceinline__ int tube_flux_slot(int k) { return k < C_BX ? k : k - 1; }

template <int LIM, int SOLVER>
__device__ __forceinline__ void tube_face(const TubesParams &p, int64_t base, int nt, int f,
                                          R *const *Ft, R *park) {
    using T = R;
    constexpr int S = Stencil<LIM>::S;
    constexpr int NW = 2 * S + 2;
    // work variables (reconstruction.py:269) with vel_var Wv, all eight
    // (no face-B override: sweep.py Bnf = None)
    T L[8], Rt[8];
    if (f == 0 || f == nt) {
        const int64_t ci = base + (f == 0 ? 0 : nt - 1);
        T vx = p.P[P_VX][ci], vy = p.P[P_VY][ci], vz = p.P[P_VZ][ci];
        T v2 = vx * vx + vy * vy + vz * vz;
        T W = T(1) / sqrt(clamp_lo(T(1) - v2, T(1e-14)));
        T q[8] = {p.P[P_RHO][ci], p.P[P_P][ci], W * vx, W * vy, W * vz,
                  p.P[P_BX][ci], p.P[P_BY][ci], p.P[P_BZ][ci]};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            L[k] = q[k] + T(0.5) * T(0);
            Rt[k] = q[k] - T(0.5) * T(0);
        }
    } else {
        int cw[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            int c = f - 1 - S + k;
            cw[k] = c < 0 ? 0 : (c > nt - 1 ? nt - 1 : c);
        }
        T Wf[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            const int64_t ci = base + cw[k];
            T vx = p.P[P_VX][ci], vy = p.P[P_VY][ci], vz = p.P[P_VZ][ci];
            T v2 = vx * vx + vy * vy + vz * vz;
            Wf[k] = T(1) / sqrt(clamp_lo(T(1) - v2, T(1e-14)));
        }
        T pcmL[8], pcmR[8];
        constexpr int src[8] = {P_RHO, P_P, P_VX, P_VY, P_VZ, P_BX, P_BY, P_BZ};
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            T w[NW];
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                T x = p.P[src[v]][base + cw[k]];
                w[k] = (v >= 2 && v <= 4) ? Wf[k] * x : x;
            }
            L[v] = cell_edge<LIM, true, S>(w, f - 1, nt);
            Rt[v] = cell_edge<LIM, false, S + 1>(w, f, nt);
            pcmL[v] = w[S];
            pcmR[v] = w[S + 1];
        }
        if (LIM != HLLD_LIM_PCM) {
            bool bad = (L[0] <= T(1e-12)) || (Rt[0] <= T(1e-12)) || (L[1] <= T(1e-14)) ||
                       (Rt[1] <= T(1e-14));
            if (bad) {
#pragma unroll
                for (int v = 0; v < 8; ++v) {
                    L[v] = pcmL[v] + T(0.5) * T(0);
                    Rt[v] = pcmR[v] - T(0.5) * T(0);
                }
            }
        }
    }
    T PL[NPRIM], PR[NPRIM];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        T *q = side == 0 ? L : Rt;
        T *P = side == 0 ? PL : PR;
        T z2 = q[2] * q[2] + q[3] * q[3] + q[4] * q[4];
        T fac = T(1) / sqrt(T(1) + z2);
        P[P_VX] = q[2] * fac;
        P[P_VY] = q[3] * fac;
        P[P_VZ] = q[4] * fac;
        P[P_RHO] = clamp_lo(q[0], T(1e-12));
        P[P_P] = clamp_lo(q[1], T(1e-14));
        P[P_EPS] = eos_eps(P[P_P], P[P_RHO], (T)p.gamma);
        P[P_BX] = q[5];
        P[P_BY] = q[6];
        P[P_BZ] = q[7];
    }
    FaceOut<T> o;
    if (SOLVER == HLLD_SOLVER_HLLD)
        hlld_face<0, T, RB, RS, false, kSkipBnZero, false, kTubePark>(PL, PR, (T)p.gamma, false, o,
                                                                        nullptr, false, park);
    else
        hlle_face<0, T>(PL, PR, (T)p.gamma, false, false, o);
#pragma unroll
    for (int k = 0; k < 8; ++k)
        if (k != C_BX) Ft[tube_flux_slot(k)][f] = o.F[k];
}

// One physical face of the 1D shock-tube driver (driver.py:130-189,
// reconstruction.py:354-373): every primitive, eps included, reconstructed
// as it is along the whole line (no W v, no positivity fallback, no floors).
template <int LIM, int SOLVER>
__device__ __forceinline__ void tube_face_driver1d(const TubesParams &p, int64_t base, int nt, int f,
                                                   R *const *Ft) {
    using T = R;
    constexpr int S = Stencil<LIM>::S;
    constexpr int NW = 2 * S + 2;
    int cw[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        int c = f - 1 - S + k;
        cw[k] = c < 0 ? 0 : (c > nt - 1 ? nt - 1 : c);
    }
    T PL[NPRIM], PR[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; ++v) {
        T w[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) w[k] = p.P[v][base + cw[k]];
        PL[v] = cell_edge<LIM, true, S>(w, f - 1, nt);
        PR[v] = cell_edge<LIM, false, S + 1>(w, f, nt);
    }
    FaceOut<T> o;
    if (SOLVER == HLLD_SOLVER_HLLD)
        hlld_face<0, T, RB, RS, false, kSkipBnZero>(PL, PR, (T)p.gamma, false, o, nullptr, false);
    else
        hlle_face<0, T>(PL, PR, (T)p.gamma, false, false, o);
#pragma unroll
    for (int k = 0; k < 8; ++k)
        if (k != C_BX) Ft[tube_flux_slot(k)][f] = o.F[k];
}

__device__ __forceinline__ unsigned long long block_max_any(unsigned long long x,
                                                            unsigned long long *sm) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long y = __shfl_down_sync(0xffffffffu, x, o);
        x = x > y ? x : y;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long r = sm[0];
        for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww) r = r > sm[ww] ? r : sm[ww];
        sm[32] = r;
    }
    __syncthreads();
    unsigned long long r = sm[32];
    __syncthreads();
    return r;
}

// |vx| + v_fast of one cell (driver.py:77-127 compute_dt), as the bits of a
// non-negative double (ordered like the values; NaN above every number)
__device__ __forceinline__ unsigned long long tube_speed_bits(double rho, double eps, double vx,
                                                              double vy, double vz, double Bx,
                                                              double By, double Bz, double gamma) {
    double pr, cs2;
    eos_press_cs2(eps, rho, gamma, pr, cs2);
    double v2 = vx * vx + vy * vy + vz * vz;
    double W = 1.0 / sqrt(clamp_lo(1.0 - v2, 1e-10));
    double B2 = Bx * Bx + By * By + Bz * Bz;
    double vdotB = vx * Bx + vy * By + vz * Bz;
    double b2 = (B2 + vdotB * vdotB) / (W * W);
    double h = 1.0 + eps + pr / rho;
    double v02 = cs2 + (b2 / (rho * h + b2)) * (1.0 - cs2);
    double vf = sqrt(clamp_hi(clamp_lo(v02, 0.0), 1.0));
    return abs_bits(fabs(vx) + vf);
}

// DRV = false: driver2d.rk_step on a ny = 1 grid; DRV = true: the 1D
// driver's rk2_step (driver.py:192-236) and run loop (driver.py:388-412).
template <int LIM, int SOLVER, bool DRV>
// Up to 512 threads per CTA at 128 registers: one CTA of 512 threads per SM
// keeps all its warps in the same phase of the tube (faces, update, C2P),
// which the instruction cache rewards (measured on B200: +26 % over two CTAs
// of 256 on the batched workload).
//
// A stage is two passes separated by block barriers: the faces (fluxes into
// shared memory when the tube's faces fit, else into the face arrays), then
// per physical cell the RK update, the C2P and the outflow copies into the
// ghost cells that this cell feeds.  The fused second pass reads and writes
// each cell's state once per stage; its arithmetic is that of the separate
// update, boundary, C2P and boundary passes of the reference's stage.
__global__ void __launch_bounds__(512, 1) tubes_kernel(const TubesParams p) {
    __shared__ unsigned long long red[33];
    __shared__ int s_tube;
    extern __shared__ __align__(16) unsigned char tube_smem[];
    const int ng = p.ng;
    for (;;) {
        if (threadIdx.x == 0) s_tube = (int)atomicAdd(p.next, 1u);
        __syncthreads();
        const int q = s_tube;
        __syncthreads();
        if (q >= p.ntubes) return;
        const int ti = p.order ? p.order[q] : q;
        const int L = p.ncells[ti];
        const int nt = L + 2 * ng;
        const int64_t base = p.cell_off[ti];
        const int64_t fbase = base + ti;  // tube ti has nt + 1 faces
        const double dx = p.dx[ti];
        R *Ft[7];  // the tube's flux slots, indexed by face 0 .. nt
        {
            const bool in_smem = nt + 1 <= p.smem_faces;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (k == C_BX) continue;
                const int sl = tube_flux_slot(k);
                Ft[sl] = in_smem ? reinterpret_cast<R *>(tube_smem + kTubeParkBytes) + (int64_t)sl * (nt + 1)
                                 : p.F[k] + fbase;
            }
        }
        // conserved variables from the primitives (hlld.py:185-217)
        for (int c = threadIdx.x; c < nt && !p.resume; c += blockDim.x) {
            RS Pd[NPRIM], Cd[NCONS];
#pragma unroll
            for (int k = 0; k < NPRIM; ++k) Pd[k] = (RS)p.P[k][base + c];
            prim_to_cons<RS>(Pd, Cd);
#pragma unroll
            for (int k = 0; k < NCONS; ++k) p.U[k][base + c] = Cd[k];
        }
        __syncthreads();
        double t = 0.0;
        int steps = 0;
        const int nst = DRV ? 2 : (p.scheme == 3 ? 3 : 2);
        // this thread's max of |vx| + v_fast (as bits) over the cells it
        // updates; after the first step of the launch it comes from the last
        // stage's primitives, still in registers
        unsigned long long mloc = 0;
        while ((DRV ? t < p.tend : t < p.tend - 1e-14) && steps < p.max_steps) {
            // dt = (cfl dx) / max(|vx| + v_fast) over the physical cells
            if (steps == 0) {
                for (int c = ng + threadIdx.x; c < ng + L; c += blockDim.x) {
                    const int64_t ci = base + c;
                    const unsigned long long b = tube_speed_bits(
                        p.P[P_RHO][ci], p.P[P_EPS][ci], p.P[P_VX][ci], p.P[P_VY][ci],
                        p.P[P_VZ][ci], p.P[P_BX][ci], p.P[P_BY][ci], p.P[P_BZ][ci], p.gamma);
                    mloc = mloc > b ? mloc : b;
                }
            }
            double mx = __longlong_as_double((long long)block_max_any(mloc, red));
            mloc = 0;
            if (DRV && p.light) mx = 1.0;  // driver.py:120-125
            double dt = isnan(mx) ? mx : (1.0 / clamp_lo(mx, 1e-14)) * (p.cfl * dx);
            if (dt > p.tend - t) dt = p.tend - t;
            if (!(dt > 0.0)) break;
            for (int st = 0; st < nst; ++st) {
                const double *w = p.scheme == 3 ? kRK3d[st] : kRK2d[st];
                const RS w0 = RS(w[0]), w1 = RS(w[1]), w2 = RS(w[2] * dt);
                const RS rdt = RS(dt);
                if (DRV) {
                    // physical faces ng .. ng + L (reconstruction.py:354-373)
                    for (int f = ng + threadIdx.x; f <= ng + L; f += blockDim.x)
                        tube_face_driver1d<LIM, SOLVER>(p, base, nt, f, Ft);
                } else {
                    for (int f = threadIdx.x; f <= nt; f += blockDim.x)
                        tube_face<LIM, SOLVER>(p, base, nt, f, Ft,
                                               reinterpret_cast<R *>(tube_smem) + threadIdx.x);
                }
                __syncthreads();
                // per physical cell: the update -- Heun (driver.py:223-232): U1 = U
                // + dt L(U), U' = 0.5 (U + U1 + dt L(U1)), rhs = (F_c - F_c+1) / dx,
                // Bx held; or the SSP-RK combine of rk_step with F[Bx] = 0 --
                // then the C2P, then the outflow copies (grid.py:93-113) of U
                // and of the primitives into the ghost cells next to an edge
                for (int c = ng + threadIdx.x; c < ng + L; c += blockDim.x) {
                    const int64_t ci = base + c;
                    // (each thread loads all it needs before its first store:
                    // the arrays may alias for all the compiler knows, so a
                    // load after a store would wait for it)
                    RS u0[8], u[8];
                    R fl[8], fr[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        u[k] = p.U[k][ci];
                        // the first stage starts the step: U0 is U, stored here
                        // for the later stages (physical cells only; no stage
                        // reads U0 in a ghost cell)
                        u0[k] = st == 0 ? u[k] : p.U0[k][ci];
                        if (k != C_BX) {
                            fl[k] = Ft[tube_flux_slot(k)][c];
                            fr[k] = Ft[tube_flux_slot(k)][c + 1];
                        }
                    }
                    // mixed form: the root search starts from the root of the
                    // cell's primitives before the stage, which this C2P
                    // overwrites (the 2D step's first-stage start)
                    RS mu0 = RS(0);
                    if constexpr (sizeof(R) == sizeof(float) && sizeof(RS) == sizeof(double))
                        mu0 = kastaun_mu_of_prims<RS>(p.P, ci);
                    RS un[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        if (DRV) {
                            if (k == C_BX) {
                                un[k] = u[k];
                                continue;
                            }
                            const RS rhs = (RS)((fl[k] - fr[k]) / R(dx));
                            un[k] = st == 0 ? u0[k] + rdt * rhs : RS(0.5) * (u0[k] + u[k] + rdt * rhs);
                        } else {
                            RS rhs;
                            if (k == C_BX) {
                                rhs = -(RS(0) - RS(0)) / RS(dx) + RS(-0.0);
                            } else {
                                const R d = fr[k] - fl[k];
                                rhs = (RS)(-d / R(dx)) + RS(-0.0);
                            }
                            const RS v = w0 * u0[k] + w1 * u[k];
                            un[k] = v + w2 * rhs;
                        }
                    }
                    RS Pd[NPRIM];
                    cons_to_prim<RS>(un, RS(p.gamma), RS(p.atmo_rho), RS(1e-10), Pd, nullptr, mu0);
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        if (st == 0 && nst > 1) p.U0[k][ci] = u[k];
                        p.U[k][ci] = un[k];
                    }
#pragma unroll
                    for (int k = 0; k < NPRIM; ++k) p.P[k][ci] = (R)Pd[k];
                    if (st == nst - 1) {
                        // the next step's speed, from the primitives as stored:
                        // read back through volatile loads, so that the values
                        // are the rounded ones in memory (in registers, a
                        // contracting build could fuse the C2P's last products
                        // into the speed's sums)
                        auto stored = [&](int k) -> double {
                            return (double)*(const volatile R *)&p.P[k][ci];
                        };
                        const unsigned long long b = tube_speed_bits(
                            stored(P_RHO), stored(P_EPS), stored(P_VX), stored(P_VY),
                            stored(P_VZ), stored(P_BX), stored(P_BY), stored(P_BZ), p.gamma);
                        mloc = mloc > b ? mloc : b;
                    }
                    for (int side = 0; side < 2; ++side) {
                        if (c != (side == 0 ? ng : ng + L - 1)) continue;
                        const int g0 = side == 0 ? 0 : ng + L;
                        for (int gc = g0; gc < g0 + ng; ++gc) {
#pragma unroll
                            for (int k = 0; k < 8; ++k) p.U[k][base + gc] = un[k];
#pragma unroll
                            for (int k = 0; k < NPRIM; ++k) p.P[k][base + gc] = (R)Pd[k];
                        }
                    }
                }
                __syncthreads();
            }
            t += dt;
            ++steps;
        }
        if (threadIdx.x == 0) {
            p.t_out[ti] = t;
            p.steps_out[ti] = steps;
        }
        __syncthreads();
    }
}

// ── host-side launchers of this variant ──────────────────────────────────
// (HLLD_DEVICE_ONLY: a translation unit that needs only the device code and
// calls another unit's launchers)
#ifndef HLLD_DEVICE_ONLY

static inline unsigned grid1d(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

template <int IDIR>
static void launch_faces_idir(int solver, const FacesParams &fp, cudaStream_t st) {
    unsigned nb = grid1d(fp.n);
    if (solver == HLLD_SOLVER_HLLD)
        riemann_faces_kernel<IDIR, HLLD_SOLVER_HLLD><<<nb, kThreads, 0, st>>>(fp);
    else if (solver == HLLD_SOLVER_HLLC)
        riemann_faces_kernel<IDIR, HLLD_SOLVER_HLLC><<<nb, kThreads, 0, st>>>(fp);
    else
        riemann_faces_kernel<IDIR, HLLD_SOLVER_HLLE><<<nb, kThreads, 0, st>>>(fp);
}

void launch_riemann_faces(int64_t n, const void *const *sL, const void *const *sR, int idir,
                          int solver, double gamma, void *const *F, void *const *U, void *pstar,
                          int32_t *err, int32_t *iters, uint8_t *flags, hlld_flux_diag_t *diag,
                          cudaStream_t st) {
    FacesParams fp = {};
    fp.n = n;
    for (int k = 0; k < 9; ++k) {
        fp.sL[k] = (const double *)sL[k];
        fp.sR[k] = (const double *)sR[k];
    }
    for (int k = 0; k < 8; ++k) {
        fp.F[k] = (double *)F[k];
        fp.U[k] = U ? (double *)U[k] : nullptr;
    }
    fp.pstar = (double *)pstar;
    fp.err = err;
    fp.iters = iters;
    fp.flags = flags;
    fp.diag = diag;
    fp.gamma = gamma;
    if (idir == 0) launch_faces_idir<0>(solver, fp, st);
    else if (idir == 1) launch_faces_idir<1>(solver, fp, st);
    else launch_faces_idir<2>(solver, fp, st);
}

void launch_cons_to_prim(int64_t n, const void *const *cons, double gamma, double atmo_rho,
                         double atmo_eps, void *const *prim, uint8_t *status, cudaStream_t st) {
    CellsParams cp = {};
    cp.n = n;
    for (int k = 0; k < 8; ++k) cp.in[k] = (const double *)cons[k];
    for (int k = 0; k < 9; ++k) cp.out[k] = (double *)prim[k];
    cp.status = status;
    cp.gamma = gamma;
    cp.atmo_rho = atmo_rho;
    cp.atmo_eps = atmo_eps;
    c2p_kernel<<<grid1d(n), kThreads, 0, st>>>(cp);
}

void launch_prim_to_cons(int64_t n, const void *const *prim, void *const *cons, cudaStream_t st) {
    CellsParams cp = {};
    cp.n = n;
    for (int k = 0; k < 9; ++k) cp.in[k] = (const double *)prim[k];
    for (int k = 0; k < 8; ++k) cp.out[k] = (double *)cons[k];
    p2c_kernel<<<grid1d(n), kThreads, 0, st>>>(cp);
}

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
    G.emf_hll = g->emf_mode == HLLD_EMF_HLL;
    return G;
}

template <int AXIS, int LIM, bool EMF_HLL>
static void launch_sweep_emf(int solver, const SweepParams &sp, cudaStream_t st) {
    static_assert(kThreads == kTileAlong * kTileLanes, "one face per thread of a tile");
    const int rows = AXIS == 0 ? sp.g.nxt + 1 : sp.g.nxt;
    const int cols = AXIS == 0 ? sp.g.nyt : sp.g.nyt + 1;
    const unsigned nb = (unsigned)((int64_t)((rows + kTileAlong - 1) / kTileAlong) *
                                   ((cols + kTileLanes - 1) / kTileLanes));
    if (solver == HLLD_SOLVER_HLLD)
        sweep_kernel<AXIS, LIM, HLLD_SOLVER_HLLD, EMF_HLL><<<nb, kThreads, 0, st>>>(sp);
    else if (solver == HLLD_SOLVER_HLLC)
        sweep_kernel<AXIS, LIM, HLLD_SOLVER_HLLC, EMF_HLL><<<nb, kThreads, 0, st>>>(sp);
    else
        sweep_kernel<AXIS, LIM, HLLD_SOLVER_HLLE, EMF_HLL><<<nb, kThreads, 0, st>>>(sp);
}

// the HLL face EMF is a separate instantiation, so that the default sweep
// carries none of its code
template <int AXIS, int LIM>
static void launch_sweep_lim(int solver, const SweepParams &sp, cudaStream_t st) {
    if (sp.g.emf_hll) launch_sweep_emf<AXIS, LIM, true>(solver, sp, st);
    else launch_sweep_emf<AXIS, LIM, false>(solver, sp, st);
}

template <int AXIS>
static void launch_sweep(int limiter, int solver, const SweepParams &sp, cudaStream_t st) {
    switch (limiter) {
    case HLLD_LIM_PCM: launch_sweep_lim<AXIS, HLLD_LIM_PCM>(solver, sp, st); break;
    case HLLD_LIM_MC: launch_sweep_lim<AXIS, HLLD_LIM_MC>(solver, sp, st); break;
    case HLLD_LIM_MINMOD: launch_sweep_lim<AXIS, HLLD_LIM_MINMOD>(solver, sp, st); break;
    case HLLD_LIM_WENO5Z: launch_sweep_lim<AXIS, HLLD_LIM_WENO5Z>(solver, sp, st); break;
    case HLLD_LIM_MP5: launch_sweep_lim<AXIS, HLLD_LIM_MP5>(solver, sp, st); break;
    default: launch_sweep_lim<AXIS, HLLD_LIM_MP7>(solver, sp, st); break;
    }
}

template <typename E>
static void launch_ghost_cc(const Grid &G, E *const *arrs, int narr, cudaStream_t st) {
    GhostParams<E> gp = {};
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
    int64_t cnt = (int64_t)gp.n0 * gp.n1 - (int64_t)(gp.b0 - gp.a0) * (gp.b1 - gp.a1);
    ghost_kernel<E><<<dim3(grid1d(cnt), narr), kThreads, 0, st>>>(gp);
}

static void launch_ghost_faces(const Grid &G, RS *Bxf, RS *Byf, cudaStream_t st) {
    // Bxf: face rule along x, cell rule along y (grid.py:250-251)
    GhostParams<RS> gp = {};
    gp.v[0] = Bxf;
    gp.n0 = G.nxt + 1;
    gp.n1 = G.nyt;
    gp.a0 = G.ng;
    gp.b0 = G.ng + G.nx + (G.bc_x == HLLD_BC_OUTFLOW ? 1 : 0);
    gp.a1 = G.ng;
    gp.b1 = G.ng + G.ny;
    gp.n_ph0 = G.nx;
    gp.n_ph1 = G.ny;
    gp.ng = G.ng;
    gp.kind0 = G.bc_x;
    gp.kind1 = G.bc_y;
    gp.face0 = 1;
    gp.face1 = 0;
    int64_t cnt = (int64_t)gp.n0 * gp.n1 - (int64_t)(gp.b0 - gp.a0) * (gp.b1 - gp.a1);
    ghost_kernel<RS><<<dim3(grid1d(cnt), 1), kThreads, 0, st>>>(gp);
    // Byf: cell rule along x, face rule along y (grid.py:253-254)
    GhostParams<RS> gq = {};
    gq.v[0] = Byf;
    gq.n0 = G.nxt;
    gq.n1 = G.nyt + 1;
    gq.a0 = G.ng;
    gq.b0 = G.ng + G.nx;
    gq.a1 = G.ng;
    gq.b1 = G.ng + G.ny + (G.bc_y == HLLD_BC_OUTFLOW ? 1 : 0);
    gq.n_ph0 = G.nx;
    gq.n_ph1 = G.ny;
    gq.ng = G.ng;
    gq.kind0 = G.bc_x;
    gq.kind1 = G.bc_y;
    gq.face0 = 0;
    gq.face1 = 1;
    cnt = (int64_t)gq.n0 * gq.n1 - (int64_t)(gq.b0 - gq.a0) * (gq.b1 - gq.a1);
    ghost_kernel<RS><<<dim3(grid1d(cnt), 1), kThreads, 0, st>>>(gq);
}

void launch_sync_state(const hlld_grid2d_t *g, const hlld_state2d_t *s, uint8_t *status,
                       hlld_step_diag_t *diag, cudaStream_t st, double *mu_out, double *mu_warm,
                       bool start_from_prims, cudaEvent_t after_cons) {
    Grid G = make_grid(g);
    RS *cons[6];
    for (int k = 0; k < 6; ++k) cons[k] = (RS *)s->cons[k];
    R *prims[9];
    for (int k = 0; k < 9; ++k) prims[k] = (R *)s->prims[k];
    launch_ghost_faces(G, (RS *)s->Bxf, (RS *)s->Byf, st);
    launch_ghost_cc<RS>(G, cons, 6, st);
    // the conserved arrays and the faces are final here: the C2P and the
    // primitive ghosts only read them
    if (after_cons) cudaEventRecord(after_cons, st);
    C2PCellsParams cp = {};
    cp.g = G;
    for (int k = 0; k < 6; ++k) cp.U[k] = cons[k];
    cp.Bxf = (const RS *)s->Bxf;
    cp.Byf = (const RS *)s->Byf;
    for (int k = 0; k < 9; ++k) cp.P[k] = prims[k];
    cp.status = status;
    cp.diag = diag;
    cp.mu_out = mu_out;
    cp.mu_warm = mu_warm;
    if (start_from_prims)
        c2p_cells_kernel<true><<<grid1d((int64_t)G.nx * G.ny), kThreads, 0, st>>>(cp);
    else
        c2p_cells_kernel<false><<<grid1d((int64_t)G.nx * G.ny), kThreads, 0, st>>>(cp);
    launch_ghost_cc<R>(G, prims, 9, st);
}

void launch_sweep2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, int axis, void *const *F,
                    hlld_flux_diag_t *fdiag, cudaStream_t st, double *pstar_out, uint8_t *fail_out) {
    SweepParams sp = {};
    sp.pstar_out = pstar_out;
    sp.fail_out = fail_out;
    sp.g = make_grid(g);
    sp.rho = (const R *)s->prims[P_RHO];
    sp.p = (const R *)s->prims[P_P];
    sp.vx = (const R *)s->prims[P_VX];
    sp.vy = (const R *)s->prims[P_VY];
    sp.vz = (const R *)s->prims[P_VZ];
    sp.bz = (const R *)s->prims[P_BZ];
    sp.Bxf = (const RS *)s->Bxf;
    sp.Byf = (const RS *)s->Byf;
    for (int k = 0; k < NFLUX; ++k) sp.F[k] = (R *)F[k];
    sp.diag = fdiag;
    if (axis == 0) launch_sweep<0>(g->limiter, g->solver, sp, st);
    else launch_sweep<1>(g->limiter, g->solver, sp, st);
}

// driver2d.py:104-105
static const double kRK3[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
static const double kRK2[2][3] = {{1.0, 0.0, 1.0}, {0.5, 0.5, 0.5}};

void launch_ct_update2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, const Scratch2D &sc,
                        const hlld_step_diag_t *diag, int stage, int scheme, double dt_host,
                        const double *dt_dev, cudaStream_t st) {
    Grid G = make_grid(g);
    const double *w = scheme == 3 ? kRK3[stage] : kRK2[stage];
    const int64_t ncorner = (int64_t)(G.nxt + 1) * (G.nyt + 1);
    CtParams cp = {};
    cp.g = G;
    cp.vx = (const R *)s->prims[P_VX];
    cp.vy = (const R *)s->prims[P_VY];
    cp.Bxf = (const RS *)s->Bxf;
    cp.Byf = (const RS *)s->Byf;
    cp.FxD = (const R *)sc.Fx[F_D];
    cp.FyD = (const R *)sc.Fy[F_D];
    cp.FxBt = (const R *)sc.Fx[F_BT];
    cp.FyBt = (const R *)sc.Fy[F_BT];
    cp.diag = diag;
    cp.upwind = g->upwind;
    cp.Ez = (R *)sc.Ez;
    ct_emf_kernel<<<grid1d(ncorner), kThreads, 0, st>>>(cp);
    UpdateParams up = {};
    up.g = G;
    for (int k = 0; k < 6; ++k) {
        up.U[k] = (RS *)s->cons[k];
        up.U0[k] = (RS *)sc.U0[k];
        up.Fx[k] = (const R *)sc.Fx[k];
        up.Fy[k] = (const R *)sc.Fy[k];
    }
    up.Bxf = (RS *)s->Bxf;
    up.Byf = (RS *)s->Byf;
    up.Bx0 = (RS *)sc.Bx0;
    up.By0 = (RS *)sc.By0;
    up.Ez = (const R *)sc.Ez;
    up.dt_dev = dt_dev;
    up.dt_host = dt_host;
    up.a = w[0];
    up.b = w[1];
    up.c = w[2];
    up.first_stage = stage == 0;
    ct_update_kernel<<<grid1d((int64_t)(G.nx + 1) * (G.ny + 1)), kThreads, 0, st>>>(up);
}

// cons_in (may be NULL): waited for before the first stage's update, the
// first launch that reads the conserved cell arrays; cons_out (may be NULL):
// recorded once the conserved arrays and the faces hold the step's result.
void launch_rk_step_ct(const hlld_grid2d_t *g, const hlld_state2d_t *s, const Scratch2D &sc,
                       double dt_host, const double *dt_dev, int scheme, hlld_step_diag_t *diag,
                       cudaStream_t st, cudaEvent_t cons_in, cudaEvent_t cons_out) {
    const int nst = scheme == 3 ? 3 : 2;
    for (int stage = 0; stage < nst; ++stage) {
        // sweep counters and max |F_D| restart every stage; the CT scale is
        // the current stage's (ct.py:114)
        cudaMemsetAsync(diag, 0, sizeof(hlld_step_diag_t), st);
        launch_sweep2d(g, s, 0, sc.Fx, &diag->sweep[0], st);
        launch_sweep2d(g, s, 1, sc.Fy, &diag->sweep[1], st);
        if (stage == 0 && cons_in) cudaStreamWaitEvent(st, cons_in, 0);
        launch_ct_update2d(g, s, sc, diag, stage, scheme, dt_host, dt_dev, st);
        cudaEvent_t last = stage == nst - 1 ? cons_out : nullptr;
        // mixed form: stage 0 starts every cell's C2P root search from the
        // step's input primitives (mu = 1 / (h W)) and keeps the roots; the
        // later stages start from those (so a step depends on its input
        // state alone)
        if (stage == 0) launch_sync_state(g, s, nullptr, diag, st, sc.mu_warm, nullptr,
                                            sc.mu_warm != nullptr, last);
        else launch_sync_state(g, s, nullptr, diag, st, nullptr, sc.mu_warm, false, last);
    }
}

// Dynamic shared memory of a tube CTA for the fluxes of its tube: at most
// 120 KB (the faces of a 4096-cell tube in the FP32 flux types), and no more
// than the SM's share for the CTAs that run on it, so that the stencil loads
// keep the rest of the SM's 256 KB of L1 / shared memory as cache.
static constexpr int kTubeSmemCap = 120 * 1024;

template <typename K>
static void tube_launch(K kernel, TubesParams tp, int blocks, int threads, cudaStream_t st) {
    int dev = 0, sms = 1, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    const int ctas_per_sm = (blocks + sms - 1) / (sms > 0 ? sms : 1);
    // the parking slot first (always), then the fluxes in what the SM's
    // share leaves
    int bytes = per_sm / (ctas_per_sm > 0 ? ctas_per_sm : 1) - 2048 - kTubeParkBytes;
    if (bytes > kTubeSmemCap) bytes = kTubeSmemCap;
    if (bytes < 0) bytes = 0;
    tp.smem_faces = bytes / (7 * (int)sizeof(R));
    bytes = kTubeParkBytes + tp.smem_faces * 7 * (int)sizeof(R);
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) {
        cudaGetLastError();  // clear it: fall back to the face arrays
        tp.smem_faces = 0;
        bytes = kTubeParkBytes;
    }
    kernel<<<blocks, threads, bytes, st>>>(tp);
}

template <int LIM>
static void launch_tubes_lim(int solver, bool drv, const TubesParams &tp, int blocks, int threads,
                             cudaStream_t st) {
    if (solver == HLLD_SOLVER_HLLD) {
        if (drv) tube_launch(tubes_kernel<LIM, HLLD_SOLVER_HLLD, true>, tp, blocks, threads, st);
        else tube_launch(tubes_kernel<LIM, HLLD_SOLVER_HLLD, false>, tp, blocks, threads, st);
    } else {
        if (drv) tube_launch(tubes_kernel<LIM, HLLD_SOLVER_HLLE, true>, tp, blocks, threads, st);
        else tube_launch(tubes_kernel<LIM, HLLD_SOLVER_HLLE, false>, tp, blocks, threads, st);
    }
}

void launch_tubes_run(const hlld_tubes_t *b, void *const *cons, void *const *prims,
                      void *const *U0, void *const *F, double *t_out, int32_t *steps_out,
                      unsigned int *next, int threads, int blocks, cudaStream_t st) {
    TubesParams tp = {};
    tp.ntubes = b->ntubes;
    tp.ng = b->ng;
    tp.max_steps = b->max_steps;
    tp.scheme = b->scheme;
    tp.light = b->flavor == HLLD_TUBE_DRIVER1D_LIGHT;
    tp.resume = b->resume;
    const bool drv = b->flavor != HLLD_TUBE_RK_STEP;
    tp.ncells = b->ncells;
    tp.cell_off = b->cell_off;
    tp.dx = b->dx;
    tp.order = b->order;
    tp.cfl = b->cfl;
    tp.tend = b->tend;
    tp.gamma = b->gamma;
    tp.atmo_rho = b->atmo_rho;
    for (int k = 0; k < 8; ++k) {
        tp.U[k] = (RS *)cons[k];
        tp.U0[k] = (RS *)U0[k];
        tp.F[k] = (R *)F[k];
    }
    for (int k = 0; k < 9; ++k) tp.P[k] = (R *)prims[k];
    tp.t_out = t_out;
    tp.steps_out = steps_out;
    tp.next = next;
    cudaMemsetAsync(next, 0, sizeof(unsigned int), st);
    switch (b->limiter) {
    case HLLD_LIM_PCM: launch_tubes_lim<HLLD_LIM_PCM>(b->solver, drv, tp, blocks, threads, st); break;
    case HLLD_LIM_MC: launch_tubes_lim<HLLD_LIM_MC>(b->solver, drv, tp, blocks, threads, st); break;
    case HLLD_LIM_MINMOD: launch_tubes_lim<HLLD_LIM_MINMOD>(b->solver, drv, tp, blocks, threads, st); break;
    case HLLD_LIM_WENO5Z: launch_tubes_lim<HLLD_LIM_WENO5Z>(b->solver, drv, tp, blocks, threads, st); break;
    case HLLD_LIM_MP5: launch_tubes_lim<HLLD_LIM_MP5>(b->solver, drv, tp, blocks, threads, st); break;
    default: launch_tubes_lim<HLLD_LIM_MP7>(b->solver, drv, tp, blocks, threads, st); break;
    }
}

void launch_compute_dt_2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, double cfl,
                          double *dt_dev, unsigned long long *work, cudaStream_t st) {
    Grid G = make_grid(g);
    cudaMemsetAsync(work, 0, 2 * sizeof(unsigned long long), st);
    SpeedParams sp = {};
    sp.g = G;
    for (int k = 0; k < 9; ++k) sp.P[k] = (const R *)s->prims[k];
    sp.out = work;
    speed_kernel<<<grid1d((int64_t)G.nx * G.ny), kThreads, 0, st>>>(sp);
    dt_kernel<<<1, 1, 0, st>>>(work, g->dx, g->dy, cfl, dt_dev);
}

#endif  // HLLD_DEVICE_ONLY

}  // namespace HLLD_NS
}  // namespace hlld
