"""Generate the golden vectors in this directory from the reference itself.

Run in a checkout that has kemi2805/HLLD-AI available (read-only):

    python tests/golden/make_golden.py /path/to/HLLD-AI

It imports the reference's ``src.physics`` modules and records, on seeded
inputs, the outputs the oracle is pinned against (tests/test_oracle_golden.py):

  riemann.npz  hlle_flux / hlld_flux on 512 face states for idir 0, 1, 2
               (batched calls), and hlld_flux face by face on 64 of them
  c2p.npz      conservative_to_primitive on seeded batches of six regimes,
               the Komissarov-1 left state and the hot-fast-gas batch
  recon.npz    reconstruct() for every limiter and axis on a random field,
               reconstruct_prims() for mc / weno5z / mp5
  ct.npz       corner_emf() on random EMFs and mass fluxes (upwind on/off)
  step2d.npz   sync_state + two rk_step_ct steps of four small 2D problems
  tube1d.npz   six rk2_step steps of the 800-cell Brio-Wu tube (PLM-MC, HLLD)
  tubes.npz    three batched-workload tubes (WENO5-Z, HLLD, SSP-RK3): driver2d
               rk_step on ny = 1 grids with driver.compute_dt, four steps each
  hllc.npz     hllc_flux for idir 0-2 on 512 seeded face pairs, a quarter of
               them with zero normal field (``python make_golden.py REF hllc``
               writes only this file)
  emf_hll.npz  sync_state + two rk_step_ct steps with emf_mode="hll" (the
               HLL face EMF, ct.py:63-88) of the rotor and the Orszag-Tang
               vortex, HLLD and HLLE (``python make_golden.py REF emf_hll``
               writes only this file)
  rotor_gradient.npz  the gradient of J = sum w |B|^2 / 2 through
               rk_step_ct on the tapered rotor, by central differences of
               the reference and by shimmed torch autograd (``python
               make_golden.py REF gradient N STEPS``, only this file; see
               make_gradient)

The reference is not needed to run the tests; only this script reads it.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    sys.dont_write_bytecode = True
    os.environ.pop("RMHD_PSTAR_METHOD", None)
    sys.path.insert(0, ref_root)
    import torch
    from src.physics.c2p import conservative_to_primitive
    from src.physics.ct import corner_emf
    from src.physics.driver import compute_rhs, rk2_step  # noqa: F401
    from src.physics.driver2d import prims_to_cons_2d, rk_step_ct, sync_state, compute_dt_2d
    from src.physics.eos import hybrid_eos
    from src.physics.grid import Grid1D, Grid2D
    from src.physics.hlld import hlld_flux, hlle_flux, primitive_to_conserved
    from src.physics.initial_data import brio_wu, init_shocktube
    from src.physics.initial_data2d import (b_from_potential, magnetic_rotor, orszag_tang,
                                            riemann2d)
    from src.physics import reconstruction as rec
    from src.physics.state import EVOLVED_KEYS, State2D

    torch.set_num_threads(4)
    PK = ("rho", "vx", "vy", "vz", "p", "eps", "Bx", "By", "Bz")
    CK = ("D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz")
    G = 5.0 / 3.0
    eos = hybrid_eos(K=0.0, gamma=G, gamma_th=G)

    # ── riemann ─────────────────────────────────────────────────────────
    n = 512
    g = torch.Generator().manual_seed(20260824)

    def u(lo, hi, m=n):
        return torch.empty(m, dtype=torch.float64).uniform_(lo, hi, generator=g)

    def one():
        rho = 10.0 ** u(-1.0, 1.0)
        p = 10.0 ** u(-1.5, 1.0)
        W = 1.0 + 10.0 ** u(-3.0, math.log10(4.0))
        sp = torch.sqrt(1.0 - 1.0 / W**2)
        th, ph = u(0, math.pi), u(0, 2 * math.pi)
        s = {"rho": rho, "p": p, "vx": sp * torch.sin(th) * torch.cos(ph),
             "vy": sp * torch.sin(th) * torch.sin(ph), "vz": sp * torch.cos(th),
             "Bx": u(-3, 3), "By": u(-3, 3), "Bz": u(-3, 3)}
        s["eps"] = eos.eps__press_rho(s["p"], s["rho"])
        return s

    sL, sR = one(), one()
    for k in ("Bx", "By", "Bz"):
        sR[k] = sL[k].clone()
    out = {f"L_{k}": sL[k].numpy() for k in PK}
    out.update({f"R_{k}": sR[k].numpy() for k in PK})
    out["gamma"] = np.float64(G)
    for name, fn in (("hlle", hlle_flux), ("hlld", hlld_flux)):
        for idir in (0, 1, 2):
            F, U, ps = fn(sL, sR, eos, idir=idir)
            for k in CK:
                out[f"{name}{idir}_F_{k}"] = F[k].numpy()
                out[f"{name}{idir}_U_{k}"] = U[k].numpy()
            out[f"{name}{idir}_pstar"] = ps.numpy()
    single = {k: [] for k in CK}
    ps1 = []
    for i in range(64):
        F, U, ps = hlld_flux({k: v[i:i + 1] for k, v in sL.items()},
                             {k: v[i:i + 1] for k, v in sR.items()}, eos, idir=0)
        for k in CK:
            single[k].append(F[k].item())
        ps1.append(ps.item())
    for k in CK:
        out[f"single_F_{k}"] = np.array(single[k])
    out["single_pstar"] = np.array(ps1)
    np.savez_compressed(os.path.join(HERE, "riemann.npz"), **out)

    # ── c2p ─────────────────────────────────────────────────────────────
    cases = {"hydro": dict(zero_B=True, W=(1, 2), rho=(1e-3, 1e2), B=1.0, seed=1),
             "mhd": dict(zero_B=False, W=(1, 2), rho=(1e-3, 1e2), B=5.0, seed=3),
             "W2_10": dict(zero_B=False, W=(2, 10), rho=(1e-3, 1e2), B=3.0, seed=6),
             "low_rho": dict(zero_B=False, W=(1, 2), rho=(1e-8, 1e-4), B=0.1, seed=7),
             "B_dom": dict(zero_B=False, W=(1, 2), rho=(1e-3, 1e-1), B=20.0, seed=8),
             "mild": dict(zero_B=False, W=(1, 2), rho=(1e-3, 1e2), B=3.0, seed=5)}
    out = {"gamma": np.float64(G)}
    m = 200
    for name, c in cases.items():
        gg = torch.Generator().manual_seed(c["seed"])
        r = lambda: torch.rand(m, dtype=torch.float64, generator=gg)
        lo, hi = math.log10(c["rho"][0]), math.log10(c["rho"][1])
        rho = 10.0 ** (lo + (hi - lo) * r())
        p = rho * (0.01 + r())
        W = c["W"][0] + (c["W"][1] - c["W"][0]) * r()
        v = torch.sqrt(1.0 - 1.0 / W**2)
        ct = 2 * r() - 1
        st = torch.sqrt(torch.clamp(1 - ct**2, min=0.0))
        ph = 2 * math.pi * r()
        if c["zero_B"]:
            B = [torch.zeros(m, dtype=torch.float64)] * 3
        else:
            Bm, cb, pb = c["B"] * r(), 2 * r() - 1, 2 * math.pi * r()
            sb = torch.sqrt(torch.clamp(1 - cb**2, min=0.0))
            B = [Bm * sb * torch.cos(pb), Bm * sb * torch.sin(pb), Bm * cb]
        pr = {"rho": rho, "vx": v * st * torch.cos(ph), "vy": v * st * torch.sin(ph),
              "vz": v * ct, "p": p, "Bx": B[0], "By": B[1], "Bz": B[2]}
        pr["eps"] = eos.eps__press_rho(p, rho)
        cons = primitive_to_conserved(pr)
        o, s = conservative_to_primitive(cons, eos, atmo_rho=1e-12, return_status=True)
        for k in CK:
            out[f"{name}_C_{k}"] = cons[k].numpy()
        for k in PK:
            out[f"{name}_in_{k}"] = pr[k].numpy()
            out[f"{name}_P_{k}"] = o[k].numpy()
        out[f"{name}_converged"] = s["converged"].numpy()
    # hot fast gas (reference tests/test_c2p.py:303-318)
    b = 0.5 * math.cos(math.radians(45))
    t = lambda *v: torch.tensor(v, dtype=torch.float64)
    hp = {"rho": t(0.1, 0.1, 0.5, 0.1, 0.1, 1.0, 10.0, 0.22), "p": t(1.0, 0.01, 1.0, 1.0, 1.0, 1.0, 1.0, 0.13),
          "vx": t(0.99, 0.0, 0.0, 0.0, 0.99, 0.3, 0.995, 0.7), "vy": t(0.0, 0.0, 0.0, 0.99, 0.0, 0.1, 0.0, 0.7),
          "vz": t(0, 0, 0, 0, 0, 0, 0, 0), "Bx": t(b, b, b, b, 0.0, 0.5, 1.0, 0.28),
          "By": t(b, b, b, b, 0.0, 0.0, 0.0, 0.28), "Bz": t(0, 0, 0, 0, 0, 0, 0, 0)}
    hp["eps"] = eos.eps__press_rho(hp["p"], hp["rho"])
    hc = primitive_to_conserved(hp)
    ho, hs = conservative_to_primitive(hc, eos, return_status=True)
    for k in CK:
        out[f"hot_C_{k}"] = hc[k].numpy()
    for k in PK:
        out[f"hot_in_{k}"] = hp[k].numpy()
        out[f"hot_P_{k}"] = ho[k].numpy()
    out["hot_converged"] = hs["converged"].numpy()
    np.savez_compressed(os.path.join(HERE, "c2p.npz"), **out)

    # ── reconstruction ──────────────────────────────────────────────────
    gen = torch.Generator().manual_seed(99)
    q = torch.randn(14, 12, dtype=torch.float64, generator=gen)
    out = {"q": q.numpy()}
    for lim in ("pcm", "mc", "minmod", "weno5z", "mp5", "mp7"):
        for axis in (0, 1):
            QL, QR = rec.reconstruct(q, axis=axis, limiter=lim)
            out[f"{lim}{axis}_L"] = QL.numpy()
            out[f"{lim}{axis}_R"] = QR.numpy()
    # primitive field for reconstruct_prims
    r = lambda: torch.rand(12, 10, dtype=torch.float64, generator=gen)
    pr = {"rho": 0.1 + 2 * r(), "p": 0.05 + r(), "vx": 0.6 * (r() - 0.5), "vy": 0.6 * (r() - 0.5),
          "vz": 0.6 * (r() - 0.5), "Bx": r() - 0.5, "By": r() - 0.5, "Bz": r() - 0.5}
    pr["rho"][3, 4] = 1e-13  # a face pair that falls back to PCM
    pr["eps"] = eos.eps__press_rho(pr["p"], pr["rho"])
    for k in PK:
        out[f"prim_{k}"] = pr[k].numpy()
    for lim in ("mc", "weno5z", "mp5"):
        for axis in (0, 1):
            L, R = rec.reconstruct_prims(pr, axis, eos, limiter=lim)
            for k in PK:
                out[f"rp_{lim}{axis}_L_{k}"] = L[k].numpy()
                out[f"rp_{lim}{axis}_R_{k}"] = R[k].numpy()
    np.savez_compressed(os.path.join(HERE, "recon.npz"), **out)

    # ── corner EMF ──────────────────────────────────────────────────────
    gen = torch.Generator().manual_seed(4242)
    NXT, NYT = 14, 12
    Ec = torch.randn(NXT, NYT, dtype=torch.float64, generator=gen)
    Efx = torch.randn(NXT + 1, NYT, dtype=torch.float64, generator=gen)
    Efy = torch.randn(NXT, NYT + 1, dtype=torch.float64, generator=gen)
    Fx = torch.randn(NXT + 1, NYT, dtype=torch.float64, generator=gen)
    Fy = torch.randn(NXT, NYT + 1, dtype=torch.float64, generator=gen)
    Fx[2, 3] = 1e-12  # inside the deadband
    out = {"Ec": Ec.numpy(), "Efx": Efx.numpy(), "Efy": Efy.numpy(), "Fx": Fx.numpy(),
           "Fy": Fy.numpy()}
    out["Ez_up"] = corner_emf(Ec, Efx, Efy, Fx, Fy, upwind=True).numpy()
    out["Ez_flux_ct"] = corner_emf(Ec, Efx, Efy, Fx, Fy, upwind=False).numpy()
    np.savez_compressed(os.path.join(HERE, "ct.npz"), **out)

    # ── 2D steps ────────────────────────────────────────────────────────
    out = {}
    probs = {
        "rotor": (magnetic_rotor, (-0.5, 0.5), 5 / 3, ("outflow", "outflow"), "mc", 16),
        "ot": (orszag_tang, (0.0, 1.0), 4 / 3, ("periodic", "periodic"), "mc", 16),
        "r2d_weno": (riemann2d, (-0.5, 0.5), 5 / 3, ("outflow", "outflow"), "weno5z", 16),
        "ot_mp5": (orszag_tang, (0.0, 1.0), 4 / 3, ("periodic", "periodic"), "mp5", 14),
    }
    for name, (build, box, gam, bc, lim, nn) in probs.items():
        e = hybrid_eos(K=0.0, gamma=gam, gamma_th=gam)
        gr = Grid2D(box[0], box[1], nn, box[0], box[1], nn, ng=rec.ghosts_needed(lim))
        prims, Az = build(gr, e)
        Bxf, Byf = b_from_potential(Az, gr.dx, gr.dy)
        for k in PK:
            out[f"{name}_init_{k}"] = prims[k].numpy().copy()
        out[f"{name}_init_Bxf"] = Bxf.numpy().copy()
        out[f"{name}_init_Byf"] = Byf.numpy().copy()
        c = prims_to_cons_2d(prims, gr)
        st = State2D(cons={k: c[k] for k in EVOLVED_KEYS}, Bxf=Bxf, Byf=Byf, prims=prims)
        st = sync_state(st, gr, e, *bc)
        dts = []
        for _ in range(2):
            dt = compute_dt_2d(st.prims, gr, e, 0.4)
            dts.append(dt)
            st, _ = rk_step_ct(st, gr, e, dt, scheme="rk3", bc_x=bc[0], bc_y=bc[1], limiter=lim)
        out[f"{name}_dt"] = np.array(dts)
        for k in EVOLVED_KEYS:
            out[f"{name}_cons_{k}"] = st.cons[k].numpy()
        for k in PK:
            out[f"{name}_prims_{k}"] = st.prims[k].numpy()
        out[f"{name}_Bxf"] = st.Bxf.numpy()
        out[f"{name}_Byf"] = st.Byf.numpy()
        out[f"{name}_meta"] = np.array([nn, rec.ghosts_needed(lim), gam, gr.dx, gr.dy])
    np.savez_compressed(os.path.join(HERE, "step2d.npz"), **out)

    # ── 1D Brio-Wu tube (driver.py rk2_step, PLM-MC, HLLD) ──────────────
    e = hybrid_eos(K=0.0, gamma=2.0, gamma_th=2.0)
    gr = Grid1D(0.0, 1.0, 800, ng=2)
    pL, pR, x0 = brio_wu()
    for pp in (pL, pR):
        pp["eps"] = e.eps__press_rho(pp["p"], pp["rho"])
    prims = init_shocktube(gr, pL, pR, x0)
    cons = primitive_to_conserved(prims)
    gr.apply_outflow_bc(prims)
    gr.apply_outflow_bc(cons)
    out = {f"init_{k}": prims[k].numpy().copy() for k in prims}
    dt = 0.4 * gr.dx
    for _ in range(6):
        cons, prims = rk2_step(cons, prims, gr, e, torch.tensor(dt, dtype=torch.float64), 1e-10,
                               flux_fn=hlld_flux, limiter="mc")
    out.update({f"prims_{k}": prims[k].numpy() for k in prims})
    out.update({f"cons_{k}": cons[k].numpy() for k in cons})
    out["dt"] = np.float64(dt)
    np.savez_compressed(os.path.join(HERE, "tube1d.npz"), **out)

    # ── batched-workload tubes (driver2d.rk_step on ny = 1, driver.compute_dt) ──
    from src.physics.driver import compute_dt
    from src.physics.driver2d import rk_step
    out = {}
    gen = np.random.default_rng(20261203)
    for ti, L in enumerate((64, 96, 128)):
        e = hybrid_eos(K=0.0, gamma=G, gamma_th=G)
        gr = Grid2D(0.0, 1.0, L, 0.0, 1.0, 1, ng=3)
        rho = 10.0 ** gen.uniform(-1, 1, 2)
        p = 10.0 ** gen.uniform(-2, 2, 2)
        v = gen.uniform(-0.5, 0.5, (2, 3))
        Bt = gen.uniform(-2, 2, (2, 2))
        bx = gen.uniform(-1, 1)
        left = gr.X < 0.5
        pick = lambda a, b: torch.where(left, torch.full_like(gr.X, float(a)), torch.full_like(gr.X, float(b)))
        prims = {"rho": pick(rho[0], rho[1]), "p": pick(p[0], p[1]),
                 "vx": pick(v[0, 0], v[1, 0]), "vy": pick(v[0, 1], v[1, 1]),
                 "vz": pick(v[0, 2], v[1, 2]), "Bx": torch.full_like(gr.X, float(bx)),
                 "By": pick(Bt[0, 0], Bt[1, 0]), "Bz": pick(Bt[0, 1], Bt[1, 1])}
        prims = {k: vv.contiguous().clone() for k, vv in prims.items()}
        prims["eps"] = e.eps__press_rho(prims["p"], prims["rho"])
        for k in PK:
            out[f"t{ti}_init_{k}"] = prims[k][:, 3].numpy().copy()
        cons = prims_to_cons_2d(prims, gr)
        cons = {k: cons[k] for k in CK}
        dts = []
        for _ in range(4):
            row = {k: prims[k][:, 3] for k in PK}
            dt = float(compute_dt(row, e, gr.dx, 0.4, gr.ng, L))
            dts.append(dt)
            cons, prims, _ = rk_step(cons, prims, gr, e, dt, scheme="rk3", bc_x="outflow",
                                     bc_y="periodic", limiter="weno5z")
        out[f"t{ti}_dt"] = np.array(dts)
        out[f"t{ti}_L"] = np.int64(L)
        for k in PK:
            out[f"t{ti}_prims_{k}"] = prims[k][:, 3].numpy().copy()
    np.savez_compressed(os.path.join(HERE, "tubes.npz"), **out)
    print("golden vectors written to", HERE)


def make_hllc(ref_root: str) -> None:
    """hllc.npz: the reference's hllc_flux (hlld.py:1549-1765)."""
    sys.dont_write_bytecode = True
    sys.path.insert(0, ref_root)
    import torch
    from src.physics.eos import hybrid_eos
    from src.physics.hlld import hllc_flux

    PK = ("rho", "vx", "vy", "vz", "p", "eps", "Bx", "By", "Bz")
    CK = ("D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz")
    G = 5.0 / 3.0
    eos = hybrid_eos(K=0.0, gamma=G, gamma_th=G)
    n = 512
    g = torch.Generator().manual_seed(20261203)

    def u(lo, hi):
        return torch.empty(n, dtype=torch.float64).uniform_(lo, hi, generator=g)

    def one():
        rho = 10.0 ** u(-1.0, 1.0)
        p = 10.0 ** u(-1.5, 1.0)
        W = 1.0 + 10.0 ** u(-3.0, math.log10(4.0))
        sp = torch.sqrt(1.0 - 1.0 / W**2)
        th, ph = u(0, math.pi), u(0, 2 * math.pi)
        s = {"rho": rho, "p": p, "vx": sp * torch.sin(th) * torch.cos(ph),
             "vy": sp * torch.sin(th) * torch.sin(ph), "vz": sp * torch.cos(th),
             "Bx": u(-3, 3), "By": u(-3, 3), "Bz": u(-3, 3)}
        s["eps"] = eos.eps__press_rho(s["p"], s["rho"])
        return s

    sL, sR = one(), one()
    for k in ("Bx", "By", "Bz"):
        sR[k] = sL[k].clone()
    out = {"gamma": np.float64(G)}
    for idir in (0, 1, 2):
        bk = ("Bx", "By", "Bz")[idir]
        L = {k: v.clone() for k, v in sL.items()}
        R = {k: v.clone() for k, v in sR.items()}
        L[bk][: n // 4] = 0.0
        R[bk][: n // 4] = 0.0
        for k in PK:
            out[f"{idir}_L_{k}"] = L[k].numpy()
            out[f"{idir}_R_{k}"] = R[k].numpy()
        F, U, ps = hllc_flux(L, R, eos, idir=idir)
        for k in CK:
            out[f"{idir}_F_{k}"] = F[k].numpy()
            out[f"{idir}_U_{k}"] = U[k].numpy()
        out[f"{idir}_pstar"] = ps.numpy()
    np.savez_compressed(os.path.join(HERE, "hllc.npz"), **out)
    print("hllc.npz written to", HERE)


def make_emf_hll(ref_root: str) -> None:
    """emf_hll.npz: rk_step_ct with emf_mode="hll" (driver2d.py:162-249,
    ct.py:63-96, sweep.py:106-119)."""
    sys.dont_write_bytecode = True
    os.environ.pop("RMHD_PSTAR_METHOD", None)
    sys.path.insert(0, ref_root)
    import torch
    from src.physics.driver2d import compute_dt_2d, prims_to_cons_2d, rk_step_ct, sync_state
    from src.physics.eos import hybrid_eos
    from src.physics.grid import Grid2D
    from src.physics.hlld import hlle_flux
    from src.physics.initial_data2d import b_from_potential, magnetic_rotor, orszag_tang
    from src.physics import reconstruction as rec
    from src.physics.state import EVOLVED_KEYS, State2D

    torch.set_num_threads(4)
    PK = ("rho", "vx", "vy", "vz", "p", "eps", "Bx", "By", "Bz")
    out = {}
    probs = {
        "rotor": (magnetic_rotor, (-0.5, 0.5), 5 / 3, ("outflow", "outflow"), "mc", "hlld", 16),
        "ot": (orszag_tang, (0.0, 1.0), 4 / 3, ("periodic", "periodic"), "mc", "hlld", 16),
        "ot_hlle": (orszag_tang, (0.0, 1.0), 4 / 3, ("periodic", "periodic"), "mc", "hlle", 16),
    }
    for name, (build, box, gam, bc, lim, solver, nn) in probs.items():
        e = hybrid_eos(K=0.0, gamma=gam, gamma_th=gam)
        gr = Grid2D(box[0], box[1], nn, box[0], box[1], nn, ng=rec.ghosts_needed(lim))
        prims, Az = build(gr, e)
        Bxf, Byf = b_from_potential(Az, gr.dx, gr.dy)
        for k in PK:
            out[f"{name}_init_{k}"] = prims[k].numpy().copy()
        out[f"{name}_init_Bxf"] = Bxf.numpy().copy()
        out[f"{name}_init_Byf"] = Byf.numpy().copy()
        c = prims_to_cons_2d(prims, gr)
        st = State2D(cons={k: c[k] for k in EVOLVED_KEYS}, Bxf=Bxf, Byf=Byf, prims=prims)
        st = sync_state(st, gr, e, *bc)
        kw = {"flux_fn": hlle_flux} if solver == "hlle" else {}
        dts = []
        for _ in range(2):
            dt = compute_dt_2d(st.prims, gr, e, 0.4)
            dts.append(dt)
            st, _ = rk_step_ct(st, gr, e, dt, scheme="rk3", bc_x=bc[0], bc_y=bc[1], limiter=lim,
                               emf_mode="hll", **kw)
        out[f"{name}_dt"] = np.array(dts)
        for k in EVOLVED_KEYS:
            out[f"{name}_cons_{k}"] = st.cons[k].numpy()
        for k in PK:
            out[f"{name}_prims_{k}"] = st.prims[k].numpy()
        out[f"{name}_Bxf"] = st.Bxf.numpy()
        out[f"{name}_Byf"] = st.Byf.numpy()
        out[f"{name}_meta"] = np.array([nn, rec.ghosts_needed(lim), gam, gr.dx, gr.dy])
    np.savez_compressed(os.path.join(HERE, "emf_hll.npz"), **out)
    print("emf_hll.npz written to", HERE)


def make_gradient(ref_root: str, n: int = 128, steps: int = 4) -> None:
    """rotor_gradient.npz: the reference's gradient of the config-5 objective
    on the tapered rotor at n^2 after `steps` FP64 HLLD + PLM-MC + SSP-RK3 +
    CT steps of rk_step_ct (driver2d.py:221-249, periodic), the dt sequence
    frozen: J = sum over cells of w |B_c|^2 / 2 (Gaussian w at (0.6, 0.5),
    sigma 0.1), with respect to omega and to the initial density field.

    Two estimates are recorded:
      * central differences of the reference itself: d J / d omega at
        h = 1e-5 and 1e-6, and d J / d rho0 along the eight seeded directions
        of gradient_directions at h = 1e-5 and 2e-5 (a pair that agrees
        marks a direction whose perturbed runs take the same discrete
        decisions, limiter branches, HLLD fallbacks, CT upwind signs);
      * torch autograd through the reference.  As shipped it cannot be
        differentiated: its C2P, boundary fills and sync write in place into
        tensors autograd has saved, and every torch.where whose unselected
        branch divides by a tiny number or takes the square root of 0 sends
        0 * inf = NaN into the backward pass.  Here wrappers hand the
        in-place writes fresh copies (KastaunC2P.invert / invert_bisection
        results, the arrays apply_bc_cc fills, the state sync_state fills),
        which changes no forward value, and a hook on every backward node
        sets non-finite input gradients to zero.  The result is recorded as
        it comes out; it does not agree with the central differences."""
    sys.dont_write_bytecode = True
    os.environ.pop("RMHD_PSTAR_METHOD", None)
    sys.path.insert(0, ref_root)
    import torch
    import src.physics.c2p as C
    import src.physics.driver2d as D
    import src.physics.grid as GR
    from src.physics.eos import hybrid_eos
    from src.physics.initial_data2d import b_from_potential
    from src.physics.state import EVOLVED_KEYS, State2D

    torch.set_num_threads(os.cpu_count() or 1)
    G = 5.0 / 3.0
    eos = hybrid_eos(K=0.0, gamma=G, gamma_th=G)
    g = GR.Grid2D(0.0, 1.0, n, 0.0, 1.0, n, ng=2)
    X, Y = g.X - 0.5, g.Y - 0.5
    f = ((0.115 - torch.sqrt(X * X + Y * Y)) / 0.015).clamp(0.0, 1.0)
    w = torch.exp(-((g.X - 0.6) ** 2 + (g.Y - 0.5) ** 2) / (2 * 0.1 ** 2))
    ph = g.phys
    _, YF = torch.meshgrid(g.xf, g.yf, indexing="ij")

    def run(rho, omega, dts=None):
        zero = torch.zeros_like(f)
        prims = {"rho": rho, "p": torch.ones_like(f), "vx": -omega * Y * f, "vy": omega * X * f,
                 "vz": zero, "Bx": torch.ones_like(f), "By": zero.clone(), "Bz": zero.clone()}
        prims["eps"] = eos.eps__press_rho(prims["p"], prims["rho"])
        Bxf, Byf = b_from_potential(YF.clone(), g.dx, g.dy)
        c = D.prims_to_cons_2d(prims, g)
        st = State2D(cons={k: c[k] for k in EVOLVED_KEYS}, Bxf=Bxf, Byf=Byf, prims=prims)
        st = D.sync_state(st, g, eos, "periodic", "periodic")
        out = []
        for k in range(steps):
            if dts is None:
                with torch.no_grad():
                    dt = D.compute_dt_2d({q: v.detach() for q, v in st.prims.items()}, g, eos, 0.4)
            else:
                dt = dts[k]
            out.append(dt)
            st, _ = D.rk_step_ct(st, g, eos, dt, scheme="rk3", bc_x="periodic", bc_y="periodic")
        B2 = st.prims["Bx"] ** 2 + st.prims["By"] ** 2 + st.prims["Bz"] ** 2
        return (w[ph] * B2[ph]).sum() / 2, out

    sys.path.insert(0, os.path.dirname(HERE))
    from helpers import gradient_directions

    rho_base = 1.0 + 9.0 * f
    with torch.no_grad():
        J0, dts = run(rho_base, 9.95)
        fd_omega = [float((run(rho_base, 9.95 + h, dts)[0] - run(rho_base, 9.95 - h, dts)[0])
                          / (2 * h)) for h in (1e-5, 1e-6)]
        fd_dir = np.zeros((8, 2))
        full = torch.zeros_like(f)
        for k in range(8):
            dirn = full.clone()
            dirn[ph] = gradient_directions(X[ph], Y[ph], k)
            for j, h in enumerate((1e-5, 2e-5)):
                fd_dir[k, j] = float((run(rho_base + h * dirn, 9.95, dts)[0]
                                      - run(rho_base - h * dirn, 9.95, dts)[0]) / (2 * h))
            print("direction", k, fd_dir[k], flush=True)

    # torch autograd through the reference, shimmed as described above
    inv, bis = C.KastaunC2P.invert, C.KastaunC2P.invert_bisection
    C.KastaunC2P.invert = lambda self, *a, **k: {q: v.clone() for q, v in inv(self, *a, **k).items()}
    C.KastaunC2P.invert_bisection = lambda self, *a, **k: {q: v.clone()
                                                           for q, v in bis(self, *a, **k).items()}
    bc_cc = GR.Grid2D.apply_bc_cc

    def fresh_bc_cc(self, U, *a, **k):
        for q in list(U):
            U[q] = U[q].clone()
        return bc_cc(self, U, *a, **k)

    GR.Grid2D.apply_bc_cc = fresh_bc_cc
    sync = D.sync_state

    def fresh_sync(state, *a, **k):
        state.Bxf, state.Byf = state.Bxf.clone(), state.Byf.clone()
        state.cons = {q: v.clone() for q, v in state.cons.items()}
        return sync(state, *a, **k)

    D.sync_state = fresh_sync
    rho0 = rho_base.clone().requires_grad_(True)
    omega = torch.tensor(9.95, dtype=torch.float64, requires_grad=True)
    J, _ = run(rho0, omega, dts)

    def finite(grad_inputs, grad_outputs):
        return tuple(None if x is None else torch.nan_to_num(x, nan=0.0, posinf=0.0, neginf=0.0)
                     for x in grad_inputs)

    seen, todo = set(), [J.grad_fn]
    while todo:
        node = todo.pop()
        if node is None or node in seen:
            continue
        seen.add(node)
        node.register_hook(finite)
        todo.extend(nx for nx, _ in node.next_functions)
    J.backward()
    np.savez_compressed(os.path.join(HERE, "rotor_gradient.npz"), n=n, steps=steps,
                        dts=np.array(dts), J=float(J0), fd_omega=np.array(fd_omega),
                        fd_h_omega=np.array([1e-5, 1e-6]), fd_dir=fd_dir,
                        fd_h_dir=np.array([1e-5, 2e-5]),
                        autograd_omega=float(omega.grad), autograd_rho0=rho0.grad[ph].numpy())
    print("rotor_gradient.npz written to", HERE, "J", float(J0), "FD dJ/domega", fd_omega,
          "autograd", float(omega.grad))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_CHECKOUT "
                 "[hllc | emf_hll | gradient N STEPS]")
    root = sys.argv[1]
    if len(sys.argv) > 2 and sys.argv[2] == "hllc":
        make_hllc(root)
    elif len(sys.argv) > 2 and sys.argv[2] == "emf_hll":
        make_emf_hll(root)
    elif len(sys.argv) > 2 and sys.argv[2] == "gradient":
        make_gradient(root, *(int(x) for x in sys.argv[3:5]))
    else:
        main(root)
        make_hllc(root)
        make_emf_hll(root)
