"""Generate the golden vectors under tests/golden/ by running the reference's
own CPU code (oracle/_ref/libstokesdt_ref.so, built from the unmodified
reference sources by oracle/Makefile) on the reference's own test geometries
(tests/data/*.xyz of the reference project) and on the synthetic config-1
geometry.  Needs the reference tree, so it runs in the build container only;
the GPU tests read the committed .npz files.

    python tests/golden/make_golden.py [--ref /root/reference]

Cases (reference test that each one follows):
  spme_N1000_K256_p6  tests/spme/test.sh:2-3   MobSpme vs MobEwald, 3 RHS, alpha 2.1 beta 1.1
  spme_N1000_K256_p8  tests/spme/test.sh:5-6
  spme_N412_poly      tests/spme/test.sh:8-9   polydisperse radii from poly.mod
  spme_N1000_K64      same geometry at the config-1 grid (K=64, p=6, xi=0.5, rmax=8)
  spme_N3             N3_Phi0.1.xyz, K=32, p=6 (tiny case)
  spme_cfg1           synthetic config 1: RSA N=1000 phi=0.1, K=64, p=6, xi=0.30
  lanczos_N1000       tests/lanczos/testlanczos.cc:81-148: BrwnLanczos on MobEwald,
                      1 and 3 RHS, plus the dense symmetric square root
  steric_N412_poly    StericForce (r0 2.5, k0 125) on N412.xyz + poly.mod radii
  steric_cfg3         StericForce (r0 2, k0 125 as data/example.mod) on a config-3-like
                      system: RSA N=2000 phi=0.3, jittered
  bd_cfg3_traj        config 3 (N=2e4, phi=0.3, K=128, steric): the first 10 BD steps composed
                      from the reference's MobSpme, BrwnLanczos and StericForce (--bd only)
  bd_cfg3_traj_tight  the same with Lanczos tol 1e-8, max_iters 200 (--bd-tight only)
  lanczos_cfg2_proj   config 2 at full size (N=1e5, K=256, p=6, xi=0.35): BrwnLanczos
                      (tol 1e-6, max_iters 100, 16 RHS) on the reference's MobSpme;
                      the iteration count and 64 random projections of the first two
                      Brownian vectors (--cfg2 only: ~15 minutes on 8 cores)
  batch_sys6          6 autotuned batch systems (N in [300, 3000]): MobSpme MulVector on 3 RHS
                      (alpha 0.8, beta 0.5) per system (--batch only)
  mf_cfg2_proj        config 2 at full size: MobSpme MulVector / RealMulVector /
                      RecipMulVector on 4 RHS (alpha 1.3, beta 0.7); 64 random projections,
                      norms and the first 512 particles' outputs per mode (--mf-cfg2 only)
Random inputs come from numpy's PCG64 with fixed seeds (the reference's MKL
VSL stream cannot be reproduced here).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from oracle import spme_oracle as so  # noqa: E402

ALPHA, BETA = 2.1, 1.1


def spme_case(name, pos, rdi, L, K, p, xi, rmax, seed, nrhs=3, ewald=True):
    N = len(rdi)
    n3 = 3 * N
    ld = ref.pad_len(n3)
    rng = np.random.default_rng(seed)
    f = np.zeros((nrhs, ld))
    f[:, :n3] = rng.uniform(0.0, 1.0, (nrhs, n3))
    sp = ref.RefMob.spme(rdi, L, xi, rmax, K, p)
    sp.update(pos, rdi)
    out = {}
    for mode, key in ((0, "v_full"), (1, "v_real"), (2, "v_recip")):
        out[key] = sp.mulvec(f, ALPHA, BETA, f.copy(), mode=mode)[:, :n3]
    if ewald:
        ew = ref.RefMob.ewald(rdi, L, 1e-12)
        ew.update(pos, rdi)
        out["v_ewald"] = ew.mulvec(f, ALPHA, BETA, f.copy())[:, :n3]
        err = np.linalg.norm(out["v_ewald"] - out["v_full"]) / np.linalg.norm(out["v_ewald"])
        out["err_spme_vs_ewald"] = np.array(err)
        print(f"{name}: reference SPME vs dense Ewald error {err:.3e}")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), pos=pos, rdi=rdi, box=np.array(L),
                        K=np.array(K), p=np.array(p), xi=np.array(xi), rmax=np.array(rmax),
                        alpha=np.array(ALPHA), beta=np.array(BETA), f=f[:, :n3], **out)


def lanczos_case(name, pos, rdi, L, seed):
    N = len(rdi)
    n3 = 3 * N
    ld = ref.pad_len(n3)
    ew = ref.RefMob.ewald(rdi, L, 1e-12)
    ew.update(pos, rdi)
    M = ew.matrix()
    w, V = np.linalg.eigh(M)
    S = (V * np.sqrt(w)) @ V.T
    rng = np.random.default_rng(seed)
    z = np.zeros((3, ld))
    z[:, :n3] = rng.uniform(0.0, 1.0, (3, n3))
    lz = ref.RefLanczos(n3, 100, 16, 1e-7)
    y1, it1 = lz.compute(ew, z[:1])
    y3, it3 = lz.compute(ew, z[:3])
    # iteration counts at tol 1e-5, where the FP32 rounding of a mobility
    # product is far below the convergence increments
    lz5 = ref.RefLanczos(n3, 100, 16, 1e-5)
    _, it1_5 = lz5.compute(ew, z[:1])
    _, it3_5 = lz5.compute(ew, z[:3])
    y0 = (S @ z[:, :n3].T).T
    e1 = np.linalg.norm(y1[:, :n3] - y0[:1]) / np.linalg.norm(y0[:1])
    e3 = np.linalg.norm(y3[:, :n3] - y0) / np.linalg.norm(y0)
    print(f"{name}: reference Lanczos errors 1-RHS {e1:.3e} ({it1}) 3-RHS {e3:.3e} ({it3})")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), pos=pos, rdi=rdi, box=np.array(L),
                        z=z[:, :n3], y_ref1=y1[:, :n3], y_ref3=y3[:, :n3], y_sqrt=y0,
                        iters1=np.array(it1), iters3=np.array(it3), iters1_tol5=np.array(it1_5),
                        iters3_tol5=np.array(it3_5))


def steric_case(name, pos, rdi, L, r0, k0, seed):
    """StericForce::Accumulate (src/force/force_steric.cc:91-104) on f0."""
    N = len(rdi)
    f0 = np.random.default_rng(seed).standard_normal(3 * N)
    st = ref.RefSteric(rdi, L, r0, k0)
    f = st.accumulate(pos, f0)
    npairs = int(np.count_nonzero(np.abs(f - f0) > 0) // 3)
    print(f"{name}: {npairs} particles with steric contacts")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), pos=pos, rdi=rdi, box=np.array(L),
                        r0=np.array(r0), k0=np.array(k0), f0=f0, f=f)


def steric_cases(refdir):
    data = os.path.join(refdir, "tests", "data")
    radii = ref.parse_mod(os.path.join(data, "poly.mod"))
    ppos, prdi, pL = ref.parse_xyz(os.path.join(data, "N412.xyz"), radii)
    # r0 2.5: the reference geometry has no pair closer than (a_i + a_j)
    steric_case("steric_N412_poly", ppos, prdi, pL, 2.5, 125.0, 7)
    # config-3-like: RSA at phi = 0.3 (minimum separation 2a) jittered so that
    # pairs come closer than the steric cutoff r0 (a_i + a_j)/2 = 2
    N = 2000
    L = so.box_for(N, 0.3)
    pos = so.rsa_positions(N, L, 21) + np.random.default_rng(22).normal(0.0, 0.08, (N, 3))
    steric_case("steric_cfg3", pos, np.ones(N), L, 2.0, 125.0, 23)


def bd_cfg3_case(name, nsteps=10, tol=None, max_iters=None):
    """Config 3, first `nsteps` steps of BDSimBox::Advance
    (src/simbox/simbox_bd.cc:296-366) composed from the reference's own
    MobSpme, BrwnLanczos (1 RHS per step, tol 1e-5) and StericForce, FP64,
    driven by the random vectors of the device integrator (numpy restatement
    of its Philox4x32-10 + Box-Muller draw, counter = (pair, step)).  The
    reference's SPME indexes out of bounds for positions outside [0, L)
    (src/mob/spme.cc:404-417), so it is given wrapped positions; the physics
    is periodic, so this changes nothing else.  Stores 64 random projections
    and the norm of pos(k) - pos(0) after every step."""
    from stokesdt_b200 import workloads as wl
    w = wl.WORKLOADS["cfg3"]
    N, n3, L = w.npos, 3 * w.npos, w.box
    rdi = np.ones(N)
    pos0 = wl.rsa_positions(N, L, w.seed_pos).reshape(-1)
    sp = ref.RefMob.spme(rdi, L, w.xi, w.rmax, w.dim, w.porder)
    tol = w.lanczos_tol if tol is None else tol
    lz = ref.RefLanczos(n3, max_iters or w.max_iters, 1, tol)
    st = ref.RefSteric(rdi, L, w.steric_r0, w.steric_k0)
    P = cfg2_projector(n3, seed=CFG2_PROJ_SEED + 3)
    pos = pos0.copy()
    proj, norms, iters = [], [], []
    for k in range(nsteps):
        wrapped = np.mod(pos, L)
        z = so.bd_gaussian(w.seed_z, k, 1, n3)
        sp.update(wrapped, rdi)
        y, its = lz.compute(sp, z)
        f = st.accumulate(wrapped, np.zeros(n3))
        disp = sp.mulvec(f[None, :], w.dt, np.sqrt(2.0 * w.dt), y)[0, :n3]
        pos = pos + disp
        d = pos - pos0
        proj.append(P.astype(np.float64) @ d)
        norms.append(np.linalg.norm(d))
        iters.append(its[0])
        print(f"{name}: step {k + 1}, |pos - pos0| {norms[-1]:.6f}, Lanczos iterations {its[0]}")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), proj=np.array(proj), norms=np.array(norms),
                        iters=np.array(iters), seed_proj=np.array(CFG2_PROJ_SEED + 3),
                        nsteps=np.array(nsteps), tol=np.array(tol))


# Dense-Ewald trajectory: a small suspension on the reference driver's
# default mobility (mob-method ewald) with Lanczos, 4 RHS per interval; 3N is
# a multiple of 8 (the reference's PadLen), so the random block needs no
# padding.
BD_EWALD = dict(npos=304, phi=0.2, seed_pos=17, seed_z=31, dt=1e-3, interval=4, nsteps=8, ewald_tol=1e-4,
                lanczos_tol=1e-8, max_iters=100, steric_r0=2.0, steric_k0=125.0)


def bd_ewald_case(name):
    """First BD_EWALD["nsteps"] steps of BDSimBox::Advance
    (src/simbox/simbox_bd.cc:296-366) with the reference's MobEwald
    (ewald-tol 1e-4, default xi), BrwnLanczos (4 RHS every 4 steps, tol
    1e-8) and StericForce, FP64, driven by the device integrator's random
    vectors (numpy restatement of its Philox4x32-10 + Box-Muller draw).
    Stores pos(k) - pos(0) after every step."""
    from stokesdt_b200 import workloads as wl
    c = BD_EWALD
    N, n3 = c["npos"], 3 * c["npos"]
    L = wl.box_for(N, c["phi"])
    rdi = np.ones(N)
    pos0 = wl.rsa_positions(N, L, c["seed_pos"]).reshape(-1)
    ew = ref.RefMob.ewald(rdi, L, tol=c["ewald_tol"])
    lz = ref.RefLanczos(n3, c["max_iters"], c["interval"], c["lanczos_tol"])
    st = ref.RefSteric(rdi, L, c["steric_r0"], c["steric_k0"])
    pos = pos0.copy()
    disp_all, iters = [], []
    y = None
    for k in range(c["nsteps"]):
        irhs = k % c["interval"]
        if irhs == 0:
            z = so.bd_gaussian(c["seed_z"], k, c["interval"], n3)
            ew.update(pos, rdi)
            y, its = lz.compute(ew, z)
            iters.append(its[0])
        f = st.accumulate(np.mod(pos, L), np.zeros(n3))
        disp = ew.mulvec(f[None, :], c["dt"], np.sqrt(2.0 * c["dt"]), y[irhs][None, :])[0, :n3]
        pos = pos + disp
        disp_all.append(pos - pos0)
        print(f"{name}: step {k + 1}, |pos - pos0| {np.linalg.norm(pos - pos0):.6f}")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), d=np.array(disp_all), iters=np.array(iters),
                        box=np.array(L), **{k: np.array(v) for k, v in c.items()})


CFG2_PROJ_SEED, CFG2_NPROJ = 2024, 64


def cfg2_projector(n3, seed=CFG2_PROJ_SEED, nproj=CFG2_NPROJ):
    """Fixed Gaussian projection rows (nproj x n3) / sqrt(n3), FP32."""
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((nproj, n3), dtype=np.float32) / np.sqrt(n3)).astype(np.float32)


def lanczos_cfg2_case(name):
    """The reference's block Lanczos keeps (max_iters+1)^2 nrhs^2 doubles on
    the stack (src/brwn/brwn_lanczos.cc:97): 21 MB here, so it runs on a
    thread with a 256 MB stack."""
    import threading
    from stokesdt_b200 import workloads as wl
    w = wl.WORKLOADS["cfg2"]
    N, n3 = w.npos, 3 * w.npos
    pos = wl.rsa_positions(N, w.box, w.seed_pos)
    rdi = np.ones(N)
    z = np.random.default_rng(w.seed_z).standard_normal((w.nrhs, n3))
    out = {}

    def run():
        sp = ref.RefMob.spme(rdi, w.box, w.xi, w.rmax, w.dim, w.porder)
        sp.update(pos, rdi)
        lz = ref.RefLanczos(n3, w.max_iters, w.nrhs, w.lanczos_tol)
        out["y"], out["its"] = lz.compute(sp, z)

    threading.stack_size(256 << 20)
    th = threading.Thread(target=run)
    th.start()
    th.join()
    y = out["y"][:2, :n3]
    P = cfg2_projector(n3)
    proj = (P.astype(np.float64) @ y.T).T
    print(f"{name}: reference iterations {out['its']}, |y0| {np.linalg.norm(y[0]):.6f}")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), iters=np.array(out["its"]), proj=proj,
                        norms=np.linalg.norm(y, axis=1), tol=np.array(w.lanczos_tol),
                        seed_proj=np.array(CFG2_PROJ_SEED))


MF_CFG2_NRHS, MF_CFG2_HEAD = 4, 512
MF_CFG2_ALPHA, MF_CFG2_BETA = 1.3, 0.7


def mf_cfg2_inputs(n3):
    """Forces F (4 x 3N) and the initial v (4 x 3N, scaled by beta) of the
    config-2 mobility-product fixture, seeded."""
    rng = np.random.default_rng(9012)
    return rng.standard_normal((MF_CFG2_NRHS, n3)), rng.standard_normal((MF_CFG2_NRHS, n3))


def mf_cfg2_case(name):
    """Config 2 at full size (N=1e5, phi=0.2, K=256, p=6, xi=0.35, rmax from
    the tol-1e-6 rule): the reference's MobSpme MulVector (mode 0),
    RealMulVector (1) and RecipMulVector (2) (src/mob/mob_spme.cc:219-263,
    src/mob/spme.cc:714-839) on 4 RHS with alpha 1.3, beta 0.7.  Stores per
    mode 64 fixed random projections of every output vector, their norms and
    the outputs of the first 512 particles in full (~4 minutes on 8 cores)."""
    from stokesdt_b200 import workloads as wl
    w = wl.WORKLOADS["cfg2"]
    N, n3 = w.npos, 3 * w.npos
    pos = wl.rsa_positions(N, w.box, w.seed_pos)
    rdi = np.ones(N)
    F, V0 = mf_cfg2_inputs(n3)
    sp = ref.RefMob.spme(rdi, w.box, w.xi, w.rmax, w.dim, w.porder)
    sp.update(pos, rdi)
    P = cfg2_projector(n3, seed=CFG2_PROJ_SEED + 7).astype(np.float64)
    out = {}
    for mode in (0, 1, 2):
        v = sp.mulvec(F, MF_CFG2_ALPHA, MF_CFG2_BETA, V0.copy(), mode=mode)
        out[f"proj{mode}"] = (P @ v.T).T
        out[f"norms{mode}"] = np.linalg.norm(v, axis=1)
        out[f"head{mode}"] = v[:, :3 * MF_CFG2_HEAD].copy()
        print(f"{name}: mode {mode}, |v| {out[f'norms{mode}']}")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), seed_proj=np.array(CFG2_PROJ_SEED + 7),
                        alpha=np.array(MF_CFG2_ALPHA), beta=np.array(MF_CFG2_BETA),
                        head=np.array(MF_CFG2_HEAD), **out)


def batch_sys_case(name):
    """Config-4-style batch (6 systems, N log-uniform in [300, 3000], grid and
    Ewald split by the autotuner, seed 8): the reference's MobSpme MulVector
    (alpha 0.8, beta 0.5, 3 RHS) for each system, so a packed batch product is
    checked against the reference on every system."""
    from stokesdt_b200 import workloads as wl
    sy = wl.batch_systems(nsys=6, seed=8, nmin=300, nmax=3000)
    out = {}
    for s, d in enumerate(sy):
        N, n3 = d["npos"], 3 * d["npos"]
        pos = wl.rsa_positions(N, d["box"], d["seed"])
        rng = np.random.default_rng(500 + s)
        f = rng.standard_normal((3, n3))
        v0 = rng.standard_normal((3, n3))
        sp = ref.RefMob.spme(np.ones(N), d["box"], d["xi"], d["rmax"], d["K"], 6)
        sp.update(pos, np.ones(N))
        out[f"f{s}"] = f
        out[f"v0_{s}"] = v0
        out[f"v{s}"] = sp.mulvec(f, 0.8, 0.5, v0.copy())
        print(f"{name}: system {s} N={N} K={d['K']}")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), nsys=np.array(len(sy)), alpha=np.array(0.8),
                        beta=np.array(0.5), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--cfg2", action="store_true", help="only the config-2 Lanczos fixture")
    ap.add_argument("--mf-cfg2", action="store_true", help="only the config-2 mobility-product fixture")
    ap.add_argument("--batch", action="store_true", help="only the batch-systems fixture")
    ap.add_argument("--lanczos", action="store_true", help="only the N1000 Lanczos fixture")
    ap.add_argument("--steric", action="store_true", help="only the steric-force fixtures")
    ap.add_argument("--bd", action="store_true", help="only the config-3 trajectory fixture")
    ap.add_argument("--bd-tight", action="store_true",
                    help="only the config-3 trajectory fixture at Lanczos tol 1e-8")
    ap.add_argument("--bd-ewald", action="store_true", help="only the dense-Ewald trajectory fixture")
    a = ap.parse_args()
    if a.bd_ewald:
        bd_ewald_case("bd_ewald_traj")
        return
    if a.bd:
        bd_cfg3_case("bd_cfg3_traj")
        return
    if a.bd_tight:
        bd_cfg3_case("bd_cfg3_traj_tight", tol=1e-8, max_iters=200)
        return
    if a.steric:
        steric_cases(a.ref)
        return
    if a.cfg2:
        lanczos_cfg2_case("lanczos_cfg2_proj")
        return
    if a.mf_cfg2:
        mf_cfg2_case("mf_cfg2_proj")
        return
    if a.batch:
        batch_sys_case("batch_sys6")
        return
    if a.lanczos:
        pos, rdi, L = ref.parse_xyz(os.path.join(a.ref, "tests", "data", "N1000_Phi0.1.xyz"))
        lanczos_case("lanczos_N1000", pos, rdi, L, 1234)
        return
    data = os.path.join(a.ref, "tests", "data")
    pos, rdi, L = ref.parse_xyz(os.path.join(data, "N1000_Phi0.1.xyz"))
    spme_case("spme_N1000_K256_p6", pos, rdi, L, 256, 6, 0.8, 8.371887, 1234)
    spme_case("spme_N1000_K256_p8", pos, rdi, L, 256, 8, 0.8, 8.371887, 1234)
    spme_case("spme_N1000_K64", pos, rdi, L, 64, 6, 0.5, 8.0, 99, nrhs=2, ewald=False)
    radii = ref.parse_mod(os.path.join(data, "poly.mod"))
    ppos, prdi, pL = ref.parse_xyz(os.path.join(data, "N412.xyz"), radii)
    spme_case("spme_N412_poly", ppos, prdi, pL, 256, 8, 0.04, 200.37188, 1234)
    tpos, trdi, tL = ref.parse_xyz(os.path.join(data, "N3_Phi0.1.xyz"))
    # rmax < L/2 = 2.50 and 4p <= K
    spme_case("spme_N3", tpos, trdi, tL, 32, 6, 1.2, 2.45, 5, nrhs=2)
    N = 1000
    cL = so.box_for(N, 0.1)
    cpos = so.rsa_positions(N, cL, 1)
    spme_case("spme_cfg1", cpos, np.ones(N), cL, 64, 6, 0.30, so.xi_to_rmax(0.30, 1e-6, cL), 2)
    lanczos_case("lanczos_N1000", pos, rdi, L, 1234)
    steric_cases(a.ref)


if __name__ == "__main__":
    main()
