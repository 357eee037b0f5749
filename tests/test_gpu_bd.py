"""Device-resident BD integrator (BDSimBox::Advance step loop,
src/simbox/simbox_bd.cc:296-366) against a host composition of the oracle
pieces: the same random vectors (numpy restatement of the Philox4x32-10 +
Box-Muller draw), the FP64 oracle SPME and block Lanczos, and the steric
oracle.  Tolerance: 1e-5 relative on the displacement (the sqrt(M) z bound)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _system(N=300, phi=0.2, K=32, seed=4):
    from oracle import spme_oracle as so
    L = so.box_for(N, phi)
    pos = so.rsa_positions(N, L, seed) + np.random.default_rng(seed + 1).normal(0.0, 0.05, (N, 3))
    xi = 0.5
    rmax = min(so.xi_to_rmax(xi, 1e-6, L), 0.49 * L)
    return pos, L, xi, rmax, K


def test_gaussian_draw_matches_restatement(gpu_available):
    import stokesdt_b200 as sdt
    from oracle import spme_oracle as so
    pos, L, xi, rmax, K = _system()
    N = len(pos)
    m = sdt.MobSpme(N, np.ones(N), L, xi, rmax, K, 6)
    assert m.Init()
    lz = sdt.BrwnLanczos(3 * N, 50, 4, 1e-6)
    assert lz.Init()
    bd = sdt.BDIntegrator(m, lz, None, dt=1e-3, mob_interval=4, seed=987654321012)
    for step in (0, 4, 2 ** 33 + 4):
        z = bd.draw_gaussian(step, 3)
        zr = so.bd_gaussian(987654321012, step, 3, 3 * N)
        assert np.max(np.abs(z - zr)) < 1e-12
    z0, z1 = bd.draw_gaussian(0, 3), bd.draw_gaussian(4, 3)
    assert abs(z0.mean()) < 0.05 and abs(z0.std() - 1.0) < 0.05
    assert abs(np.corrcoef(z0.ravel(), z1.ravel())[0, 1]) < 0.03


def test_one_interval_matches_oracle_composition(gpu_available):
    import stokesdt_b200 as sdt
    from oracle import spme_oracle as so
    pos, L, xi, rmax, K = _system()
    N = len(pos)
    n3 = 3 * N
    dt, interval, seed, r0, k0 = 1e-3, 4, 42, 2.0, 125.0
    m = sdt.MobSpme(N, np.ones(N), L, xi, rmax, K, 6)
    assert m.Init()
    lz = sdt.BrwnLanczos(n3, 80, 4, 1e-9, reorth=True)
    assert lz.Init()
    st = sdt.StericForce(N, np.ones(N), L, r0, k0)
    assert st.Init()
    bd = sdt.BDIntegrator(m, lz, st, dt=dt, mob_interval=interval, seed=seed)
    bd.set_positions(pos)
    # host composition of the same interval
    o = so.SpmeOracle(np.ones(N), L, xi, rmax, K, 6)
    o.update(pos)
    Z = so.bd_gaussian(seed, 0, interval, n3)
    Y, _ = so.block_lanczos_sqrt(lambda X: o.mulvec(X.T).T, Z.T, 80, 1e-9)
    Y = Y.T
    p = pos.reshape(-1).copy()
    traj = []
    for k in range(interval):
        f = so.steric_force(p, np.ones(N), L, r0, k0)
        disp = dt * o.mulvec(f[None, :])[0] + np.sqrt(2.0 * dt) * Y[k]
        p = p + disp
        traj.append(p.copy())
    got = []
    for k in range(interval):
        bd.Advance(1)
        got.append(bd.get_positions())
    for k in range(interval):
        d_ref = traj[k] - pos.reshape(-1)
        d_got = got[k] - pos.reshape(-1)
        assert rel_err(d_ref, d_got) < 1e-5, k
    info = bd.info()
    assert info["istep"] == interval and info["not_converged"] == 0 and info["last_iters"] > 0
    # the next interval starts a new Update + Lanczos at the moved positions
    bd.Advance(1)
    assert bd.info()["istep"] == interval + 1


def test_restart_step_and_determinism(gpu_available):
    import stokesdt_b200 as sdt
    pos, L, xi, rmax, K = _system(N=200)
    N = len(pos)
    runs = []
    for _ in range(2):
        m = sdt.MobSpme(N, np.ones(N), L, xi, rmax, K, 6)
        assert m.Init()
        lz = sdt.BrwnLanczos(3 * N, 60, 2, 1e-6, reorth=True)
        assert lz.Init()
        bd = sdt.BDIntegrator(m, lz, None, dt=1e-3, mob_interval=2, seed=5)
        bd.set_positions(pos)
        bd.set_step(6)  # resume: a new interval starts at step 6
        bd.Advance(3)
        runs.append(bd.get_positions())
        assert bd.info()["istep"] == 9
    # same seed and step: the same random vectors; the FP32 products differ
    # only by summation order
    assert rel_err(runs[0] - pos.reshape(-1), runs[1] - pos.reshape(-1)) < 1e-5


def test_config3_first_ten_steps_vs_reference_trajectory(gpu_available):
    """Config 3 (N=20,000, phi=0.3, K=128, steric r0=2 k0=125, dt=1e-3,
    1 RHS per step, Lanczos tol 1e-5): the first 10 steps of the device
    integrator against the FP64 trajectory the reference's own MobSpme,
    BrwnLanczos and StericForce produce from the same random vectors
    (tests/golden/bd_cfg3_traj.npz: 64 projections of pos(k) - pos(0)).
    Both Lanczos runs stop at tol 1e-5, so the bar is 1e-4 relative per step."""
    _config3_vs_reference("bd_cfg3_traj", None, None, 1e-4)


def test_config3_first_ten_steps_tight_tolerance(gpu_available):
    """The same trajectory with both Lanczos runs at tol 1e-8 (max_iters 200;
    tests/golden/bd_cfg3_traj_tight.npz): the iterates are converged far
    below the sqrt(M) z bar, so the trajectory is held to 1e-5 relative per
    step."""
    _config3_vs_reference("bd_cfg3_traj_tight", 1e-8, 200, 1e-5)


def _config3_vs_reference(name, tol, max_iters, bar):
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl
    from conftest import golden
    g = golden(name)
    w = wl.WORKLOADS["cfg3"]
    N, n3 = w.npos, 3 * w.npos
    pos0 = wl.rsa_positions(N, w.box, w.seed_pos).reshape(-1)
    m = sdt.MobSpme(N, np.ones(N), w.box, w.xi, w.rmax, w.dim, w.porder)
    assert m.Init()
    lz = sdt.BrwnLanczos(n3, max_iters or w.max_iters, 1, tol or w.lanczos_tol, reorth=True)
    assert lz.Init()
    st = sdt.StericForce(N, np.ones(N), w.box, w.steric_r0, w.steric_k0)
    assert st.Init()
    bd = sdt.BDIntegrator(m, lz, st, dt=w.dt, mob_interval=w.mob_interval, seed=w.seed_z)
    bd.set_positions(pos0)
    rng = np.random.default_rng(int(g["seed_proj"]))
    P = (rng.standard_normal((g["proj"].shape[1], n3), dtype=np.float32) / np.sqrt(n3)).astype(np.float32)
    worst = 0.0
    for k in range(int(g["nsteps"])):
        bd.Advance(1)
        d = bd.get_positions() - pos0
        pk = P.astype(np.float64) @ d
        worst = max(worst, float(np.linalg.norm(pk - g["proj"][k]) / np.linalg.norm(g["proj"][k])))
        assert abs(np.linalg.norm(d) / g["norms"][k] - 1.0) < bar, k
    assert worst < bar, worst
    assert bd.info()["not_converged"] == 0


def test_dense_ewald_trajectory_vs_reference(gpu_available):
    """The integrator on the dense Ewald mobility (the reference driver's
    default mob-method): N=304, phi=0.2, ewald-tol 1e-4, 4 RHS per interval,
    Lanczos tol 1e-8, steric r0=2 k0=125, 8 steps, against the FP64
    trajectory the reference's own MobEwald, BrwnLanczos and StericForce
    produce from the same random vectors (tests/golden/bd_ewald_traj.npz).
    Everything is FP64 and the Lanczos iterates are converged far below the
    bar: 1e-6 relative on pos(k) - pos(0) per step."""
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl
    from conftest import golden
    g = golden("bd_ewald_traj")
    N, L = int(g["npos"]), float(g["box"])
    n3 = 3 * N
    pos0 = wl.rsa_positions(N, L, int(g["seed_pos"])).reshape(-1)
    m = sdt.MobEwald(N, np.ones(N), L, float(g["ewald_tol"]))
    assert m.Init(), m.last_error
    lz = sdt.BrwnLanczos(n3, int(g["max_iters"]), int(g["interval"]), float(g["lanczos_tol"]), reorth=True)
    assert lz.Init()
    st = sdt.StericForce(N, np.ones(N), L, float(g["steric_r0"]), float(g["steric_k0"]))
    assert st.Init()
    bd = sdt.BDIntegrator(m, lz, st, dt=float(g["dt"]), mob_interval=int(g["interval"]), seed=int(g["seed_z"]))
    bd.set_positions(pos0)
    for k in range(int(g["nsteps"])):
        bd.Advance(1)
        d = bd.get_positions() - pos0
        assert rel_err(g["d"][k], d) < 1e-6, k
    assert bd.info()["not_converged"] == 0
