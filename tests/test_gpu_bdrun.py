"""The bdrun driver (command line and input files of the reference's
bin/main): a short run with steric repulsion writes trajectory frames in
the reference's XYZ layout."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_bdrun_short_trajectory(gpu_available, tmp_path):
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl
    N = 400
    L = wl.box_for(N, 0.2)
    pos = wl.rsa_positions(N, L, 3)
    sdt.write_xyz(tmp_path / "start.xyz", pos, L)
    K, xi, rmax = wl.autotune_system(N, 0.2)
    (tmp_path / "run.cfg").write_text(
        f"delta-t 0.001\nmob-method spme-gpu\nbrownian-method lanczos-gpu\nmob-interval 4\n"
        f"spme-nfft-grids {K}\nspme-porder 6\nspme-xi {xi}\nspme-rmax {rmax}\nlanczos-maxiters 100\n"
        f"lanczos-maxnrhs 4\nlanczos-tol 1e-5\ntraj-interval 2\ntraj-output {tmp_path / 'traj.xyz'}\n")
    (tmp_path / "run.mod").write_text("par N 1.0 0.0\nsteric 2.0 125.0\n")
    exe = os.path.join(ROOT, "stokesdt_b200", "bdrun")
    res = subprocess.run([exe, "--config", str(tmp_path / "run.cfg"), "--model", str(tmp_path / "run.mod"),
                          "--xyz", str(tmp_path / "start.xyz"), "-n", "8"], capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    lines = (tmp_path / "traj.xyz").read_text().splitlines()
    assert len(lines) == 4 * (N + 2)                # frames at steps 2, 4, 6, 8
    last = np.array([[float(v) for v in l.split()[1:]] for l in lines[-N:]])
    d = last - pos
    assert np.all(np.isfinite(d)) and 0.0 < np.abs(d).max() < 2.0
    assert lines[-N - 1].split()[0] == "8"


def test_bdrun_config3_first_steps_vs_reference_trajectory(gpu_available, tmp_path):
    """bdrun with the config-3 run (N=20,000, phi=0.3, K=128, p=6, steric
    r0=2 k0=125, dt=1e-3, mob-interval 1, Lanczos tol 1e-5, seed 22): its
    trajectory frames for steps 1..10 against the FP64 trajectory the
    reference's own MobSpme, BrwnLanczos and StericForce produce from the same
    random vectors (tests/golden/bd_cfg3_traj.npz, BDSimBox::Advance,
    src/simbox/simbox_bd.cc:296-366 of the reference).  Both Lanczos runs stop
    at tol 1e-5: bar 1e-4 relative on the displacement per step."""
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl
    from conftest import golden
    g = golden("bd_cfg3_traj")
    w = wl.WORKLOADS["cfg3"]
    N, n3 = w.npos, 3 * w.npos
    pos0 = wl.rsa_positions(N, w.box, w.seed_pos)
    sdt.write_xyz(tmp_path / "start.xyz", pos0, w.box)
    nsteps = int(g["nsteps"])
    (tmp_path / "run.cfg").write_text(
        f"delta-t {w.dt}\nmob-method spme-gpu\nbrownian-method lanczos-gpu\nmob-interval 1\n"
        f"spme-nfft-grids {w.dim}\nspme-porder {w.porder}\nspme-xi {w.xi!r}\nspme-rmax {w.rmax!r}\n"
        f"lanczos-maxiters {w.max_iters}\nlanczos-maxnrhs 1\nlanczos-tol {w.lanczos_tol}\n"
        f"traj-startstep 0\ntraj-interval 1\ntraj-output {tmp_path / 'traj.xyz'}\nrandom-seed {w.seed_z}\n")
    (tmp_path / "run.mod").write_text(f"par N 1.0 0.0\nsteric {w.steric_r0} {w.steric_k0}\n")
    exe = os.path.join(ROOT, "stokesdt_b200", "bdrun")
    res = subprocess.run([exe, "--config", str(tmp_path / "run.cfg"), "--model", str(tmp_path / "run.mod"),
                          "--xyz", str(tmp_path / "start.xyz"), "-n", str(nsteps)], capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    start = sdt.read_xyz(tmp_path / "start.xyz")[0].reshape(-1)
    lines = (tmp_path / "traj.xyz").read_text().splitlines()
    assert len(lines) == nsteps * (N + 2)
    rng = np.random.default_rng(int(g["seed_proj"]))
    P = (rng.standard_normal((g["proj"].shape[1], n3), dtype=np.float32) / np.sqrt(n3)).astype(np.float64)
    for k in range(nsteps):
        frame = lines[k * (N + 2):(k + 1) * (N + 2)]
        assert int(frame[1].split()[0]) == k + 1
        pos = np.array([[float(v) for v in l.split()[1:4]] for l in frame[2:]]).reshape(-1)
        d = pos - start
        pk = P @ d
        assert np.linalg.norm(pk - g["proj"][k]) / np.linalg.norm(g["proj"][k]) < 1e-4, k
        assert abs(np.linalg.norm(d) / g["norms"][k] - 1.0) < 1e-4, k


def test_bdrun_dense_ewald_vs_reference_trajectory(gpu_available, tmp_path):
    """bdrun with `mob-method ewald` (the reference driver's default
    mobility, src/simbox/simbox_bd.cc:93-103; ewald-tol 1e-4) and Lanczos
    (4 RHS per interval, tol 1e-8) on N=304: its frames for steps 1..8
    against the FP64 trajectory of the reference's own MobEwald, BrwnLanczos
    and StericForce from the same random vectors
    (tests/golden/bd_ewald_traj.npz): 1e-6 relative per step."""
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl
    from conftest import golden
    g = golden("bd_ewald_traj")
    N, L = int(g["npos"]), float(g["box"])
    n3 = 3 * N
    nsteps = int(g["nsteps"])
    pos0 = wl.rsa_positions(N, L, int(g["seed_pos"]))
    sdt.write_xyz(tmp_path / "start.xyz", pos0, L)
    (tmp_path / "run.cfg").write_text(
        f"delta-t {float(g['dt'])!r}\nmob-method ewald\newald-tol {float(g['ewald_tol'])!r}\n"
        f"brownian-method lanczos\nmob-interval {int(g['interval'])}\nlanczos-maxiters {int(g['max_iters'])}\n"
        f"lanczos-maxnrhs {int(g['interval'])}\nlanczos-tol {float(g['lanczos_tol'])!r}\n"
        f"traj-startstep 0\ntraj-interval 1\ntraj-output {tmp_path / 'traj.xyz'}\nrandom-seed {int(g['seed_z'])}\n")
    (tmp_path / "run.mod").write_text(f"par N 1.0 0.0\nsteric {float(g['steric_r0'])} {float(g['steric_k0'])}\n")
    exe = os.path.join(ROOT, "stokesdt_b200", "bdrun")
    res = subprocess.run([exe, "--config", str(tmp_path / "run.cfg"), "--model", str(tmp_path / "run.mod"),
                          "--xyz", str(tmp_path / "start.xyz"), "-n", str(nsteps)], capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "dense Ewald" in res.stdout
    start = sdt.read_xyz(tmp_path / "start.xyz")[0].reshape(-1)
    lines = (tmp_path / "traj.xyz").read_text().splitlines()
    assert len(lines) == nsteps * (N + 2)
    for k in range(nsteps):
        frame = lines[k * (N + 2):(k + 1) * (N + 2)]
        assert int(frame[1].split()[0]) == k + 1
        pos = np.array([[float(v) for v in l.split()[1:4]] for l in frame[2:]]).reshape(-1)
        d = pos - start
        assert np.linalg.norm(d - g["d"][k]) / np.linalg.norm(g["d"][k]) < 1e-6, k
    assert n3 == g["d"].shape[1]
