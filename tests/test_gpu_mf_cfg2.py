"""Mobility product at the headline size (config 2: N = 100,000 spheres, phi
= 0.2, 256^3 grid, p = 6, xi = 0.35, rmax from the tol-1e-6 rule) against the
reference's own FP64 MobSpme (MulVector / RealMulVector / RecipMulVector,
src/mob/mob_spme.cc:219-263, src/mob/spme.cc:714-839 of the reference) on the
same positions and forces.

The fixture (tests/golden/mf_cfg2_proj.npz, made by
``tests/golden/make_golden.py --mf-cfg2`` with the compiled reference) holds,
for each mode and each of 4 RHS with alpha = 1.3 and beta = 0.7, 64 fixed
random projections of the output, its norm and the outputs of the first 512
particles in full.  The GPU product runs at the benchmark's exact parameters
through both spreads: 16 RHS in one call (the tcgen05 tensor-core spread
takes calls of >= 8 RHS) and single-RHS calls (shared-memory spread).

Bar: relative Frobenius error <= 1e-6 (the M.f bound) on the projections and
on the first 512 particles, and each output norm within 1e-6."""
import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-6


@pytest.fixture(scope="module")
def cfg2():
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import cfg2_projector, mf_cfg2_inputs
    g = golden("mf_cfg2_proj")
    w = wl.WORKLOADS["cfg2"]
    N, n3 = w.npos, 3 * w.npos
    pos = wl.rsa_positions(N, w.box, w.seed_pos)
    F, V0 = mf_cfg2_inputs(n3)
    m = sdt.MobSpme(N, np.ones(N), w.box, w.xi, w.rmax, w.dim, w.porder)
    assert m.Init(), m.last_error
    m.Update(pos)
    P = cfg2_projector(n3, seed=int(g["seed_proj"])).astype(np.float64)
    return m, g, F, V0, P, n3


def _check(g, mode, V, P, head):
    proj = (P @ V.T).T
    assert rel_err(g[f"proj{mode}"], proj) < TOL, (mode, rel_err(g[f"proj{mode}"], proj))
    h = g[f"head{mode}"]
    assert rel_err(h, V[:, :3 * head]) < TOL, (mode, rel_err(h, V[:, :3 * head]))
    ratio = np.linalg.norm(V, axis=1) / g[f"norms{mode}"]
    assert np.max(np.abs(ratio - 1.0)) < TOL, (mode, ratio)


def _methods(m):
    return {0: m.MulVector, 1: m.RealMulVector, 2: m.RecipMulVector}


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_cfg2_mulvec_16rhs_tensor_core_spread(gpu_available, cfg2, mode):
    """16 RHS in one call (the forces of the fixture's 4 RHS, each 4 times):
    the tcgen05 spread at the benchmark's RHS count."""
    m, g, F, V0, P, n3 = cfg2
    a, b = float(g["alpha"]), float(g["beta"])
    nr = 16
    f = np.ascontiguousarray(np.tile(F, (4, 1)))
    v = np.ascontiguousarray(np.tile(V0, (4, 1)))
    _methods(m)[mode](nr, a, n3, f, b, n3, v)
    for rep in range(4):
        _check(g, mode, v[4 * rep:4 * rep + 4], P, int(g["head"]))


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_cfg2_mulvec_single_rhs_shared_memory_spread(gpu_available, cfg2, mode):
    """One RHS per call (the BD steps' M.F products): the shared-memory spread."""
    m, g, F, V0, P, n3 = cfg2
    a, b = float(g["alpha"]), float(g["beta"])
    V = V0.copy()
    for j in range(F.shape[0]):
        _methods(m)[mode](1, a, n3, np.ascontiguousarray(F[j]), b, n3, V[j])
    _check(g, mode, V, P, int(g["head"]))
