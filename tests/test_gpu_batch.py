"""Batched independent systems (sdt_batch_*): every system's product and
Brownian vectors equal those of a single-system engine with the same
parameters (MobSpme / BrwnLanczos through the C ABI) and, for one system,
the FP64 oracle.  Tolerances: 1e-6 (M.f), 1e-5 (sqrt(M) z)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _batch(nsys=6, seed=8, lanes=3):
    from stokesdt_b200 import workloads as wl
    sy = wl.batch_systems(nsys=nsys, seed=seed, nmin=300, nmax=3000)
    pos = [wl.rsa_positions(s["npos"], s["box"], s["seed"]).reshape(-1) for s in sy]
    return sy, pos


def test_batch_matches_single_systems(gpu_available):
    import stokesdt_b200 as sdt
    sy, pos = _batch()
    npos = [s["npos"] for s in sy]
    rdi = np.ones(sum(npos))
    b = sdt.MobSpmeBatch(npos, rdi, [s["box"] for s in sy], [s["K"] for s in sy], [s["xi"] for s in sy],
                         [s["rmax"] for s in sy], porder=6, max_iters=100, max_nrhs=4, tol=1e-6, lanes=3)
    b.Update(np.concatenate(pos))
    tot = int(b.offsets[-1])
    rng = np.random.default_rng(1)
    nr = 2
    F = rng.standard_normal(nr * tot)
    V = np.zeros(nr * tot)
    b.MulVector(nr, 1.0, F, 0.0, V)
    Z = rng.standard_normal(4 * tot)
    Y = np.zeros(4 * tot)
    its = b.Lanczos(4, Z, Y)
    assert all(i > 0 for i in its)
    for s, (sysd, p) in enumerate(zip(sy, pos)):
        N, n3 = sysd["npos"], 3 * sysd["npos"]
        m = sdt.MobSpme(N, np.ones(N), sysd["box"], sysd["xi"], sysd["rmax"], sysd["K"], 6)
        assert m.Init()
        m.Update(p)
        f = b.split(F, nr)[s]
        v = np.zeros((nr, n3))
        m.MulVector(nr, 1.0, n3, np.ascontiguousarray(f), 0.0, n3, v)
        assert rel_err(v, b.split(V, nr)[s]) < 1e-6, s
        lz = sdt.BrwnLanczos(n3, 100, 4, 1e-6, reorth=True)
        assert lz.Init()
        y = np.zeros((4, n3))
        lz.Compute(m, 4, n3, np.ascontiguousarray(b.split(Z, 4)[s]), n3, y)
        assert rel_err(y, b.split(Y, 4)[s]) < 1e-5, s


def test_batch_device_api_and_oracle(gpu_available):
    import torch
    import stokesdt_b200 as sdt
    from oracle import spme_oracle as so
    sy, pos = _batch(nsys=3, seed=2)
    npos = [s["npos"] for s in sy]
    b = sdt.MobSpmeBatch(npos, np.ones(sum(npos)), [s["box"] for s in sy], [s["K"] for s in sy],
                         [s["xi"] for s in sy], [s["rmax"] for s in sy], lanes=2, max_nrhs=4)
    dpos = torch.tensor(np.concatenate(pos), device="cuda")
    b.update_device(dpos.data_ptr())
    tot = int(b.offsets[-1])
    F = np.random.default_rng(4).standard_normal(tot)
    dF = torch.tensor(F, device="cuda")
    dV = torch.zeros(tot, dtype=torch.float64, device="cuda")
    b.mulvec_device(1, 1.0, dF.data_ptr(), 0.0, dV.data_ptr())
    b.synchronize()
    V = dV.cpu().numpy()
    s = 0
    o = so.SpmeOracle(np.ones(npos[s]), sy[s]["box"], sy[s]["xi"], sy[s]["rmax"], sy[s]["K"], 6)
    o.update(pos[s].reshape(-1, 3))
    vo = o.mulvec(b.split(F, 1)[s])
    assert rel_err(vo, b.split(V, 1)[s]) < 1e-6


def test_batch_rejects_bad_systems(gpu_available):
    import stokesdt_b200 as sdt
    with pytest.raises(sdt.StokesError):
        # rmax >= L/2 for the second system
        sdt.MobSpmeBatch([100, 100], np.ones(200), [20.0, 20.0], [32, 32], [0.5, 0.5], [8.0, 12.0])


def _make(sy, **kw):
    import stokesdt_b200 as sdt
    npos = [s["npos"] for s in sy]
    args = dict(porder=6, max_iters=100, max_nrhs=4, tol=1e-6, lanes=3)
    args.update(kw)
    return sdt.MobSpmeBatch(npos, np.ones(sum(npos)), [s["box"] for s in sy], [s["K"] for s in sy],
                            [s["xi"] for s in sy], [s["rmax"] for s in sy], **args)


def test_packed_batch_product_vs_reference(gpu_available):
    """The packed product (one launch sequence over all systems) against the
    reference's own MobSpme MulVector on every system of a 6-system batch
    (tests/golden/batch_sys6.npz; alpha 0.8, beta 0.5, 3 RHS): 1e-6."""
    from conftest import golden
    from stokesdt_b200 import workloads as wl
    g = golden("batch_sys6")
    sy = wl.batch_systems(nsys=6, seed=8, nmin=300, nmax=3000)
    b = _make(sy)
    assert b.packed
    b.Update(np.concatenate([wl.rsa_positions(s["npos"], s["box"], s["seed"]).reshape(-1) for s in sy]))
    nr = 3
    F = np.concatenate([g[f"f{s}"].reshape(-1) for s in range(len(sy))])
    V = np.concatenate([g[f"v0_{s}"].reshape(-1) for s in range(len(sy))])
    b.MulVector(nr, float(g["alpha"]), F, float(g["beta"]), V)
    for s in range(len(sy)):
        assert rel_err(g[f"v{s}"], b.split(V, nr)[s]) < 1e-6, s


def test_packed_and_lanes_agree_on_mixed_grids(gpu_available):
    """Systems with 64^3 and 128^3 grids (two grid classes of the packed
    launches): packed products and packed lockstep block Lanczos equal the
    per-system launches of the lanes mode (1e-6 for M.f, 1e-5 for
    sqrt(M) z), with the same iteration counts to within 2."""
    from stokesdt_b200 import workloads as wl
    sy = wl.batch_systems(nsys=8, seed=7, nmin=500, nmax=6000)
    assert len({s["K"] for s in sy}) == 2
    pos = np.concatenate([wl.rsa_positions(s["npos"], s["box"], s["seed"]).reshape(-1) for s in sy])
    b = _make(sy)
    assert b.packed
    tot = int(b.offsets[-1])
    rng = np.random.default_rng(3)
    F = rng.standard_normal(2 * tot)
    V0 = rng.standard_normal(2 * tot)
    Z = rng.standard_normal(4 * tot)
    out = {}
    for packed in (True, False):
        b.set_packed(packed)
        assert b.packed == packed
        b.Update(pos)
        V = V0.copy()
        b.MulVector(2, 1.1, F, -0.3, V)
        Y = np.zeros(4 * tot)
        its = b.Lanczos(4, Z, Y)
        out[packed] = (V, Y, its)
    Vp, Yp, itp = out[True]
    Vl, Yl, itl = out[False]
    assert all(i > 0 for i in itp) and all(i > 0 for i in itl)
    for s in range(len(sy)):
        assert rel_err(b.split(Vl, 2)[s], b.split(Vp, 2)[s]) < 1e-6, s
        assert rel_err(b.split(Yl, 4)[s], b.split(Yp, 4)[s]) < 1e-5, s
        assert abs(itp[s] - itl[s]) <= 2, (s, itp[s], itl[s])
