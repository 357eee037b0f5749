"""Served request stream (sdt_serve_*): queued mobility applies and Brownian
steps on device-resident systems give the results of direct MobSpme /
BrwnLanczos calls; systems are admitted against the HBM budget."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _systems():
    from stokesdt_b200 import workloads as wl
    out = []
    for n, phi, seed in ((400, 0.2, 1), (900, 0.1, 2), (1500, 0.25, 3)):
        K, xi, rmax = wl.autotune_system(n, phi)
        L = wl.box_for(n, phi)
        out.append(dict(npos=n, box=L, K=K, xi=xi, rmax=rmax, pos=wl.rsa_positions(n, L, seed).reshape(-1)))
    return out


def test_requests_match_direct_calls(gpu_available):
    import stokesdt_b200 as sdt
    sy = _systems()
    srv = sdt.MobilityServer(hbm_budget_bytes=20e9, lanes=3, max_npos=2000, max_iters=100, max_nrhs=16,
                             tol=1e-6)
    ids = [srv.register(s["npos"], np.ones(s["npos"]), s["box"], s["K"], s["xi"], s["rmax"], 6, s["pos"])
           for s in sy]
    rng = np.random.default_rng(7)
    reqs = []
    for rep in range(3):
        for i, s in enumerate(sy):
            n3 = 3 * s["npos"]
            for kind, k in ((0, 1), (1, 4), (0, 16)):
                x = rng.standard_normal((k, n3))
                out = np.zeros((k, n3))
                reqs.append((i, kind, k, x, out, srv.submit(ids[i], kind, k, x, out)))
    lat = [srv.wait(t) for (_, _, _, _, _, t) in reqs]
    assert all(v > 0.0 for v in lat)
    assert srv.stats()["completed"] == len(reqs)
    direct = {}
    for i, s in enumerate(sy):
        m = sdt.MobSpme(s["npos"], np.ones(s["npos"]), s["box"], s["xi"], s["rmax"], s["K"], 6)
        assert m.Init()
        m.Update(s["pos"])
        lz = sdt.BrwnLanczos(3 * s["npos"], 100, 16, 1e-6, reorth=True)
        assert lz.Init()
        direct[i] = (m, lz)
    for i, kind, k, x, out, _ in reqs:
        m, lz = direct[i]
        n3 = 3 * sy[i]["npos"]
        ref = np.zeros((k, n3))
        if kind == 0:
            m.MulVector(k, 1.0, n3, x, 0.0, n3, ref)
            assert rel_err(ref, out) < 1e-6
        else:
            lz.Compute(m, k, n3, x, n3, ref)
            assert rel_err(ref, out) < 1e-5
    srv.close()


def test_admission_by_hbm_budget(gpu_available):
    import stokesdt_b200 as sdt
    sy = _systems()
    s = sy[0]
    assert s["K"] == 128 and sy[2]["K"] == 64
    srv = sdt.MobilityServer(hbm_budget_bytes=6.0e7, lanes=1, max_npos=2000, max_nrhs=4)
    # the small box needs a 128^3 grid (~117 MB with 4 RHS): not admitted in
    # 60 MB; the 1500-particle system on a 64^3 grid (~35 MB) is
    with pytest.raises(sdt.StokesError):
        srv.register(s["npos"], np.ones(s["npos"]), s["box"], s["K"], s["xi"], s["rmax"], 6, s["pos"])
    assert srv.stats()["rejected"] == 1
    s0 = sy[2]
    sid = srv.register(s0["npos"], np.ones(s0["npos"]), s0["box"], s0["K"], s0["xi"], s0["rmax"], 6, s0["pos"])
    x = np.ones((1, 3 * s0["npos"]))
    out = np.zeros_like(x)
    srv.wait(srv.submit(sid, 0, 1, x, out))
    assert np.all(np.isfinite(out)) and np.linalg.norm(out) > 0
    with pytest.raises(sdt.StokesError):
        srv.submit(sid, 0, 8, np.ones((8, 3 * s0["npos"])), np.zeros((8, 3 * s0["npos"])))  # > max_nrhs
    srv.close()


def test_mix_formed_while_a_batch_is_in_flight(gpu_available, monkeypatch):
    """Continuous batching (STOKESDT_SERVE_BATCH=all: every batchable request
    goes to the batch lanes, so the batch counts do not depend on thread
    timing): a Brownian batch (k = 16 on every system) is in flight when
    mobility applies on the same systems arrive; they wait for their systems
    and run together as later batches.  Every result equals the same request
    served alone on a fresh server in the default mode (1e-6 for M.f, 1e-5
    for sqrt(M) z), and the batches held more than one request each on
    average."""
    import stokesdt_b200 as sdt
    sy = _systems()

    def server():
        srv = sdt.MobilityServer(hbm_budget_bytes=20e9, lanes=2, max_npos=2000, max_iters=100, max_nrhs=16,
                                 tol=1e-6)
        ids = [srv.register(s["npos"], np.ones(s["npos"]), s["box"], s["K"], s["xi"], s["rmax"], 6, s["pos"])
               for s in sy]
        return srv, ids

    rng = np.random.default_rng(11)
    inputs = []
    for i, s in enumerate(sy):
        n3 = 3 * s["npos"]
        inputs.append((i, 1, 16, rng.standard_normal((16, n3))))
    for i, s in enumerate(sy):
        n3 = 3 * s["npos"]
        inputs.append((i, 0, 4, rng.standard_normal((4, n3))))
        inputs.append((i, 0, 1, rng.standard_normal((1, n3))))
    monkeypatch.setenv("STOKESDT_SERVE_BATCH", "all")
    srv, ids = server()
    monkeypatch.delenv("STOKESDT_SERVE_BATCH")
    outs, tickets = [], []
    for (i, kind, k, x) in inputs:
        out = np.zeros_like(x)
        outs.append(out)
        tickets.append(srv.submit(ids[i], kind, k, x, out))
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    assert st["completed"] == len(inputs)
    assert st["batch_lanes"] >= 1 and st["batches"] >= 1
    assert st["batched_requests"] == len(inputs) and st["batched_requests"] > st["batches"]
    srv.close()
    # each request alone
    for (i, kind, k, x), out in zip(inputs, outs):
        srv, ids = server()
        ref = np.zeros_like(x)
        srv.wait(srv.submit(ids[i], kind, k, x, ref))
        srv.close()
        assert rel_err(ref, out) < (1e-6 if kind == 0 else 1e-5), (i, kind, k)


def test_default_mode_routes_lone_and_batched_requests(gpu_available):
    """Default continuous batching: requests with a partner (same kind and k
    on another idle system) run as batches, lone ones on the per-request
    workers.  Whatever the split, every request completes once and equals
    the direct engine calls."""
    import stokesdt_b200 as sdt
    sy = _systems()
    srv = sdt.MobilityServer(hbm_budget_bytes=20e9, lanes=1, max_npos=2000, max_iters=100, max_nrhs=16, tol=1e-6)
    ids = [srv.register(s["npos"], np.ones(s["npos"]), s["box"], s["K"], s["xi"], s["rmax"], 6, s["pos"])
           for s in sy]
    rng = np.random.default_rng(5)
    reqs = []
    for rep in range(4):
        for i, s in enumerate(sy):
            n3 = 3 * s["npos"]
            kind, k = (1, 4) if rep % 2 else (0, 4)
            x = rng.standard_normal((k, n3))
            out = np.zeros((k, n3))
            reqs.append((i, kind, k, x, out, srv.submit(ids[i], kind, k, x, out)))
    for r in reqs:
        srv.wait(r[-1])
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["batched_requests"] <= len(reqs)
    srv.close()
    for i, s in enumerate(sy):
        m = sdt.MobSpme(s["npos"], np.ones(s["npos"]), s["box"], s["xi"], s["rmax"], s["K"], 6)
        assert m.Init()
        m.Update(s["pos"])
        lz = sdt.BrwnLanczos(3 * s["npos"], 100, 16, 1e-6, reorth=True)
        assert lz.Init()
        for (j, kind, k, x, out, _) in reqs:
            if j != i:
                continue
            n3 = 3 * s["npos"]
            ref = np.zeros((k, n3))
            if kind == 0:
                m.MulVector(k, 1.0, n3, x, 0.0, n3, ref)
                assert rel_err(ref, out) < 1e-6
            else:
                lz.Compute(m, k, n3, x, n3, ref)
                assert rel_err(ref, out) < 1e-5
